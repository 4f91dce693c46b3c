"""Generate tests/golden/fixtures.npz and tests/golden/golden_counts.json.

Run in a container that has the reference checkout (read-only) at
/root/reference:

    python tests/golden/make_fixtures.py [/path/to/neighborlist-rs]

* Positions and cells are parsed from the reference's fixture files
  (tests/data/*.xyz, written by the reference's tests/generate_data.py with
  np.random.default_rng(42)).  The extxyz ``Lattice=`` header lists the
  lattice vectors as rows (ASE convention), stored here as ``<name>_cell``
  (rows = lattice vectors, zeros for the isolated files).
* Golden counts are the "Total Edges RS" numbers (edges with i != j) that the
  reference's benchmark printed for each fixture and cutoff, copied from
  benchmarks/benchmark_grace.txt (lines 7-47 rc 6, 58-98 rc 14, 109-149 rc 30).

Nothing under tests/ reads the reference at run time; the GPU box only sees
the files this script writes.
"""

from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Fixtures small enough to keep in the repository.
KEEP = [
    "isolated_100",
    "isolated_two_clusters",
    "isolated_1000",
    "isolated_10000",
    "ethanol_1000",
    "ethanol_10000",
    "si_bulk",
]

NAME_OF_LABEL = {
    "100 (non-PBC)": "isolated_100",
    "Two Clusters (non-PBC)": "isolated_two_clusters",
    "1,000 (non-PBC)": "isolated_1000",
    "10,000 (non-PBC)": "isolated_10000",
    "20,000 (non-PBC)": "isolated_20000",
    "1,000 (Ethanol PBC)": "ethanol_1000",
    "10,000 (Ethanol PBC)": "ethanol_10000",
    "20,000 (Ethanol PBC)": "ethanol_20000",
    "Si Bulk (PBC)": "si_bulk",
}


def read_xyz(path):
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[0].strip())
    header = lines[1]
    pos = np.array([[float(x) for x in ln.split()[1:4]] for ln in lines[2 : 2 + n]],
                   dtype=np.float64)
    cell = np.zeros((3, 3), dtype=np.float64)
    m = re.search(r'Lattice="([^"]+)"', header)
    if m:
        cell = np.array([float(x) for x in m.group(1).split()], dtype=np.float64).reshape(3, 3)
    return pos, cell


def parse_counts(path):
    counts: dict[str, dict[str, int]] = {}
    cutoff = None
    pat = re.compile(r"Correctness: PASSED for (.+) \(Cutoff ([0-9.]+)\) - Unique Pairs V:(\d+) "
                     r"RS:(\d+) \| Total Edges V:(\d+) RS:(\d+)")
    with open(path) as f:
        for line in f:
            m = pat.search(line)
            if not m:
                continue
            label, rc = m.group(1), m.group(2)
            name = NAME_OF_LABEL[label]
            counts.setdefault(rc, {})[name] = {
                "edges_i_ne_j": int(m.group(6)),
                "unique_pairs": int(m.group(4)),
            }
            cutoff = rc
    assert cutoff is not None
    return counts


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    arrays = {}
    for name in KEEP:
        pos, cell = read_xyz(os.path.join(ref, "tests", "data", f"{name}.xyz"))
        arrays[f"{name}_pos"] = pos
        arrays[f"{name}_cell"] = cell
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **arrays)
    counts = parse_counts(os.path.join(ref, "benchmarks", "benchmark_grace.txt"))
    with open(os.path.join(HERE, "golden_counts.json"), "w") as f:
        json.dump({"source": "benchmarks/benchmark_grace.txt (Total Edges RS, i != j)",
                   "counts": counts}, f, indent=1, sort_keys=True)
    print("wrote", sorted(arrays), "and counts for cutoffs", sorted(counts))


if __name__ == "__main__":
    main()

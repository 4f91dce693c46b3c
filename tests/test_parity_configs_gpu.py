"""Parity at the configured sizes, against the CPU oracle:

* the full uneven batch (4096 systems, N uniform in [8, 256], half isolated,
  half triclinic PBC with boxes often smaller than 2 rc, rc 5), single cutoff
  with the per-system offset table, and multi-cutoff (plain and disjoint);
* a served stream drawn from the full request distribution (N log-uniform up
  to 1e6 atoms; 70 % orthorhombic, 20 % triclinic, 10 % isolated; rc in
  {5, 6, 8}) with every result, host-resident or device-resident, compared
  with the oracle.
"""

import numpy as np
import pytest

from helpers import assert_same

pytestmark = pytest.mark.gpu

PBC3 = [True, True, True]


@pytest.fixture(scope="module")
def nl():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs
    import neighborlist_rs.serving  # noqa: F401

    return neighborlist_rs


def per_system_counts(ei, batch, n_systems):
    """Edges per system of a concatenated list (sources are global atom ids)."""
    return np.bincount(batch[ei[0]], minlength=n_systems) if ei.shape[1] else \
        np.zeros(n_systems, np.int64)


def test_uneven_batch_4096_matches_oracle(nl, oracle):
    from neighborlist_rs import workloads as W

    systems = W.uneven_batch()
    assert len(systems) == 4096
    pos, batch, cells = W.concat_batch(systems)
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=16)
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0,
                                       return_offsets=True)
    assert_same(got, ref, "4096-system batch, rc 5")
    off = got["system_offsets"]
    want = np.concatenate([[0], np.cumsum(per_system_counts(ref[0], batch, 4096))])
    assert np.array_equal(off, want)
    # the same call again (steady state: tuned shape, reused buffers)
    again = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    assert_same(again, ref, "4096-system batch, second call")


@pytest.mark.parametrize("disjoint", [False, True])
def test_uneven_batch_4096_multi_matches_oracle(nl, oracle, disjoint):
    from neighborlist_rs import workloads as W

    pos, batch, cells = W.concat_batch(W.uneven_batch())
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    cutoffs = [5.0, 3.0, 4.0]
    ref = oracle.search_batch(pos, batch, ocells, cutoffs, disjoint=disjoint, nthreads=16)
    got = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=cutoffs,
                                             disjoint=disjoint, return_offsets=True)
    for q, rc in enumerate(cutoffs):
        assert_same(got[q], ref[q], f"4096-system batch, rc {rc}, disjoint={disjoint}")
        want = np.concatenate([[0], np.cumsum(per_system_counts(ref[q][0], batch, 4096))])
        assert np.array_equal(got[q]["system_offsets"], want)


def full_range_stream():
    """36 requests of the served distribution, with at least two above 1e5
    atoms (one of each periodic kind) so the single-system pipeline and the
    batched kernels both serve them."""
    from neighborlist_rs import workloads as W

    reqs = W.request_stream(32, seed=23, max_atoms=400_000)
    rng = np.random.default_rng(24)
    for n, kind, rc in [(150_000, "ortho", 8.0), (120_000, "tri", 6.0),
                        (100_000, "iso", 5.0), (262_144, "ortho", 5.0)]:
        if kind == "iso":
            side = (n / 0.1) ** (1.0 / 3.0)
            reqs.append(W.System(rng.random((n, 3)) * side, None, rc))
        else:
            rows = W.density_cell(n, 0.1, rng, (75.0, 105.0), ortho=kind == "ortho")
            reqs.append(W.System(rng.random((n, 3)) @ rows, rows, rc))
    return reqs


@pytest.mark.parametrize("device_result", [False, True])
def test_served_full_range_matches_oracle(nl, oracle, device_result):
    import torch

    from neighborlist_rs.serving import Server

    reqs = full_range_stream()
    assert max(s.positions.shape[0] for s in reqs) >= 100_000
    with Server(hbm_budget_bytes=40 << 30, workers=4, max_batch=4096) as srv:
        tickets = [srv.submit(None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist()),
                              s.positions, s.cutoff, device_result=device_result)
                   for s in reqs]
        for i, (s, t) in enumerate(zip(reqs, tickets)):
            got = srv.wait(t, timeout=300.0)
            if device_result:
                dev = got.to_torch()
                torch.cuda.synchronize()
                got.release()
                got = {"edge_index": dev["edge_index"].cpu().numpy(),
                       "shift": dev["shift"].cpu().numpy()}
                del dev
            h = None if s.cell_rows is None else s.cell_rows.T
            pbc = None if s.cell_rows is None else PBC3
            ref = oracle.search_single(s.positions, h, pbc, s.cutoff, nthreads=16)
            assert_same(got, ref, f"request {i} (n={s.positions.shape[0]}, rc={s.cutoff}, "
                                  f"device={device_result})")
            del got
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0

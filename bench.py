"""Benchmark of the B200 neighbour-list engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Headline workload: the periodic cluster liquid (1112 rigid 9-atom clusters,
N = 10,008, cubic L = 46.4 A, full PBC) at rc = 6 A; one step = one complete
neighbour-list build of that system (cell list build, count, scan, emit of the
exact-sized edge_index int64 (2, M) and shift int32 (M, 3)).

* value      : edges/s over all ranks, device-resident: positions already in
               HBM, edge arrays left in HBM (nlb_build_device); CUDA events on
               the launching stream around each step; L2 flushed (256 MB write)
               between steps, outside the timed spans.
* e2e        : same metric through the reference-facing call with host buffers
               (neighborlist_rs.build_neighborlists: numpy positions in, numpy
               edge arrays out), host<->device copies inside the timed region.
* roofline   : the dominant kernel's algorithmic bytes / its CUDA-event time
               (the one-launch search on the headline's sparse grid; the emit
               pass, with the count pass beside it, on grids that keep the
               three launches).
* cpu_baseline: the CPU oracle (C++ restatement of the reference's rayon
               count/fill path) on the host cores, rank 0, bounded sample.
* extra      : other configurations (rc 14, isolated N=1000, triclinic
               multi-cutoff, batched uneven systems) measured the same way.

Multi-GPU: systems are independent, so each rank builds its own copy of the
workload (weak scaling, no collective on the data path); the step time is the
max over ranks.  `--impl reference` times the CPU oracle on all host threads
(rank 0 only).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "neighborlist-rs_b200")
for _p in (ROOT, PKG_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "edges/s (exact edges; cluster-liquid N=10008 PBC rc=6)"
UNIT = "edges/s"
WORKLOAD = "cluster_liquid N=10008 (1112 x 9-atom clusters) cubic L=46.4 A full PBC rc=6.0 A"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-extra", action="store_true", help="headline workload only")
    ap.add_argument("--rc", type=float, default=6.0,
                    help="cutoff of the timed workload (6.0 = headline; 14.0 for profiling)")
    ap.add_argument("--case", default=None, choices=sorted(CASES),
                    help="run only this workload --steps times after --warmup (for profilers; "
                         "prints one summary line, not the bench JSON)")
    return ap.parse_args()


def _case_device(rc):
    def run(nl, torch, steps, warmup):
        pos, rows = headline_system()
        dt = DeviceTimer(nl, torch, pos, rows, rc)
        ms, edges, launches = dt.run(steps, warmup)
        return {"edges_per_step": edges // steps, "ms_per_step": ms / steps, "launches": launches}
    return run


def settle_batch_tuner(nl, fn, limit=64):
    """Calls fn() until the launch-shape tuner has chosen a shape for every
    kind of batch fn issues (the batched path's steady state); returns the
    chosen shapes."""
    for _ in range(limit):
        fn()
        state = nl.batch_tuner_state()
        if state and all(e["shape"] >= 0 for e in state):
            break
    return [dict(e, **nl.batch_shape_info(e["shape"])) for e in nl.batch_tuner_state()
            if e["shape"] >= 0]


def _case_batch(nl, torch, steps, warmup):
    W = workloads()

    pb, bb, cb = W.concat_batch(W.uneven_batch())
    settle_batch_tuner(nl, lambda: nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0))
    for _ in range(warmup):
        nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0)
    t0 = time.perf_counter()
    for _ in range(steps):
        r = nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0)
    return {"edges": int(r["edge_index"].shape[1]), "ms_per_call": 1e3 * (time.perf_counter() - t0) / steps}


def _case_served(nl, torch, steps, warmup):
    W = workloads()
    from neighborlist_rs.serving import Server

    reqs = [(None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist()), s.positions,
             s.cutoff) for s in W.request_stream(1024, seed=21, n_range=(16, 2048))]
    with Server(hbm_budget_bytes=40 << 30, workers=2) as srv:
        for _ in range(warmup):
            run_stream_raw(srv, reqs)
        for _ in range(steps):
            r = run_stream_raw(srv, reqs)
    return r


def _case_multi(nl, torch, steps, warmup):
    W = workloads()

    p3, r3 = W.triclinic_uniform()
    cell = nl.PyCell(r3.T.tolist())
    for _ in range(warmup):
        nl.build_neighborlists_multi(cell, p3, [5.0, 6.0, 12.0])
    t0 = time.perf_counter()
    for _ in range(steps):
        r = nl.build_neighborlists_multi(cell, p3, [5.0, 6.0, 12.0])
    return {"edges": sum(int(v["edge_index"].shape[1]) for v in r.values()),
            "ms_per_call": 1e3 * (time.perf_counter() - t0) / steps}


def _case_every_kernel(nl, torch, steps, warmup):
    """Each kernel of the library on a modest workload, `steps` rounds after
    `warmup` rounds (for an ncu capture of every kernel): the headline build
    in both single-system pipelines, rc 14 (chunk boxes), an isolated
    device-resident build (auto-box bounds), a 512-system batch (plan, count
    with records, expansion), the output options (directed list, vectors,
    distances) and Verlet updates."""
    W = workloads()
    from neighborlist_rs.verlet import VerletList

    pos, rows = headline_system()
    cell = nl.PyCell(rows.T.tolist())
    d = torch.from_numpy(pos).cuda()
    iso = torch.from_numpy(W.isolated_cube()).cuda()
    pb, bb, cb = W.concat_batch(W.uneven_batch(n_systems=512, seed=71))
    vl = VerletList(6.0, 1.0)
    moved = d + 0.01

    def one_round():
        nl.build_neighborlists_torch(cell, d, 6.0)
        nl.set_single_pipeline(1)
        nl.build_neighborlists_torch(cell, d, 6.0)
        nl.set_single_pipeline(0)
        nl.build_neighborlists_torch(cell, d, 14.0)
        nl.build_neighborlists_torch(None, iso, 6.0)
        nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0)
        nl.build_neighborlists_torch(cell, d, 6.0, directed=True, vectors=True, distances=True)
        vl.update(cell, d)
        vl.update(cell, moved)
        torch.cuda.synchronize()

    for _ in range(warmup):
        one_round()
    t0 = time.perf_counter()
    for _ in range(steps):
        one_round()
    vl.close()
    return {"rounds": steps, "ms_per_round": 1e3 * (time.perf_counter() - t0) / max(steps, 1)}


CASES = {
    "every_kernel": _case_every_kernel,
    "cluster_liquid_rc6": _case_device(6.0),
    "cluster_liquid_rc14": _case_device(14.0),
    "uneven_batch_4096": _case_batch,
    "served_small_mix_1024": _case_served,
    "triclinic_multi_20k": _case_multi,
}


def run_case(args):
    import torch

    import neighborlist_rs as nl

    out = CASES[args.case](nl, torch, args.steps, args.warmup)
    print(json.dumps({"case": args.case, **out}), flush=True)


# ---------------------------------------------------------------- distributed

def dist_init(backend):
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and not dist.is_initialized():
        import datetime

        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, local, world


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (every 100 ms) while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- workloads

_WORKLOADS = None


def workloads():
    """The seeded workload generators (neighborlist_rs/workloads.py), loaded
    from their file so that the CPU reference arm never imports the
    neighborlist_rs package (whose import maps the CUDA library)."""
    global _WORKLOADS
    if _WORKLOADS is None:
        import importlib.util

        path = os.path.join(PKG_DIR, "neighborlist_rs", "workloads.py")
        spec = importlib.util.spec_from_file_location("nlb_bench_workloads", path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = mod  # dataclasses resolve their module by name
        spec.loader.exec_module(mod)
        _WORKLOADS = mod
    return _WORKLOADS


def headline_system():
    W = workloads()

    pos, rows = W.cluster_liquid()
    return pos, rows


def ncu_traffic(rc, pass_name):
    """DRAM bytes (read + write) per launch of the pair-task pass at cutoff rc,
    and the capture they come from, from the committed ncu traffic table
    (profiles/ncu_traffic.txt); (None, None) when it has no such row."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if not parts or parts[0].startswith("#") or len(parts) < 5:
                    continue
                if parts[0] == pass_name and float(parts[1]) == float(rc):
                    return float(parts[2]) + float(parts[3]), parts[4]
    except (OSError, ValueError):
        pass
    return None, None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------- device timing

class DeviceTimer:
    """Times device-resident builds of one system with CUDA events on the
    stream the library launches on; L2 flushed between steps."""

    def __init__(self, nl, torch, pos, rows, rc):
        self.nl, self.torch = nl, torch
        self.cell = None if rows is None else nl.PyCell(rows.T.tolist())
        self.dpos = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
        self.n = pos.shape[0]
        self.rc = rc
        self.flush = torch.empty(256 << 20, dtype=torch.int8, device="cuda")
        # A dedicated (non-default) stream: the library launches on it and the
        # timing events are recorded on it.
        self.stream = torch.cuda.Stream()
        nl.set_stream(self.stream.cuda_stream)

    def step(self):
        return self.nl.build_device_raw(self.cell, self.dpos.data_ptr(), self.n, self.rc)[0]

    def run(self, steps, warmup):
        torch = self.torch
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        edges = 0
        l0 = self.nl.kernel_launches()
        for k in range(steps):
            with torch.cuda.stream(self.stream):
                self.flush.zero_()
            starts[k].record(self.stream)
            edges += self.step()
            ends[k].record(self.stream)
        torch.cuda.synchronize()
        launches = self.nl.kernel_launches() - l0
        ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        self.nl.set_stream(self.stream.cuda_stream)
        return ms, edges, launches

    def sustain(self, seconds):
        """Back-to-back builds for `seconds` of wall time (untimed): keeps the
        GPU under the same load while the clock sampler records."""
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < seconds:
            self.step()
            k += 1
            if k % 64 == 0:
                self.torch.cuda.synchronize()
        self.torch.cuda.synchronize()
        return k

    def phases(self, steps):
        self.nl.profile(True)
        for _ in range(steps):
            with self.torch.cuda.stream(self.stream):
                self.flush.zero_()
            self.step()
        self.torch.cuda.synchronize()
        calls, ph = self.nl.profile_read()
        self.nl.profile(False)
        return {k: v / max(calls, 1) for k, v in ph.items()}


def e2e_time(nl, pos, rows, rc, steps, warmup):
    cell = None if rows is None else nl.PyCell(rows.T.tolist())
    for _ in range(warmup):
        nl.build_neighborlists(cell, pos, rc)
    t = 0.0
    m = 0
    for _ in range(steps):
        t0 = time.perf_counter()
        r = nl.build_neighborlists(cell, pos, rc)
        t += time.perf_counter() - t0
        m = r["edge_index"].shape[1]
        del r
    return t, m


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_oracle_time(pos, rows, rc, budget_s=4.0, min_reps=15, threads=None):
    import oracle

    threads = threads or (os.cpu_count() or 1)
    h = None if rows is None else rows.T
    pbc = None if rows is None else [True] * 3
    for _ in range(2):
        ei, _ = oracle.search_single(pos, h, pbc, rc, nthreads=threads)
    times = []
    t_start = time.perf_counter()
    while len(times) < min_reps or time.perf_counter() - t_start < budget_s:
        t0 = time.perf_counter()
        ei, _ = oracle.search_single(pos, h, pbc, rc, nthreads=threads)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > 3 * budget_s:
            break
    return statistics.mean(times), ei.shape[1], threads, len(times)


# ---------------------------------------------------------------- arms

def bench_config(workload, atoms, edges_per_step):
    """The `config` dict both arms print (identical for the same workload)."""
    return {"workload": workload, "atoms": atoms, "edges_per_step": edges_per_step,
            "l2": "flushed between steps (256 MB write)"}


def run_reference(args):
    rank, _, world = dist_init("gloo")
    if rank != 0:
        return
    pos, rows = headline_system()
    import oracle

    threads = os.cpu_count() or 1
    h, pbc = rows.T, [True] * 3
    for _ in range(args.warmup):
        oracle.search_single(pos, h, pbc, args.rc, nthreads=threads)
    # Host caches are flushed between steps like the GPU arm's L2: a 256 MB
    # write outside the timed spans.
    flush = np.empty(256 << 20, np.uint8)
    t = 0.0
    m = 0
    for _ in range(args.steps):
        flush.fill(1)
        t0 = time.perf_counter()
        ei, _ = oracle.search_single(pos, h, pbc, args.rc, nthreads=threads)
        t += time.perf_counter() - t0
        m = ei.shape[1]
    value = m * args.steps / t
    metric, workload = METRIC, WORKLOAD
    if args.rc != 6.0:
        metric = METRIC.replace("rc=6", f"rc={args.rc:g}")
        workload = WORKLOAD.replace("rc=6.0", f"rc={args.rc:g}")
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cluster liquid)",
        "config": bench_config(workload, int(pos.shape[0]), m),
        "parallelism": f"{threads} host threads (rank 0 only)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full builds of the workload (C++ restatement "
                                   "of the reference rayon count/fill path; the Rust crate "
                                   "cannot be built here)",
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch

    rank, local, world = dist_init("nccl")
    torch.cuda.set_device(local)
    import neighborlist_rs as nl

    pos, rows = headline_system()
    n = pos.shape[0]
    dt = DeviceTimer(nl, torch, pos, rows, args.rc)
    barrier(world)
    torch.cuda.synchronize()
    # The timed steps last a few ms, far shorter than the sampler's period: the
    # sampled window is the timed steps plus 1.5 s of the same builds back to
    # back right after them.
    with ClockSampler(local) as clk:
        ms, edges, launches = dt.run(args.steps, args.warmup)
        sustained = dt.sustain(1.5)
    torch.cuda.synchronize()
    barrier(world)
    ms_max = max_over_ranks(ms, world, "cuda")
    m_step = edges // args.steps
    value = edges * world / (ms_max * 1e-3)

    # per-phase CUDA-event times -> roofline of the dominant kernel
    ph = dt.phases(max(5, args.steps // 3))
    peak, peak_kind = peaks()
    # Algorithmic bytes per launch: the emit (or the one-launch kernel) writes
    # the 28 B/edge output and reads the sorted SoA (positions, FP32
    # coordinates, meta) once; the count pass of the three-launch pipeline
    # reads the sorted FP32 coordinates and writes one count per (atom,
    # stencil cell).
    cells = 27  # stencil cells of this grid (n_search = 1 on every axis)
    bytes_emit = 28 * m_step + 48 * n
    bytes_count = 16 * n + 4 * cells * n
    fused = nl.last_single_pipeline() == 0  # one-launch pipeline (sparse grids)
    dominant = "emit"
    alg = bytes_emit
    achieved = alg / (ph[dominant] * 1e-3) / 1e9
    # DRAM bytes (read + write) per launch of the same kernel on the same
    # workload, from an ncu capture (not measured by this run).
    traffic, capture = ncu_traffic(args.rc, "fused" if fused else dominant)
    count_traffic, _ = ncu_traffic(args.rc, "count")
    if fused:
        kernel_name = ("k_pair_fused (count, offsets by look-back over groups, emit and the move "
                       "of the destinations behind the sources: one launch)")
        second = {"note": "no separate count pass or offsets scan: both are inside k_pair_fused"}
    else:
        # The emit pass has the largest share of the ncu launch list; the
        # count pass, within a few us of it in live timing and issue-bound,
        # is reported beside it.
        kernel_name = "k_pair_tasks<1> (emit pass)"
        second = {"kernel": "k_pair_tasks<0> (count pass)",
                  "bound": "instruction issue (61-78 % issue-active in ncu)",
                  "algorithmic_bytes": bytes_count, "kernel_ms": ph["count"],
                  "achieved_gbs": bytes_count / (ph["count"] * 1e-3) / 1e9,
                  "traffic": count_traffic}
    step_bytes = 24 * n + 72 + 28 * m_step

    # e2e through the reference-facing call (host buffers)
    nl.set_stream(None)
    t_e2e, m_e2e = e2e_time(nl, pos, rows, args.rc, args.steps, args.warmup)
    e2e_value = m_e2e * args.steps * world / max_over_ranks(t_e2e, world, "cuda")

    metric, workload = METRIC, WORKLOAD
    if args.rc != 6.0:
        metric = METRIC.replace("rc=6", f"rc={args.rc:g}")
        workload = WORKLOAD.replace("rc=6.0", f"rc={args.rc:g}")
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cluster liquid)",
        "config": bench_config(workload, n, m_step),
        "parallelism": f"replicas x{world} (independent systems)",
        "gpu_launches": launches,
        "clocks": dict(clk.summary(), window=f"timed steps + {sustained} back-to-back builds "
                                               "(1.5 s) of the same workload"),
        "roofline": {"bound": "hbm", "kernel": kernel_name, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": alg, "kernel_ms": ph[dominant], "traffic": traffic,
                     "traffic_source": f"ncu capture {capture} (committed traffic table)"
                     if traffic is not None else None,
                     "phases_ms": ph, "pipeline": "one launch" if fused else "three launches",
                     "count_pass": second,
                     "whole_step": {"algorithmic_bytes": step_bytes,
                                    "ms": ms_max / args.steps,
                                    "achieved_gbs": step_bytes / (ms_max / args.steps * 1e-3) / 1e9,
                                    "frac": step_bytes / (ms_max / args.steps * 1e-3) / 1e9 / peak}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * n + 72,
                "d2h_bytes_per_step": 28 * m_e2e},
    }
    if rank == 0:
        t_cpu, m_cpu, threads, reps = cpu_oracle_time(pos, rows, args.rc)
        t_one, m_one, _, reps_one = cpu_oracle_time(pos, rows, args.rc, budget_s=1.0,
                                                    min_reps=3, threads=1)
        line["cpu_baseline"] = {
            "value": m_cpu / t_cpu, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{reps} full builds of the workload (mean), C++ restatement of the "
                      "reference's rayon count/fill path",
            "cpu_model": cpu_model(),
            "one_thread": {"value": m_one / t_one, "unit": UNIT, "builds": reps_one}}
        if not args.no_extra:
            line["extra"] = extra_measurements(nl, torch, args)
        print(json.dumps(line), flush=True)
    barrier(world)


def median_call(fn, reps=5, warmup=2):
    """Median wall time of fn() over reps calls (results released between
    calls so pinned result buffers are reused); returns (seconds, result)."""
    for _ in range(warmup):
        r = fn()
        del r
    ts = []
    r = None
    for _ in range(reps):
        r = None
        t0 = time.perf_counter()
        r = fn()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts), r


def extra_measurements(nl, torch, args):
    W = workloads()

    out = {}
    steps = max(5, args.steps // 3)
    pos, rows = headline_system()
    dt = DeviceTimer(nl, torch, pos, rows, 14.0)
    ms, edges, _ = dt.run(steps, 2)
    out["cluster_liquid_rc14"] = {"edges_per_s": edges / (ms * 1e-3), "ms_per_step": ms / steps,
                                  "edges": edges // steps}
    p1 = W.isolated_cube()
    dt = DeviceTimer(nl, torch, p1, None, 6.0)
    ms, edges, _ = dt.run(steps, 2)
    out["isolated_cube_1000_rc6"] = {"edges_per_s": edges / (ms * 1e-3),
                                     "ms_per_step": ms / steps, "edges": edges // steps}
    nl.set_stream(None)
    # triclinic multi-cutoff (host-buffer call)
    p3, r3 = W.triclinic_uniform()
    cell = nl.PyCell(r3.T.tolist())
    t3, r = median_call(lambda: nl.build_neighborlists_multi(cell, p3, [5.0, 6.0, 12.0]))
    m3 = sum(v["edge_index"].shape[1] for v in r.values())
    del r
    out["triclinic_multi_e2e"] = {"edges_per_s": m3 / t3, "ms_per_call": 1e3 * t3, "edges": m3}
    # batched uneven systems (host-buffer call) vs the plain per-system loop
    systems = W.uneven_batch()
    pb, bb, cb = W.concat_batch(systems)
    nl.batch_tuner_reset()
    shapes = settle_batch_tuner(
        nl, lambda: nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0))
    nl.profile(True)
    tb, rb = median_call(lambda: nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0))
    calls, ph = nl.profile_read()
    nl.profile(False)
    mb = int(rb["edge_index"].shape[1])
    del rb
    dev_ms = sum(ph.values()) / max(calls, 1)
    cells = [None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist()) for s in systems]
    sample = 512
    tp, _ = median_call(lambda: [nl.build_neighborlists(cells[i], systems[i].positions, 5.0)
                                 for i in range(sample)], reps=3, warmup=1)
    out["uneven_batch_4096"] = {
        "systems_per_s_e2e": len(systems) / tb, "edges_per_s_e2e": mb / tb,
        "ms_per_call_e2e": 1e3 * tb, "systems_per_s_device": len(systems) / (dev_ms * 1e-3),
        "device_ms_phases": {k: v / max(calls, 1) for k, v in ph.items()},
        "plain_per_system_loop_systems_per_s": sample / tp,
        "atoms": int(pb.shape[0]), "edges": mb, "tuned_launch_shape": shapes}
    out["served"] = served_measurements(nl)
    out["output_options_rc6"] = output_option_measurements(nl, torch)
    out["verlet_md_rc6"] = verlet_measurements(nl, torch)
    out["verlet_md_rc14"] = verlet_measurements(nl, torch, 14.0)
    return out


def _median_device_call(torch, fn, reps=20, warmup=3):
    """Median wall time (s) of fn() with a device sync after each call."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts)


def output_option_measurements(nl, torch):
    """Headline system through build_neighborlists_torch (device in, device
    out): half list vs directed list with vectors and distances."""
    pos, rows = headline_system()
    cell = nl.PyCell(rows.T.tolist())
    dpos = torch.from_numpy(pos).cuda()
    t_half = _median_device_call(torch, lambda: nl.build_neighborlists_torch(cell, dpos, 6.0))
    r = nl.build_neighborlists_torch(cell, dpos, 6.0, directed=True, vectors=True,
                                     distances=True)
    m = int(r["edge_index"].shape[1])
    t_full = _median_device_call(torch, lambda: nl.build_neighborlists_torch(
        cell, dpos, 6.0, directed=True, vectors=True, distances=True))
    return {"half_list_ms": 1e3 * t_half, "directed_vectors_distances_ms": 1e3 * t_full,
            "directed_edges": m, "directed_edges_per_s": m / t_full,
            "bytes_out_per_edge": 28 + 24 + 8}


def verlet_measurements(nl, torch, rc=6.0):
    """MD-style use of the headline system: Verlet list at rc with a 1 A
    skin, positions moved by 0.01 A per step (no rebuild inside the sample),
    device positions in, device lists out; against a fresh build per step."""
    from neighborlist_rs.verlet import VerletList

    pos, rows = headline_system()
    cell = nl.PyCell(rows.T.tolist())
    rng = np.random.default_rng(31)
    steps = [torch.from_numpy(pos + rng.normal(0.0, 0.01 / 3 ** 0.5, pos.shape) * (k + 1) / 20)
             .cuda() for k in range(20)]
    with VerletList(rc, 1.0) as vl:
        vl.update(cell, steps[0])
        k = [0]

        def one():
            vl.update(cell, steps[k[0] % 20])
            k[0] += 1
        t_upd = _median_device_call(torch, one, reps=40, warmup=5)
        st = vl.stats()
    t_fresh = _median_device_call(torch, lambda: nl.build_neighborlists_torch(cell, steps[5], rc))
    return {"update_ms": 1e3 * t_upd, "fresh_build_ms": 1e3 * t_fresh,
            "stored_edges_rc_plus_skin": st["stored_edges"], "edges": st["last_edges"],
            "rebuilds": st["rebuilds"], "updates": st["updates"]}


def run_stream(srv, reqs, rate, seed=0, device=False):
    """Offers `reqs` [(cell, positions, cutoff)] to the server through its
    Python API (Server.submit / wait, numpy results; device=True: results
    stay in HBM and are released right after the wait): Poisson arrivals at
    `rate` req/s (None: all at once).  One client thread submits each
    request when it is due and, in between, collects finished results in
    arrival order (results dropped).  Latency is the server's submit -> done
    time of each request; the admission wait is the mean submit -> taken-by-
    a-worker time, from the server's counters."""
    import collections

    st0 = srv.stats()
    n = len(reqs)
    arrivals = (np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n))
                if rate else np.zeros(n))
    lat = np.zeros(n)
    edges = np.zeros(n, np.int64)
    pending = collections.deque()
    t0 = time.perf_counter()
    i = 0
    while i < n or pending:
        now = time.perf_counter() - t0
        if i < n and arrivals[i] <= now:
            c, p, rc = reqs[i]
            pending.append((i, srv.submit(c, p, rc, device_result=device)))
            i += 1
            if i == n:
                t_sub = time.perf_counter() - t0
            continue
        if not pending:
            time.sleep(max(0.0, arrivals[i] - now))
            continue
        try:
            j, t = pending[0]
            r, ms = srv.wait_timed(t, None if i >= n else max(0.0, arrivals[i] - now))
        except TimeoutError:
            continue
        pending.popleft()
        lat[j] = ms
        if device:
            edges[j] = r.n_edges
            r.release()
        else:
            edges[j] = r["edge_index"].shape[1]
        del r
    t = time.perf_counter() - t0
    st1 = srv.stats()
    started = max(1, (st1["completed"] + st1["failed"]) - (st0["completed"] + st0["failed"]))
    return {"offered_req_per_s": rate, "submitted_req_per_s": n / t_sub,
            "systems_per_s": n / t, "edges_per_s": float(edges.sum()) / t,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_admission_wait_ms": 1e-3 * (st1["us_queue_wait"] - st0["us_queue_wait"]) / started,
            "max_queued": st1["max_queued"], "requests": n, "edges": int(edges.sum()),
            "results": "device" if device else "host"}


def run_stream_raw(srv, reqs, device=False):
    """All requests at once through the C ABI with arguments marshalled
    beforehand (nlb_server_submit / nlb_server_wait / nlb_result_free):
    the server's capacity without the Python API's per-call cost.  With
    device=True results stay in HBM and are released right after the wait
    (no device-to-host copies)."""
    import ctypes

    import neighborlist_rs as nl

    lib, h = nl._lib, srv._handle()
    args = []
    for c, p, rc in reqs:
        hp, pb = nl._cell_args(c)
        args.append((p.ctypes.data_as(nl._dp), p.shape[0], hp, pb, float(rc)))
    r = nl._Result()
    lat = ctypes.c_double(0.0)
    lats = np.zeros(len(reqs))
    m = 0
    t0 = time.perf_counter()
    dev = int(device)
    tickets = [lib.nlb_server_submit(h, a, n, hp, pb, rc, dev) for a, n, hp, pb, rc in args]
    t_sub = time.perf_counter() - t0
    for k, t in enumerate(tickets):
        if lib.nlb_server_wait(h, t, -1.0, ctypes.byref(r), ctypes.byref(lat)) != 0:
            raise RuntimeError(lib.nlb_last_error().decode())
        m += r.n_edges
        lats[k] = lat.value
        if device:
            lib.nlb_server_release(h, t)
        else:
            lib.nlb_result_free(ctypes.byref(r))
    t = time.perf_counter() - t0
    return {"submitted_req_per_s": len(reqs) / t_sub, "systems_per_s": len(reqs) / t,
            "edges_per_s": m / t, "p50_ms": float(np.percentile(lats, 50)),
            "p99_ms": float(np.percentile(lats, 99)), "requests": len(reqs), "edges": int(m)}


def served_measurements(nl):
    """Served loop (continuous batching, 40 GB HBM budget, 4 workers): a small-request
    mix and a bounded sample of the full request-size distribution, each
    against the plain per-request loop (build_neighborlists) over the same
    requests.  Every arm runs once untimed over the same requests first."""
    W = workloads()
    from neighborlist_rs.serving import Server

    def as_reqs(stream):
        return [(None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist()),
                 s.positions, s.cutoff) for s in stream]

    def plain(reqs):
        t0 = time.perf_counter()
        m = 0
        for c, p, rc in reqs:
            r = nl.build_neighborlists(c, p, rc)
            m += r["edge_index"].shape[1]
            del r
        t = time.perf_counter() - t0
        return {"systems_per_s": len(reqs) / t, "edges_per_s": m / t, "requests": len(reqs)}

    out = {}
    small = as_reqs(W.request_stream(8192, seed=21, n_range=(16, 2048)))
    plain(small[:1024])
    res = {"plain_per_request_loop": plain(small[:1024])}
    with Server(hbm_budget_bytes=40 << 30, workers=4, max_batch=4096) as srv:
        # Untimed: the first runs pin host blocks and decide the batch kinds.
        run_stream(srv, small[:4096], None)
        run_stream_raw(srv, small[:4096])
        res["saturated_python_api"] = run_stream(srv, small[:4096], None)
        res["saturated_c_abi"] = run_stream_raw(srv, small[:4096])
        run_stream_raw(srv, small[:4096], device=True)
        res["saturated_c_abi_device_results"] = run_stream_raw(srv, small[:4096], device=True)
        # Poisson offered loads: at least 5000 requests per rate (8192 from
        # 10k req/s up), so that each p99 rests on 50+ samples.
        for rate in (1000, 2000, 10000, 25000, 50000):
            k = 5000 if rate < 10000 else len(small)
            res[f"poisson_{rate}"] = run_stream(srv, small[:k], rate, seed=rate)
        st = srv.stats()
        res["batches"] = st["batches"]
        res["largest_batch"] = st["largest_batch"]
    out["small_mix"] = dict(
        res, workload="8192 requests, N log-uniform [16, 2048], 70% orthorhombic / 20% "
                      "triclinic / 10% isolated, rho 0.1, rc in {5, 6, 8}")
    # The served distribution itself (N log-uniform [16, 1e6]) under Poisson
    # load: device-resident results (HBM-bound) and host results (bound by
    # the ~50 GB/s host link: ~2.5 MB of results per request on average).
    full_dist = as_reqs(W.request_stream(600, seed=23))
    res = {}
    with Server(hbm_budget_bytes=40 << 30, workers=4, max_batch=4096) as srv:
        # Untimed passes over every request first: a worker grows its
        # workspace (a device-synchronising reallocation of up to several
        # GB) the first time it meets a larger request, a one-time cost per
        # worker that would otherwise land in whichever timed run meets it.
        run_stream_raw(srv, full_dist, device=True)
        run_stream(srv, full_dist, None, device=True)
        run_stream(srv, full_dist, 2000, seed=1, device=True)
        for rate in (500, 1000, 2000):
            res[f"poisson_{rate}_device"] = run_stream(srv, full_dist, rate, seed=rate, device=True)
        run_stream(srv, full_dist[:100], None)
        for rate in (100, 200):
            res[f"poisson_{rate}_host"] = run_stream(srv, full_dist[:400], rate, seed=rate)
    out["full_distribution_poisson"] = dict(
        res, workload="600 requests of the served distribution (N log-uniform [16, 1e6], "
                      "70% orthorhombic / 20% triclinic / 10% isolated, rho 0.1, rc in {5, 6, 8}); "
                      "host-result rates use the first 400")
    full = as_reqs(W.request_stream(48, seed=22))
    plain(full)
    res = {"plain_per_request_loop": plain(full)}
    with Server(hbm_budget_bytes=40 << 30, workers=4, max_batch=4096) as srv:
        # Each worker grows its workspace (a device-synchronising reallocation)
        # the first time it meets a larger request, and results of new sizes
        # take new pinned blocks: warm every path until that has settled.
        for _ in range(3):
            run_stream_raw(srv, full, device=True)
        for _ in range(2):
            run_stream(srv, full, None)
        res["saturated_python_api"] = run_stream(srv, full, None)
        res["saturated_c_abi"] = run_stream_raw(srv, full)
        # (median of three runs: a run in which a worker first meets a larger
        # request than before reallocates its workspace and is several times
        # slower)
        runs = sorted((run_stream_raw(srv, full, device=True) for _ in range(3)),
                      key=lambda r: r["systems_per_s"])
        res["saturated_c_abi_device_results"] = dict(runs[1], runs_systems_per_s=[
            r["systems_per_s"] for r in runs])
        res["poisson_100"] = run_stream(srv, full, 100, seed=100)
    out["full_range_sample_48"] = dict(
        res, workload="48 requests, N log-uniform [16, 1e6] (bounded sample of the "
                      "served distribution), same cell/density/cutoff mix")
    return out


def main():
    args = parse()
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the
max-over-ranks timing reduction, the barrier, and the reference arm's
rank-0-only output.  Systems are independent, so the GPU path has no
collective; these helpers are the only cross-rank steps."""

import json
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(args, timeout=240):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(free_port())] + args
    env = dict(os.environ, OMP_NUM_THREADS="2")
    return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)


def test_max_over_ranks_and_barrier_gloo(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(textwrap.dedent(f"""
        import json, os, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        rank, local, world = bench.dist_init("gloo")
        # Each rank reports a different step time; all must agree on the max.
        t = bench.max_over_ranks(1.5 + rank, world)
        bench.barrier(world)
        out = {{"rank": rank, "world": world, "local": local, "max": t}}
        with open(os.path.join({str(tmp_path)!r}, f"rank{{rank}}.json"), "w") as f:
            json.dump(out, f)
        import torch.distributed as dist
        dist.destroy_process_group()
    """))
    r = torchrun([str(script)])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in (0, 1)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["world"] == 2 and x["max"] == 2.5 for x in lines)
    assert sorted(x["local"] for x in lines) == [0, 1]


def test_reference_arm_prints_once_on_rank0():
    r = torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                  "--warmup", "0"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["config"]["edges_per_step"] == 490514
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["cpu_model"]


def test_reference_arm_never_maps_the_product_library():
    """The CPU reference arm builds its workload without importing the
    neighborlist_rs package, so the CUDA library is never mapped into it, and
    it prints the same `config` dict as the GPU arm's bench_config."""
    code = textwrap.dedent("""
        import json, sys
        sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
        import bench
        bench.main()
        maps = open("/proc/self/maps").read()
        print(json.dumps({"mapped": "libnlb200" in maps,
                          "imported": "neighborlist_rs" in sys.modules}))
    """)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[1]
    assert probe == {"mapped": False, "imported": False}
    import bench

    assert line["config"] == bench.bench_config(bench.WORKLOAD, 10008, 490514)

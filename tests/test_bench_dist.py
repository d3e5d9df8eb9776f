"""Multi-process plumbing of bench.py on CPU: two gloo ranks (replicas) agree
on the maximum of their timings, and the barrier and shutdown complete."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(world, backend="gloo")
    d.barrier()
    m = d.max(float(rank + 1) * 1.5)
    d.close()
    out.put((rank, m))


@pytest.mark.timeout(120)
def test_replica_timing_is_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert res == {0: 3.0, 1: 3.0}


@pytest.mark.timeout(300)
def test_reference_arm_reports_the_gpu_arms_config_and_steps():
    """The reference arm (LLALBM's own OpenMP perform_lbm on the host cores)
    prints one JSON line on the GPU arm's config object, with the K timed
    steps and W warm-up steps it was asked for."""
    import json
    import subprocess

    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_runner_fast")):
        pytest.skip("the reference runner is not built (oracle/Makefile)")
    sys.path.insert(0, ROOT)
    import bench

    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "cavity129", "--steps", "7", "--warmup", "4"], capture_output=True, text=True, timeout=240,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "MLUPS" and line["value"] > 0
    assert (line["steps"], line["warmup"]) == (7, 4)
    wl = bench.workload("cavity129")
    assert line["config"] == bench.workload_config(wl, wl["types"](), 1)
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"

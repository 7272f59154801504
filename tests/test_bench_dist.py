"""The multi-process plumbing of bench.py (one process per GPU, replicas
only): two gloo ranks on the CPU check the max-over-ranks timing, the
whole-job aggregate and that the reference arm runs on rank 0 alone."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_init(world)
    assert (r, w, local) == (rank, world, rank) and dist.get_backend() == "gloo"
    ms = bench.reduce_max(10.0 + 5.0 * rank, w)  # the slower rank sets the time
    value = bench.job_mpaths(1_000_000, w, ms)
    ref_rc = bench.run_reference(None, 1, w) if rank == 1 else 0  # other ranks return without work
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, value, ref_rc))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, ref_rc in got:
        assert ms == pytest.approx(15.0)  # max over ranks
        assert value == pytest.approx(2 * 1_000_000 / 0.015 / 1e6)
        assert ref_rc == 0


def test_reference_arm_loads_no_product_library():
    """bench.py --impl reference runs the reference's CPU path (its host build,
    or the oracle) without mapping the product library, and reports the same
    config as the product arm."""
    import json
    import subprocess
    code = (
        "import sys, json, argparse\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "import bench\n"
        "args = argparse.Namespace(spp=1, warmup=0, steps=1, cpu_seconds=0.3)\n"
        "bench.run_reference(args, 0, 1)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('MAPS', 'liboptixrender_b200' in maps)\n"
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "MAPS False"
    line = json.loads(next(l for l in lines if l.startswith("{")))
    assert line["impl"] == "reference" and line["value"] > 0
    sys.path.insert(0, str(ROOT))
    import bench
    assert line["config"] == bench.bench_config(1, 1310720 + 64 * 20000, 1)

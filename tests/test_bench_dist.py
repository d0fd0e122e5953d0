"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the job time
is the max over ranks, and the reference arm prints one line from rank 0
only."""
import json
import os
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _worker(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    out = bench.reduce_max([10.0 + rank, 5.0 - rank])
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_max_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [11.0, 5.0]


def test_reference_arm_rank_handling(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "freq-solves/s" and line["value"] > 0
    assert line["cpu_baseline"]["cores"] >= 1 and line["e2e"]["h2d_bytes_per_step"] == 0


def test_lapack_leg_on_two_problems():
    """The LAPACK CPU leg (dstebz + dstein on the oracle's matrices, one
    problem per process of a spawn-started pool): mode counts from LAPACK
    equal the oracle's, and the line carries its fields."""
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench

    freqs = np.array([0.05, 0.12])
    out = bench.lapack_baseline(freqs, every=1)
    assert out["kind"] == "lapack" and out["value"] > 0 and out["cores"] >= 1
    assert "LAPACK reported an error" not in out["sample"]
    assert out["lapack_modes"] == out["oracle_modes"] > 0

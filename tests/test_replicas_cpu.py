"""The multi-GPU path of bench.py runs independent replicas (a single state does
not shard): each rank times its own device work, the ranks agree on the slowest
time with one MAX all-reduce, and the whole-job rate is all ranks' work over that
time.  Checked here with world_size 2 over gloo on CPU; the reference arm must
print nothing and exit 0 on ranks other than 0."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    try:
        mine = [3.5, 7.25][rank]
        q.put((rank, bench.max_over_ranks(mine, dist, "cpu"), bench.whole_job_rate(43600, 2, 7.25)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    ps = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [7.25, 7.25]
    assert got[0][2] == pytest.approx(2 * 43600 / 7.25e-3)


def test_reference_arm_is_silent_on_other_ranks():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""

"""Trajectory sharding over ranks (pysmoq.shard): contiguous shares of the
trajectory ids, and one FP64 SUM all-reduce of the per-rank sums.  Checked with
world_size 2 over gloo on CPU; the per-rank compute is the oracle's replay of the
same trajectory ids (the CUDA call needs a GPU), so the combined mean must equal
the single-process mean over all ids."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_trajectory_shares_cover_every_id_once():
    sys.path.insert(0, os.path.join(ROOT, "smoq.jl_b200"))
    from pysmoq.shard import trajectory_share
    for n in (0, 1, 7, 64, 4097):
        for world in (1, 2, 3, 8):
            shares = [trajectory_share(n, r, world) for r in range(world)]
            ids = [i for off, cnt in shares for i in range(off, off + cnt)]
            assert ids == list(range(n))
            assert max(c for _, c in shares) - min(c for _, c in shares) <= 1
    with pytest.raises(ValueError):
        trajectory_share(4, 2, 2)


def _ladder(L):
    import oracle as O
    bonds = [(r * L + s + 1, r * L + s + 2, 1.0, 1.0, 0.5) for r in range(2) for s in range(L - 1)]
    bonds += [(s + 1, L + s + 1, 0.7, 0.7, 0.3) for s in range(L)]
    fields = [(q + 1, 0.5, 0.0, 0.1 * q) for q in range(2 * L)]
    return O.precompute_trotter_gates(bonds, fields, 0.1)


def _rank(rank, port, q, n_traj):
    import torch.distributed as dist
    for p in (ROOT, os.path.join(ROOT, "smoq.jl_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import oracle as O
    import pysmoq
    from pysmoq import shard
    L, T = 2, 5
    arr, n = _ladder(L)
    u = np.linspace(0.1, 0.9, T)

    def oracle_share(psi0, H_params, gates, padded_u, L_, n_rails, T_, cnt, traj_offset=0, **kw):
        return O.qrc_run(L_, arr, n, padded_u[L_:L_ + T_], cnt, n_substeps=2, seed=77, traj_offset=traj_offset)

    pysmoq.run_mcwf_simulation = oracle_share  # the GPU call, replayed by the oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    try:
        X = shard.run_mcwf_simulation_sharded(dist, None, None, None, np.concatenate([np.zeros(L), u]), L, 2, T,
                                              n_traj, traj_offset=3)
        q.put((rank, X))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_traj", [9, 1])
def test_two_ranks_combine_to_the_single_run(built, n_traj):
    import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() + 7 * n_traj) % 2000
    ps = [ctx.Process(target=_rank, args=(r, port, q, n_traj)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(180)
    assert all(p.exitcode == 0 for p in ps)
    got = dict(q.get(timeout=10) for _ in range(2))
    arr, n = _ladder(2)
    want = O.qrc_run(2, arr, n, np.linspace(0.1, 0.9, 5), n_traj, n_substeps=2, seed=77, traj_offset=3)
    for r in (0, 1):
        assert np.allclose(got[r], want, atol=1e-13, rtol=0)

"""Trajectory sharding on one GPU: the ranks' shares are run one after another
through a stand-in for the process group whose all-reduce leaves each rank's
weighted sum as it is, so the sum over ranks must equal the mean of one run over
all trajectory ids (the shares replay exactly the same Philox streams).  No
kernel waits on another rank."""
import numpy as np
import pytest

import oracle as O
import pysmoq as S
from pysmoq import shard

pytestmark = pytest.mark.gpu


class OneRankOfTwo:
    """rank r of a world of 2 whose SUM all-reduce is left to the caller"""

    class ReduceOp:
        SUM = "sum"

    def __init__(self, rank):
        self.rank = rank

    def get_rank(self, group=None):
        return self.rank

    def get_world_size(self, group=None):
        return 2

    def all_reduce(self, t, op=None, group=None):
        return t


def test_qrc_shares_sum_to_the_single_run(ctx):
    L, T, n_traj = 2, 4, 9
    bonds = [(1, 2, 1.0, 1.0, 0.5), (3, 4, 1.0, 1.0, 0.5), (1, 3, 0.7, 0.7, 0.3), (2, 4, 0.7, 0.7, 0.3)]
    arr, n = O.precompute_trotter_gates(bonds, [(q, 0.5, 0.0, 0.2 * q) for q in range(1, 5)], 0.1)
    gates = [S.FastTrotterGate(i, U) for i, U in O.gates_to_list(arr, n)]
    padded = np.concatenate([np.zeros(L), np.linspace(0.2, 0.8, T)])
    kw = dict(ctx=ctx, dtype=S.C128, n_substeps=2, seed=5)
    parts = [shard.run_mcwf_simulation_sharded(OneRankOfTwo(r), None, None, gates, padded, L, 2, T, n_traj,
                                               traj_offset=11, **kw) for r in (0, 1)]
    want = S.run_mcwf_simulation(None, None, gates, padded, L, 2, T, n_traj, traj_offset=11, **kw)
    assert np.max(np.abs(parts[0] + parts[1] - want)) < 1e-12


def test_mcwf_shares_sum_to_the_single_run(ctx):
    N, n_traj, dt, steps, rec = 6, 9, 0.02, 20, 5
    arr, n = O.precompute_trotter_gates([(i, i + 1, 0.0, 0.0, 1.0) for i in range(1, N)],
                                        [(i, 1.0, 0.0, 0.0) for i in range(1, N + 1)], dt)
    gates = [S.FastTrotterGate(i, U) for i, U in O.gates_to_list(arr, n)]
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C128)
    jumps = [S.JumpOperator("sigma_minus", q, 0.3) for q in range(1, N + 1)]
    parts = [shard.mcwf_run_sharded(OneRankOfTwo(r), ctx, plan, N, S.C128, 0, n_traj, jumps, dt, 7, steps, rec,
                                    traj_offset=2) for r in (0, 1)]
    st = S.CuState(ctx, N, S.C128, n_traj, basis=0)
    want = S.mcwf_run(plan, st, jumps, dt, 7, steps, rec, traj_offset=2)
    st.close()
    plan.close()
    assert np.max(np.abs(parts[0][0] + parts[1][0] - want["z_mean"])) < 1e-12
    assert np.max(np.abs(parts[0][1] + parts[1][1] - want["zz_mean"])) < 1e-12

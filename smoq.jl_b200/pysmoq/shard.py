"""Trajectory sharding over ranks, one process per GPU.

MCWF and QRC trajectories are independent units (the reference threads over them:
cpuQuantumChannelLindbladianEvolutionMonteCarloWaveFunction.jl:345,
cpuQRCSimulationMonteCarloWaveFunction.jl:563).  Ranks split the trajectory ids
into contiguous shares, each rank runs its share on its own GPU with the ids'
own Philox streams (so the union is exactly the single-GPU run), and one FP64 SUM
all-reduce combines the per-rank sums into the trajectory means -- the only
exchange these workloads have.  No state crosses GPUs.
"""
from __future__ import annotations

import numpy as np


def trajectory_share(n_traj: int, rank: int, world: int):
    """(offset, count) of rank's contiguous share of n_traj trajectory ids; the
    first n_traj % world ranks take one more"""
    if world < 1 or not 0 <= rank < world or n_traj < 0:
        raise ValueError("bad rank / world / trajectory count")
    base, extra = divmod(n_traj, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def combine_means(means: np.ndarray, count: int, n_total: int, dist, group=None, device=None) -> np.ndarray:
    """The mean over all ranks' trajectories from this rank's mean over `count`
    of them: one FP64 SUM all-reduce of count * mean.  `device` is where the
    collective's buffer lives (a CUDA device for NCCL, None = CPU for gloo)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(means, dtype=np.float64) * count))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy() / float(n_total)


def run_mcwf_simulation_sharded(dist, psi0, H_params, gates, padded_u, L: int, n_rails: int, T: int, n_traj: int,
                                *args, group=None, device=None, traj_offset: int = 0, **kw):
    """run_mcwf_simulation (the bitwise QRC loop) over all ranks: this rank runs
    its share of the trajectory ids traj_offset .. traj_offset + n_traj - 1 and
    every rank returns the mean over all of them"""
    from . import run_mcwf_simulation
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    off, cnt = trajectory_share(n_traj, rank, world)
    if cnt > 0:
        X = run_mcwf_simulation(psi0, H_params, gates, padded_u, L, n_rails, T, cnt, *args,
                                traj_offset=traj_offset + off, **kw)
    else:
        from . import qrc_n_ops
        X = np.zeros((T, qrc_n_ops(L, n_rails)))
    return combine_means(X, cnt, n_traj, dist, group, device)


def mcwf_run_sharded(dist, ctx, plan, N: int, dtype: int, basis: int, n_traj: int, jump_ops, dt: float, seed: int,
                     steps: int, record_every: int, group=None, device=None, traj_offset: int = 0):
    """mcwf_run over all ranks: this rank evolves its share of the trajectories
    (a batch state of its own) and every rank returns the means of <Z_i> and
    <Z_i Z_{i+1}> over all trajectories at every record"""
    from . import CuState, mcwf_run
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    off, cnt = trajectory_share(n_traj, rank, world)
    nrec = steps // record_every + 1
    z, zz = np.zeros((nrec, N)), np.zeros((nrec, N - 1))
    if cnt > 0:
        st = CuState(ctx, N, dtype, cnt, basis=basis)
        try:
            r = mcwf_run(plan, st, jump_ops, dt, seed, steps, record_every, traj_offset=traj_offset + off)
        finally:
            st.close()
        z, zz = r["z_mean"], np.asarray(r["zz_mean"]).reshape(nrec, N - 1)
    both = combine_means(np.concatenate([z.reshape(-1), zz.reshape(-1)]), cnt, n_traj, dist, group, device)
    return both[:z.size].reshape(z.shape), both[z.size:].reshape(zz.shape)

"""GPU parity of the batched MCWF (quantum-jump) evolution.

* trajectory-exact: complex128 trajectories on the GPU and the oracle's
  so_mcwf_run share the Philox4x32-10 streams (key = seed, counter =
  (step, trajectory)), so jump counts match exactly and per-trajectory
  <Z_i>, <Z_i Z_{i+1}> records agree to rounding;
* statistical: the trajectory mean converges to the density-matrix oracle
  (Euler dissipator + Trotter rho step, N=8), the check of
  scripts_quantum_simulations/demo_quantum_channels.jl:413-456;
* the full configuration (TFIM N=16, sigma- 0.1 + sigma_z 0.05 on every qubit,
  4096 trajectories, dt 0.01, 500 steps, complex64) runs and stays physical.
"""
import math

import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


def tfim(N, dt, J=1.0, h=1.0):
    arr, n = O.precompute_trotter_gates([(i, i + 1, 0.0, 0.0, J) for i in range(1, N)],
                                        [(i, h, 0.0, 0.0) for i in range(1, N + 1)], dt)
    return arr, n, [S.FastTrotterGate(idx, U) for idx, U in O.gates_to_list(arr, n)]


def jumps(N, gm=0.1, gz=0.05):
    g = [S.JumpOperator("sigma_minus", q, gm) for q in range(1, N + 1)] + \
        [S.JumpOperator("sigma_z", q, gz) for q in range(1, N + 1)]
    o = [(0, q, gm) for q in range(1, N + 1)] + [(2, q, gz) for q in range(1, N + 1)]
    return g, o


@pytest.mark.parametrize("N,init", [(6, "ones"), (9, "neel")])
def test_trajectory_exact_vs_oracle(ctx, N, init):
    dt, steps, rec, B, seed = 0.05, 40, 5, 24, 1234
    arr, n, gates = tfim(N, dt)
    gj, oj = jumps(N, 0.3, 0.1)
    idx = (1 << N) - 1 if init == "ones" else sum(1 << k for k in range(0, N, 2))
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C128)
    st = S.CuState(ctx, N, S.C128, B, basis=idx)
    res = S.mcwf_run(plan, st, gj, dt, seed, steps, rec, traj_offset=7, per_trajectory=True)
    z, zz, nj = O.mcwf_run(N, arr, n, O.make_jumps(oj), len(oj), dt, seed, 7, B, steps, rec, init_index=idx,
                           nthreads=4)
    assert np.array_equal(res["jumps"], nj), (res["jumps"], nj)
    assert nj.sum() > 0
    assert np.max(np.abs(res["z_traj"] - z)) < 1e-10
    assert np.max(np.abs(res["zz_traj"] - zz)) < 1e-10
    assert np.max(np.abs(res["z_mean"] - z.mean(axis=1))) < 1e-10
    # the returned trajectories are normalised
    assert np.allclose(S.get_norm(st), 1.0, atol=1e-12)


def test_mean_converges_to_density_matrix(ctx):
    """N=8, 4096 complex64 trajectories vs the density-matrix oracle, within 5 sigma + 0.01."""
    N, dt, steps, B = 8, 0.01, 200, 4096
    arr, n, gates = tfim(N, dt)
    gj, oj = jumps(N)
    idx = (1 << N) - 1     # all excited: amplitude damping is active from the start
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C64)
    st = S.CuState(ctx, N, S.C64, B, basis=idx)
    res = S.mcwf_run(plan, st, gj, dt, 42, steps, steps // 4, per_trajectory=True)
    rho = np.zeros((1 << N, 1 << N), complex, order="F")
    rho[idx, idx] = 1
    recs = []
    for s in range(steps + 1):
        if s % (steps // 4) == 0:
            recs.append([O.dm_expect_z(rho, k, N) for k in range(1, N + 1)])
        if s == steps:
            break
        O.dm_trotter_step(rho, arr, n, N)
        for j in oj:
            O.dm_dissipator(rho, j, dt, N)
    recs = np.array(recs)
    sig = res["z_traj"].std(axis=1) / math.sqrt(B)
    dev = np.abs(res["z_mean"] - recs)
    assert np.all(dev < 5 * sig + 0.01), (dev.max(), sig.max())
    assert res["jumps"].sum() > B  # jumps happened


def test_full_configuration_runs_and_stays_physical(ctx):
    """TFIM N=16, 4096 trajectories, dt=0.01, 500 steps, complex64 amplitudes, FP64 sums."""
    N, dt, steps, B = 16, 0.01, 500, 4096
    _, _, gates = tfim(N, dt)
    gj, _ = jumps(N)
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C64)
    st = S.CuState(ctx, N, S.C64, B, basis=0)
    res = S.mcwf_run(plan, st, gj, dt, 2026, steps, 10)
    assert res["z_mean"].shape == (51, N) and res["zz_mean"].shape == (51, N - 1)
    assert np.allclose(res["z_mean"][0], 1.0) and np.allclose(res["zz_mean"][0], 1.0)
    assert np.all(np.abs(res["z_mean"]) <= 1 + 1e-6) and np.all(np.isfinite(res["zz_mean"]))
    # dephasing + the transverse field depolarise <Z> away from 1; damping pulls it back up
    assert res["z_mean"][-1].mean() < 0.99
    assert res["jumps"].mean() > 1
    n = S.get_norm(st)
    assert np.max(np.abs(n - 1)) < 1e-5


def test_bad_arguments_are_rejected(ctx):
    N = 4
    _, _, gates = tfim(N, 0.05)
    plan2 = S.TrotterPlan(ctx, N, gates, order=2, dtype=S.C128)
    st = S.CuState(ctx, N, S.C128, 2)
    with pytest.raises(S.SmoqError):
        S.mcwf_run(plan2, st, [S.JumpOperator("sigma_minus", 1, 0.1)], 0.05, 1, 3, 1)
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C128)
    with pytest.raises(S.SmoqError):
        S.mcwf_run(plan, st, [S.JumpOperator("sigma_minus", 1, 100.0)], 0.05, 1, 3, 1)

"""GPU parity of the QRC trajectory loop (smoq_qrc_run).

The oracle (so_qrc_run) restates _run_traj_loop_bitwise! / run_mcwf_simulation
(utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:451,531) with
encode_input_ry_psi! and qrc_reset_psi! (utils/cpu/cpuQRCstep.jl:96,332) and
draws the reset's r from the same Philox stream, so every trajectory is
compared feature by feature; the trajectory mean is also compared with the
density-matrix pipeline it converges to (so_qrc_dm_run)."""
import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[-1, 0, 3], ids=["auto", "resident", "streaming"])
def qctx(request, built):
    """engine -1 (default) and 0: every trajectory's state resident in shared memory;
    3: the states stream through HBM between the plan's compiled passes"""
    c = S.Context(0)
    if request.param >= 0:
        c.set_option(S._lib.OPT_ENGINE, request.param)
    yield c
    c.close()


def ladder(L, seed=1, dt=0.1):
    """XXZ rails plus rungs with random z fields: bonds (i, j, Jxx, Jyy, Jzz), fields (q, hx, hy, hz), 1-based"""
    rng = np.random.default_rng(seed)
    bonds = [(r * L + s + 1, r * L + s + 2, 1.0, 1.0, 0.5) for r in range(2) for s in range(L - 1)]
    bonds += [(s + 1, L + s + 1, 0.7, 0.7, 0.3) for s in range(L)]
    fields = [(q + 1, 0.5, 0.0, float(rng.uniform(-1, 1))) for q in range(2 * L)]
    return bonds, fields, dt


def gates_both(L, seed=1):
    bonds, fields, dt = ladder(L, seed)
    arr, n = O.precompute_trotter_gates(bonds, fields, dt)
    return arr, n, [g for g in O.gates_to_list(arr, n)]


def run_gpu(ctx, L, gl, u, n_traj, dtype, **kw):
    padded = np.concatenate([np.zeros(L), u])
    gates = [S.FastTrotterGate(q, np.asarray(U)) for q, U in gl]
    return S.run_mcwf_simulation(kw.pop("psi0", None), None, gates, padded, L, 2, len(u), n_traj, ctx=ctx,
                                 dtype=dtype, **kw)


@pytest.mark.parametrize("reset", ["traceout_rail_1", "traceout_rail_2"])
@pytest.mark.parametrize("encoding", ["batch", "broadcast"])
def test_trajectories_equal_the_oracle(qctx, reset, encoding):
    ctx = qctx
    L, T, n_traj = 3, 12, 16
    arr, n, gl = gates_both(L)
    u = np.random.default_rng(4).uniform(0, 1, T)
    X, Xt = run_gpu(ctx, L, gl, u, n_traj, S.C128, encoding=encoding, reset_type=reset, n_substeps=3, seed=99,
                    traj_offset=5, per_trajectory=True)
    Xr, Xtr = O.qrc_run(L, arr, n, u, n_traj, n_substeps=3, encoding=encoding, reset=reset, seed=99, traj_offset=5,
                        per_trajectory=True)
    assert X.shape == (T, S.qrc_n_ops(L)) and Xt.shape == (n_traj, T, S.qrc_n_ops(L))
    assert np.max(np.abs(Xt - Xtr)) < 1e-10
    assert np.max(np.abs(X - Xr)) < 1e-12


@pytest.mark.parametrize("L,dtype,tol", [(6, S.C128, 1e-9), (7, S.C64, 2e-4), (1, S.C128, 1e-12)])
def test_sizes_and_precisions(qctx, L, dtype, tol):
    """the largest rails each precision holds in shared memory, and the smallest"""
    T, n_traj = 4, 6
    arr, n, gl = gates_both(L, seed=L)
    u = np.random.default_rng(L).uniform(0, 1, T)
    X, Xt = run_gpu(qctx, L, gl, u, n_traj, dtype, n_substeps=2, seed=3, per_trajectory=True)
    Xr, Xtr = O.qrc_run(L, arr, n, u, n_traj, n_substeps=2, seed=3, per_trajectory=True)
    assert np.max(np.abs(Xt - Xtr)) < tol


def test_initial_state_and_zero_substeps(qctx):
    """a random initial state, and n_substeps = 0 (reset and measurement only)"""
    ctx = qctx
    L, T, n_traj = 2, 6, 10
    arr, n, gl = gates_both(L, seed=8)
    rng = np.random.default_rng(8)
    psi0 = rng.normal(size=16) + 1j * rng.normal(size=16)
    psi0 /= np.linalg.norm(psi0)
    u = rng.uniform(0, 1, T)
    for sub in (0, 4):
        X, Xt = run_gpu(ctx, L, gl, u, n_traj, S.C128, n_substeps=sub, seed=21, psi0=psi0, per_trajectory=True)
        Xr, Xtr = O.qrc_run(L, arr, n, u, n_traj, n_substeps=sub, seed=21, psi0=psi0, per_trajectory=True)
        assert np.max(np.abs(Xt - Xtr)) < 1e-12


@pytest.mark.parametrize("reset", ["traceout_rail_1", "traceout_rail_2"])
def test_trajectory_mean_converges_to_density_matrix(ctx, reset):
    """E[|psi_in><psi_in| (x) |phi><phi|] = rho_in (x) rho_kept: the mean of many
    complex64 trajectories matches the density-matrix pipeline within a few
    standard errors (features are bounded by 1; 40000 trajectories: 1/sqrt(n) = 0.005)"""
    L, T, n_traj = 2, 8, 40000
    arr, n, gl = gates_both(L, seed=2)
    u = np.random.default_rng(2).uniform(0, 1, T)
    X = run_gpu(ctx, L, gl, u, n_traj, S.C64, reset_type=reset, n_substeps=3, seed=5)
    D = O.qrc_dm_run(L, arr, n, u, n_substeps=3, reset=reset)
    assert np.max(np.abs(X - D)) < 0.03


def test_rejects_what_the_reference_rejects(ctx):
    L = 2
    _, _, gl = gates_both(L)
    gates = [S.FastTrotterGate(q, np.asarray(U)) for q, U in gl]
    padded = np.zeros(L + 3)
    with pytest.raises(ValueError):
        S.run_mcwf_simulation(None, None, gates, padded, L, 3, 3, 4, ctx=ctx)       # n_rails != 2
    with pytest.raises(ValueError):
        S.run_mcwf_simulation(None, None, gates, padded, L, 2, 3, 4, ctx=ctx, integrator_type="rk4")
    with pytest.raises(S.SmoqError):
        S.run_mcwf_simulation(None, None, gates, padded, L, 2, 3, 4, ctx=ctx, reset_type="protocol1",
                              encoding="batch", n_substeps=-1)
    big = 8  # N = 16 does not fit one CTA's shared memory
    _, _, glb = gates_both(big)
    with pytest.raises(S.SmoqError):
        S.run_mcwf_simulation(None, None, [S.FastTrotterGate(q, np.asarray(U)) for q, U in glb], np.zeros(big + 2),
                              big, 2, 2, 2, ctx=ctx, dtype=S.C64)

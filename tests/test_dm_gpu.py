"""GPU density matrices: rho (N qubits, column-major as Julia's Matrix) held as a
2N-qubit state, evolved by a plan of U on the row qubits, conj(U) on the column
qubits and one 4x4 superoperator per jump on (row bit, column bit).  Parity with
the density-matrix oracle (so_trotter_step_rho + so_dissipator_dm, restating
evolve_trotter_rho_cpu! and _apply_dissipator_dm!) and its Z observables."""
import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


def tfim_xxz(N, dt, seed=3):
    rng = np.random.default_rng(seed)
    bonds = [(i, i + 1, 1.0, 0.7, 0.5) for i in range(1, N)]
    fields = [(i, float(rng.uniform(-1, 1)), 0.0, float(rng.uniform(-1, 1))) for i in range(1, N + 1)]
    arr, n = O.precompute_trotter_gates(bonds, fields, dt)
    return arr, n, O.gates_to_list(arr, n)


@pytest.mark.parametrize("N,dtype,tol", [(5, S.C128, 1e-12), (6, S.C64, 2e-5)])
def test_dm_evolution_matches_oracle(ctx, N, dtype, tol):
    dt, steps = 0.02, 12
    arr, n, gl = tfim_xxz(N, dt)
    jumps = [S.JumpOperator("sigma_minus", 1, 0.3), S.JumpOperator("sigma_z", 2, 0.2),
             S.JumpOperator("sigma_plus", 3, 0.1), S.JumpOperator("sigma_x", N, 0.15)]
    oj = [(0, 1, 0.3), (2, 2, 0.2), (1, 3, 0.1), (3, N, 0.15)]
    init = sum(1 << k for k in range(0, N, 2))
    dim = 1 << N
    rho = np.zeros((dim, dim), complex, order="F")
    rho[init, init] = 1
    for _ in range(steps):
        O.dm_trotter_step(rho, arr, n, N)
        for j in oj:
            O.dm_dissipator(rho, j, dt, N)
    plan = S.DensityMatrixPlan(ctx, N, [S.FastTrotterGate(i, U) for i, U in gl], jumps, dt, dtype=dtype)
    st = S.density_matrix_state(ctx, N, init, dtype=dtype)
    plan.step(st, steps)
    got = st.download().astype(complex).reshape(dim, dim, order="F")
    assert np.max(np.abs(got - rho)) < tol
    masks = [0] + [1 << k for k in range(N)] + [3 << k for k in range(N - 1)]
    obs = S.dm_expect_zstrings(st, N, masks)[0]
    assert abs(obs[0] - np.real(np.trace(rho))) < tol
    for k in range(N):
        assert abs(obs[1 + k] - O.dm_expect_z(rho, k + 1, N)) < tol
    for k in range(N - 1):
        assert abs(obs[1 + N + k] - O.dm_expect_zz(rho, k + 1, k + 2, N)) < tol


def test_dm_plan_is_trace_preserving_at_n12(ctx):
    """N=12 (a 24-qubit state, 256 MiB complex128): after 20 steps the trace stays 1 and
    the diagonal stays a probability distribution"""
    N, dt = 12, 0.01
    arr, n, gl = tfim_xxz(N, dt)
    jumps = [S.JumpOperator("sigma_minus", q, 0.1) for q in range(1, N + 1)] + \
            [S.JumpOperator("sigma_z", q, 0.05) for q in range(1, N + 1)]
    plan = S.DensityMatrixPlan(ctx, N, [S.FastTrotterGate(i, U) for i, U in gl], jumps, dt)
    st = S.density_matrix_state(ctx, N, (1 << N) - 1)
    plan.step(st, 20)
    obs = S.dm_expect_zstrings(st, N, [0, 1, 2])[0]
    assert abs(obs[0] - 1.0) < 1e-10
    assert np.all(np.abs(obs[1:]) <= 1 + 1e-10)

"""GPU parity: every single-gate entry point of the C ABI against the oracle,
on random states, every qubit placement (adjacent, extreme, both orders),
complex128 (rel. err <= 1e-12) and complex64 (<= 2e-6), batch > 1."""
import math

import numpy as np
import pytest

import dense_ref as D
import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu

TOL = {S.C128: 1e-12, S.C64: 2e-6}
ANG = 1.2345


def run_gpu(ctx, psi, dtype, fn):
    N = int(math.log2(psi.size))
    st = S.CuState(ctx, N, dtype, 1, basis=None)
    st.upload(psi)
    fn(st, N)
    out = st.download().astype(np.complex128)
    st.close()
    return out


def rel(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


ONE_Q = [
    ("rx", lambda s, k, N: S.apply_rx_psi(s, k, ANG, N), lambda p, k, N: O.apply_rx_psi(p, k, ANG, N)),
    ("ry", lambda s, k, N: S.apply_ry_psi(s, k, ANG, N), lambda p, k, N: O.apply_ry_psi(p, k, ANG, N)),
    ("rz", lambda s, k, N: S.apply_rz_psi(s, k, ANG, N), lambda p, k, N: O.apply_rz_psi(p, k, ANG, N)),
    ("h", S.apply_hadamard_psi, O.apply_hadamard_psi),
    ("x", S.apply_pauli_x_psi, O.apply_pauli_x_psi),
    ("y", S.apply_pauli_y_psi, O.apply_pauli_y_psi),
    ("z", S.apply_pauli_z_psi, O.apply_pauli_z_psi),
    ("s", S.apply_s_psi, O.apply_s_psi),
    ("sdg", S.apply_sdagger_psi, O.apply_sdagger_psi),
    ("t", S.apply_t_psi, O.apply_t_psi),
    ("tdg", S.apply_tdagger_psi, O.apply_tdagger_psi),
    ("sigma_minus", S.apply_sigma_minus_psi, O.apply_sigma_minus_psi),
    ("sigma_plus", S.apply_sigma_plus_psi, O.apply_sigma_plus_psi),
]


@pytest.mark.parametrize("dtype", [S.C128, S.C64])
@pytest.mark.parametrize("name,gpu,ora", ONE_Q, ids=[c[0] for c in ONE_Q])
def test_one_qubit_gate(ctx, dtype, name, gpu, ora):
    rng = np.random.default_rng(7)
    for N in (1, 2, 5, 11):
        psi = D.random_state(N, rng)
        for k in sorted({1, 2, N // 2 + 1, N}):
            if k > N:
                continue
            want = ora(psi.copy(), k, N)
            got = run_gpu(ctx, psi, dtype, lambda st, n: gpu(st, k, n))
            assert rel(got, want) < TOL[dtype], (name, N, k)


TWO_Q = [
    ("cnot", lambda s, a, b, N: S.apply_cnot_psi(s, a, b, N), O.apply_cnot_psi),
    ("cz", lambda s, a, b, N: S.apply_cz_psi(s, a, b, N), O.apply_cz_psi),
    ("cry", lambda s, a, b, N: S.apply_cry_psi(s, a, b, ANG, N), lambda p, a, b, N: O.apply_cry_psi(p, a, b, ANG, N)),
    ("rxx", lambda s, a, b, N: S.apply_rxx_psi(s, a, b, ANG, N), lambda p, a, b, N: O.apply_rxx_psi(p, a, b, ANG, N)),
    ("ryy", lambda s, a, b, N: S.apply_ryy_psi(s, a, b, ANG, N), lambda p, a, b, N: O.apply_ryy_psi(p, a, b, ANG, N)),
    ("rzz", lambda s, a, b, N: S.apply_rzz_psi(s, a, b, ANG, N), lambda p, a, b, N: O.apply_rzz_psi(p, a, b, ANG, N)),
]


@pytest.mark.parametrize("dtype", [S.C128, S.C64])
@pytest.mark.parametrize("name,gpu,ora", TWO_Q, ids=[c[0] for c in TWO_Q])
def test_two_qubit_gate(ctx, dtype, name, gpu, ora):
    rng = np.random.default_rng(8)
    for N in (2, 3, 7, 12):
        psi = D.random_state(N, rng)
        pairs = {(1, 2), (2, 1), (1, N), (N, 1), (N - 1, N), (N, N - 1), (2, N)}
        for a, b in sorted(p for p in pairs if p[0] != p[1]):
            want = ora(psi.copy(), a, b, N)
            got = run_gpu(ctx, psi, dtype, lambda st, n: gpu(st, a, b, n))
            assert rel(got, want) < TOL[dtype], (name, N, a, b)


@pytest.mark.parametrize("dtype", [S.C128, S.C64])
def test_three_qubit_gates(ctx, dtype):
    rng = np.random.default_rng(9)
    N = 6
    psi = D.random_state(N, rng)
    for qs in [(1, 2, 3), (6, 1, 4), (3, 6, 2)]:
        want = O.apply_ccz_psi(psi.copy(), *qs, N)
        got = run_gpu(ctx, psi, dtype, lambda st, n: S.apply_ccz_psi(st, *qs, n))
        assert rel(got, want) < TOL[dtype]
        want = O.apply_toffoli_psi(psi.copy(), *qs, N)
        got = run_gpu(ctx, psi, dtype, lambda st, n: S.apply_toffoli_psi(st, *qs, n))
        assert rel(got, want) < TOL[dtype]


@pytest.mark.parametrize("dtype", [S.C128, S.C64])
def test_generic_gates_both_conventions(ctx, dtype):
    rng = np.random.default_rng(10)
    N = 8
    psi = D.random_state(N, rng)
    U2 = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))[0]
    U4 = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
    for k in (1, 4, 8):
        want = O.apply_one_qubit_gate(psi.copy(), U2, k, N)
        got = run_gpu(ctx, psi, dtype, lambda st, n: S.apply_one_qubit_gate_bitwise(st, U2, k, n))
        assert rel(got, want) < TOL[dtype]
    for a, b in [(1, 2), (2, 1), (3, 8), (8, 3)]:
        want = O.apply_two_qubit_gate(psi.copy(), U4, a, b, N)
        got = run_gpu(ctx, psi, dtype, lambda st, n: S.apply_two_qubit_gate_bitwise(st, U4, a, b, n))
        assert rel(got, want) < TOL[dtype], ("trotter", a, b)
        want = O.apply_2qubit_gate_ru(psi.copy(), U4, a, b, N)
        got = run_gpu(ctx, psi, dtype, lambda st, n: S.apply_2qubit_gate(st, U4, a, b, n))
        assert rel(got, want) < TOL[dtype], ("randomunitaries", a, b)


def test_batch_states_are_independent(ctx):
    rng = np.random.default_rng(12)
    N, B = 9, 5
    psis = np.stack([D.random_state(N, rng) for _ in range(B)])
    st = S.CuState(ctx, N, S.C128, B, basis=None)
    st.upload(psis)
    S.apply_rxx_psi(st, 2, 7, 0.3, N)
    S.apply_hadamard_psi(st, 9, N)
    got = st.download()
    for b in range(B):
        want = O.apply_rxx_psi(psis[b].copy(), 2, 7, 0.3, N)
        O.apply_hadamard_psi(want, 9, N)
        assert rel(got[b], want) < 1e-12


def test_bad_input_is_reported(ctx):
    st = S.CuState(ctx, 4, S.C128)
    with pytest.raises(S.SmoqError) as e:
        S.apply_rx_psi(st, 5, 0.1, 4)
    assert e.value.status == 1 and "out of range" in str(e.value)
    with pytest.raises(S.SmoqError):
        S.apply_cnot_psi(st, 2, 2, 4)
    with pytest.raises(S.SmoqError):
        S.apply_rx_psi(st, 1, float("nan"), 4)
    with pytest.raises(S.SmoqError):
        S.expect_local(st, 1, 4, "w")


def test_closing_a_context_closes_its_states_and_plans():
    """closing a Context first closes the states and plans made on it, so objects
    released later (e.g. at interpreter exit) never reach a destroyed context"""
    import gc
    c = S.Context(0)
    st = S.CuState(c, 10, S.C64, basis=3)
    plan = S.TrotterPlan(c, 10, [S.FastTrotterGate([1, 2], np.eye(4))], order=1, dtype=S.C64)
    plan.step(st, 1)
    c.close()
    assert st.h is None and plan.h is None
    del st, plan
    gc.collect()

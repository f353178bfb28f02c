"""GPU parity of the FP64 expectation reductions against the oracle."""
import numpy as np
import pytest

import dense_ref as D
import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


def upload(ctx, psi, dtype=S.C128, batch=1):
    N = int(np.log2(psi.shape[-1]))
    st = S.CuState(ctx, N, dtype, batch, basis=None)
    st.upload(psi)
    return st


@pytest.mark.parametrize("dtype,tol", [(S.C128, 1e-12), (S.C64, 2e-6)])
def test_local_and_correlators(ctx, dtype, tol):
    rng = np.random.default_rng(21)
    for N in (1, 2, 6, 13):
        psi = D.random_state(N, rng)
        st = upload(ctx, psi, dtype)
        for k in range(1, N + 1):
            for p in "xyz":
                assert abs(S.expect_local(st, k, N, p) - O.expect_local(psi, k, N, p)) < tol, (N, k, p)
        for a in range(1, N + 1):
            for b in (1, a + 1, N):
                if b == a or b > N:
                    continue
                for pp in ("xx", "yy", "zz"):
                    assert abs(S.expect_corr(st, a, b, N, pp) - O.expect_corr(psi, a, b, N, pp)) < tol


def test_known_answer_states(ctx):
    bell = np.zeros(4, complex)
    bell[0] = bell[3] = 1 / np.sqrt(2)
    st = upload(ctx, bell)
    assert abs(S.expect_local(st, 1, 2, "z")) < 1e-15
    assert abs(S.expect_corr(st, 1, 2, 2, "zz") - 1) < 1e-15
    assert abs(S.expect_corr(st, 1, 2, 2, "xx") - 1) < 1e-15
    assert abs(S.expect_corr(st, 1, 2, 2, "yy") + 1) < 1e-15
    ghz = np.zeros(8, complex)
    ghz[0] = ghz[7] = 1 / np.sqrt(2)
    st = upload(ctx, ghz)
    assert abs(S.get_expectation_pauli_string(st, ["Z", "Z", "Z"], [1, 2, 3], 3)) < 1e-15
    assert abs(S.get_expectation_pauli_string(st, ["X", "X", "X"], [1, 2, 3], 3) - 1) < 1e-15
    assert S.get_expectation_pauli_string(st, [], [], 3) == 1.0


def test_pauli_strings_random(ctx):
    rng = np.random.default_rng(22)
    N = 9
    psi = D.random_state(N, rng)
    st = upload(ctx, psi)
    for _ in range(40):
        n = int(rng.integers(1, 6))
        qs = [int(q) for q in rng.choice(np.arange(1, N + 1), size=n, replace=False)]
        ops = list(rng.choice(["X", "Y", "Z"], size=n))
        assert abs(S.get_expectation_pauli_string(st, ops, qs, N) - O.pauli_string(psi, ops, qs, N)) < 1e-12


def test_zstrings_batch_and_norm(ctx):
    rng = np.random.default_rng(23)
    N, B = 10, 3
    psis = np.stack([D.random_state(N, rng) * (b + 1) for b in range(B)])
    st = upload(ctx, psis, S.C128, B)
    masks = [0] + [1 << q for q in range(N)] + [(1 << q) | (1 << (q + 1)) for q in range(N - 1)] + [0b1011001]
    got = S.expect_zstrings(st, masks)
    for b in range(B):
        p = np.abs(psis[b]) ** 2
        idx = np.arange(1 << N)
        for o, m in enumerate(masks):
            sign = 1 - 2 * (np.array([bin(i & m).count("1") & 1 for i in idx]))
            assert abs(got[b, o] - np.sum(p * sign)) < 1e-11 * (b + 1) ** 2
    n = S.get_norm(st)
    assert np.allclose(n, np.linalg.norm(psis, axis=1), rtol=1e-13)
    S.normalize_state(st)
    assert np.allclose(S.get_norm(st), 1.0, rtol=1e-13)
    pe = S.population_excited_psi(st, 4, N)
    for b in range(B):
        assert abs(pe[b] - O.population_excited_psi(psis[b] / np.linalg.norm(psis[b]), 4, N)) < 1e-13


def test_many_observables_in_chunks(ctx):
    """more than 32 diagonal observables are split over several passes"""
    rng = np.random.default_rng(24)
    N = 12
    psi = D.random_state(N, rng)
    st = upload(ctx, psi)
    masks = [int(m) for m in rng.integers(0, 1 << N, size=70)]
    got = S.expect_zstrings(st, masks)[0]
    p = np.abs(psi) ** 2
    for o, m in enumerate(masks):
        sign = np.array([1 - 2 * (bin(i & m).count("1") & 1) for i in range(1 << N)])
        assert abs(got[o] - np.sum(p * sign)) < 1e-12


@pytest.mark.parametrize("L,rails,dtype,tol", [(5, 2, S.C128, 1e-12), (4, 3, S.C64, 1e-5), (9, 1, S.C128, 1e-12)])
def test_measure_all_observables_ladder(ctx, L, rails, dtype, tol):
    """measure_all_observables_state_vector_cpu! order and values: local X, Y, Z per
    qubit, then XX, YY, ZZ per rail bond, then per rung, against the oracle's
    _expect_* restatements, for two states of a batch"""
    N = L * rails
    rng = np.random.default_rng(N + rails)
    states = []
    for _ in range(2):
        v = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
        states.append(v / np.linalg.norm(v))
    st = S.CuState(ctx, N, dtype, 2, basis=None)
    st.upload(np.concatenate(states).astype(np.complex128 if dtype == S.C128 else np.complex64))
    got = S.measure_all_observables_state_vector(st, L, rails)
    for b, psi in enumerate(states):
        want = []
        for k in range(1, N + 1):
            want += [O.expect_local(psi, k, N, p) for p in "xyz"]
        pairs = [(r * L + s, r * L + s + 1) for r in range(rails) for s in range(1, L)]
        pairs += [(r * L + s, (r + 1) * L + s) for r in range(rails - 1) for s in range(1, L + 1)]
        for i, j in pairs:
            want += [O.expect_corr(psi, i, j, N, pp) for pp in ("xx", "yy", "zz")]
        assert got.shape == (2, len(want))
        assert np.max(np.abs(got[b] - np.array(want))) < tol


def test_bounded_wait_times_out_and_the_context_survives(ctx):
    """the failure path of the tile kernels' bounded waits: a wait that nothing
    completes gives up after its limit and the call returns SMOQ_ERR_TIMEOUT with
    the reason; the next calls on the same context still compute"""
    from pysmoq import _lib as L
    assert L.lib.smoq_debug_wait_timeout(ctx.h, 2_000_000) == L.SMOQ_ERR_TIMEOUT
    assert b"bounded device wait" in L.lib.smoq_last_error(ctx.h)
    st = S.CuState(ctx, 12, S.C128, basis=0)
    S.apply_rx_psi(st, 3, 0.8, 12)
    assert abs(S.expect_local(st, 3, 12, "z") - np.cos(0.8)) < 1e-12
    assert L.lib.smoq_debug_wait_timeout(ctx.h, 10) == L.SMOQ_ERR_BADINPUT   # limit below 1 us
    st.close()

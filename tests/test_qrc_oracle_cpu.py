"""The QRC oracle (so_qrc_*), pinned without a GPU.

The reference ships no golden vectors for its QRC loop, so the restatement is
pinned by (1) the identity its docstring states for the MCWF reset
(utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:431-433,
E[|psi_new><psi_new|] = |psi_in><psi_in| (x) rho_reservoir): the trajectory mean
converges to the density-matrix pipeline of run_dm_simulation
(utils/cpu/cpuQRCSimulationDensityMatrix.jl:186-244); (2) the encoding
examples of encode_input_ry_psi (utils/cpu/cpuQRCstep.jl:57-63: u = 0 -> |0>,
u = 0.5 -> |+>, u = 1 -> |1>); (3) the inverse-CDF reset on states whose
outcome is known; (4) the window rule of both encodings."""
import numpy as np
import pytest

import oracle as O


def ladder_gates(L, seed=1, dt=0.1):
    rng = np.random.default_rng(seed)
    bonds = [(r * L + s + 1, r * L + s + 2, 1.0, 1.0, 0.5) for r in range(2) for s in range(L - 1)]
    bonds += [(s + 1, L + s + 1, 0.7, 0.7, 0.3) for s in range(L)]
    fields = [(q + 1, 0.5, 0.0, float(rng.uniform(-1, 1))) for q in range(2 * L)]
    return O.precompute_trotter_gates(bonds, fields, dt)


@pytest.mark.parametrize("reset", ["traceout_rail_1", "traceout_rail_2"])
@pytest.mark.parametrize("encoding", ["batch", "broadcast"])
def test_trajectory_mean_converges_to_density_matrix(reset, encoding):
    L = 2
    arr, n = ladder_gates(L, seed=3)
    u = np.random.default_rng(5).uniform(0, 1, 6)
    X = O.qrc_run(L, arr, n, u, 20000, n_substeps=3, encoding=encoding, reset=reset, seed=11, nthreads=8)
    D = O.qrc_dm_run(L, arr, n, u, n_substeps=3, encoding=encoding, reset=reset)
    assert np.max(np.abs(X - D)) < 0.025        # 1/sqrt(20000) = 0.007 per bounded feature
    # and the deviation shrinks with more trajectories (statistical, not systematic)
    X4 = O.qrc_run(L, arr, n, u, 2000, n_substeps=3, encoding=encoding, reset=reset, seed=11, nthreads=8)
    assert np.sqrt(np.mean((X - D) ** 2)) < np.sqrt(np.mean((X4 - D) ** 2))


def test_encoding_examples():
    import ctypes as C
    for uval, want in [(0.0, [1, 0]), (0.5, [2 ** -0.5, 2 ** -0.5]), (1.0, [0, 1])]:
        pin = np.zeros(2, dtype=np.complex128)
        w = np.array([uval])
        O.L.so_qrc_encode(w.ctypes.data_as(O._dp), 1, O._p(pin))
        assert np.allclose(pin, want, atol=1e-15)
    # two qubits: qubit 1 on bit 0 (little-endian), kron(Ry(pi u2)|0>, Ry(pi u1)|0>)
    w = np.array([0.3, 0.8])
    pin = np.zeros(4, dtype=np.complex128)
    O.L.so_qrc_encode(w.ctypes.data_as(O._dp), 2, O._p(pin))
    one = [np.array([np.cos(np.pi * x / 2), np.sin(np.pi * x / 2)]) for x in w]
    assert np.allclose(pin, np.kron(one[1], one[0]), atol=1e-15)


def test_window_rule():
    L, u = 3, np.array([0.1, 0.2, 0.3, 0.4])
    padded = O.qrc_padded(u, L)
    win = np.zeros(L)
    got_b, got_c = [], []
    for k in range(len(u)):
        O.L.so_qrc_window(padded.ctypes.data_as(O._dp), L, k, 0, win.ctypes.data_as(O._dp))
        got_b.append(win.copy())
        O.L.so_qrc_window(padded.ctypes.data_as(O._dp), L, k, 1, win.ctypes.data_as(O._dp))
        got_c.append(win.copy())
    # :batch -> [u_{k-L+1}, ..., u_k] with zeros before the series; :broadcast -> u_k everywhere
    assert np.allclose(got_b, [[0, 0, .1], [0, .1, .2], [.1, .2, .3], [.2, .3, .4]])
    assert np.allclose(got_c, [[u[k]] * L for k in range(len(u))])


def reset(psi, pin, L, protocol, r):
    out = np.zeros_like(psi)
    o = O.L.so_qrc_reset(O._p(out), O._p(psi), O._p(pin), L, protocol, r)
    return o, out


def test_reset_inverse_cdf_and_conditional_state():
    L = 1
    pin = np.array([0.6, 0.8], dtype=np.complex128)
    # psi = (|0>_in |a> + |1>_in |b>)/sqrt(2), M[i, j] = psi[i + 2 j]
    a, b = np.array([1, 1j]) / np.sqrt(2), np.array([1, -1]) / np.sqrt(2)
    psi = np.zeros(4, dtype=np.complex128)
    psi[0::2] = a / np.sqrt(2)
    psi[1::2] = b / np.sqrt(2)
    for r, want, kept in [(0.2, 0, a), (0.49, 0, a), (0.51, 1, b), (0.99, 1, b)]:
        o, out = reset(psi, pin, L, 1, r)
        assert o == want
        assert np.allclose(out, np.kron(kept, pin))          # psi_in on the low bits
    # rail 2 measures the reservoir (high bit): columns of M
    c0, c1 = np.array([0.6, 0.8j]), np.array([1, 0])
    psi2 = np.concatenate([c0 * np.sqrt(0.3), c1 * np.sqrt(0.7)]).astype(np.complex128)
    for r, want, kept in [(0.29, 0, c0), (0.31, 1, c1)]:
        o, out = reset(psi2, pin, L, 2, r)
        assert o == want and np.allclose(out, np.kron(kept, pin))


def test_reset_rounding_keeps_the_first_outcome():
    """r above the accumulated probability (rounding): outcome 1 of qrc_reset_psi!'s default"""
    L = 1
    psi = np.array([0, 1, 0, 0], dtype=np.complex128)       # input |1>, reservoir |0>
    o, out = reset(psi, np.array([1, 0], dtype=np.complex128), L, 1, 1.0 + 1e-12)
    assert o == 0                                           # the first (zero-probability) row
    assert np.allclose(out, [1, 0, 0, 0])                   # the norm fallback: reservoir |0>


def test_density_matrix_observables_on_pure_states():
    """so_expect_pauli_rho on |psi><psi| equals the pure-state ladder set
    (measure_all_observables_state_vector_cpu!, cpuQuantumStateObservables.jl:1483)"""
    L, N = 2, 4
    rng = np.random.default_rng(9)
    psi = rng.normal(size=16) + 1j * rng.normal(size=16)
    psi /= np.linalg.norm(psi)
    want = O.measure_all_observables(psi, L, 2)
    rho = np.ascontiguousarray(np.outer(psi, psi.conj()).T)  # column-major in memory
    got = []
    pairs = [(0, 1), (2, 3), (0, 2), (1, 3)]
    for q in range(N):
        m = 1 << q
        got += [O.L.so_expect_pauli_rho(O._p(rho), m, 0, N), O.L.so_expect_pauli_rho(O._p(rho), m, m, N),
                O.L.so_expect_pauli_rho(O._p(rho), 0, m, N)]
    for i, j in pairs:
        m = (1 << i) | (1 << j)
        got += [O.L.so_expect_pauli_rho(O._p(rho), m, 0, N), O.L.so_expect_pauli_rho(O._p(rho), m, m, N),
                O.L.so_expect_pauli_rho(O._p(rho), 0, m, N)]
    assert np.allclose(got, want, atol=1e-14)

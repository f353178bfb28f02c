"""The oracle's noise unravelings, reset and noisy-circuit executor (CPU only).

Pinned three ways:
* each branch of each routine against the reference's stated rule
  (utils/cpu/cpuQuantumChannelKrausOperators.jl:262-386): dephasing applies Z
  when u < (1 - sqrt(1 - p)) / 2, depolarizing X / Y / Z on u below p/3, 2p/3,
  p, bit and phase flip X / Z on u < p, amplitude damping the normalised
  K1 psi (jump, u < gamma <n_1>) or K0 psi;
* the mean over trajectories equals the reference's density-matrix channels of
  the same file (:84-237, restated below as Kraus sums): the MCWF unravelling
  is unbiased;
* measurements, resets and classical conditions against known outcomes
  (cpuQuantumStateMeasurements.jl:224, :555; cpuVariationalQuantumCircuitExecutor.jl:103-105).
"""
import numpy as np
import pytest

import dense_ref as D
import oracle as O

X = np.array([[0, 1], [1, 0]], complex)
Y = np.array([[0, -1j], [1j, 0]], complex)
Z = np.diag([1.0 + 0j, -1.0])
I2 = np.eye(2, dtype=complex)


def on(M, k, N):
    """the 2x2 M on 1-based qubit k of N (bit k-1), as a dense 2^N matrix"""
    out = np.array([[1.0 + 0j]])
    for q in range(N, 0, -1):
        out = np.kron(out, M if q == k else I2)
    return out


def kraus(rho, Ks):
    return sum(K @ rho @ K.conj().T for K in Ks)


def channel(kind, rho, p, k, N):
    """the reference's density-matrix channels (cpuQuantumChannelKrausOperators.jl:84-237) as Kraus sums"""
    if kind == "dephasing":        # coherences * sqrt(1 - p), :86-104
        q = (1 - np.sqrt(1 - p)) / 2
        return kraus(rho, [np.sqrt(1 - q) * on(I2, k, N), np.sqrt(q) * on(Z, k, N)])
    if kind == "depolarizing":     # (1-p) rho + p/3 (X rho X + Y rho Y + Z rho Z), :107-142
        return kraus(rho, [np.sqrt(1 - p) * on(I2, k, N)] + [np.sqrt(p / 3) * on(P, k, N) for P in (X, Y, Z)])
    if kind == "bit_flip":         # :184-215
        return kraus(rho, [np.sqrt(1 - p) * on(I2, k, N), np.sqrt(p) * on(X, k, N)])
    if kind == "phase_flip":       # coherences * (1 - 2p), :218-237
        return kraus(rho, [np.sqrt(1 - p) * on(I2, k, N), np.sqrt(p) * on(Z, k, N)])
    if kind == "amplitude_damping":  # :145-180
        K0 = np.array([[1, 0], [0, np.sqrt(1 - p)]], complex)
        K1 = np.array([[0, np.sqrt(p)], [0, 0]], complex)
        return kraus(rho, [on(K0, k, N), on(K1, k, N)])
    raise ValueError(kind)


@pytest.mark.parametrize("kind,p,branches", [
    ("dephasing", 0.36, [(0.05, Z), (0.11, I2)]),                  # q = 0.1
    ("depolarizing", 0.3, [(0.05, X), (0.15, Y), (0.25, Z), (0.5, I2)]),
    ("bit_flip", 0.2, [(0.1, X), (0.3, I2)]),
    ("phase_flip", 0.2, [(0.1, Z), (0.3, I2)]),
])
def test_pauli_unravelings_apply_the_drawn_pauli(kind, p, branches):
    N, k = 4, 3
    rng = np.random.default_rng(1)
    for u, P in branches:
        psi = D.random_state(N, rng)
        want = on(P, k, N) @ psi
        got = O.noise_u(kind, psi.copy(), p, k, N, u)
        assert np.max(np.abs(got - want)) < 1e-14, (kind, u)


def test_amplitude_damping_jump_and_no_jump():
    N, k, g = 3, 2, 0.3
    rng = np.random.default_rng(2)
    psi = D.random_state(N, rng)
    P1 = on(np.diag([0, 1.0 + 0j]), k, N)
    pop1 = float(np.vdot(psi, P1 @ psi).real)
    K0 = on(np.array([[1, 0], [0, np.sqrt(1 - g)]], complex), k, N)
    K1 = on(np.array([[0, 1], [0, 0]], complex), k, N)
    for u, K in ((0.5 * g * pop1, K1), (1.01 * g * pop1, K0)):
        want = K @ psi
        want /= np.linalg.norm(want)
        got = O.noise_u("amplitude_damping", psi.copy(), g, k, N, u)
        assert np.max(np.abs(got - want)) < 1e-14


@pytest.mark.parametrize("kind,p", [("dephasing", 0.5), ("depolarizing", 0.45), ("bit_flip", 0.3),
                                    ("phase_flip", 0.25), ("amplitude_damping", 0.4)])
def test_trajectory_mean_equals_the_density_matrix_channel(kind, p):
    """mean over trajectories of |psi><psi| after the unravelling = the reference's DM channel"""
    N, k, T = 3, 2, 6000
    rng = np.random.default_rng(3)
    psi0 = D.random_state(N, rng)
    rho = np.zeros((1 << N, 1 << N), complex)
    for t in range(T):
        v = O.noise_u(kind, psi0.copy(), p, k, N, O.circuit_draw(11, 0, t))
        rho += np.outer(v, v.conj())
    rho /= T
    want = channel(kind, np.outer(psi0, psi0.conj()), p, k, N)
    assert np.max(np.abs(rho - want)) < 0.03, np.max(np.abs(rho - want))


def test_measurement_reset_and_conditions():
    N = 3
    rng = np.random.default_rng(4)
    # reset to every target from a random state: qubit 2 ends in the target, the rest is the conditional state
    targets = {"zero": np.array([1, 0], complex), "one": np.array([0, 1], complex),
               "plus": np.array([1, 1], complex) / np.sqrt(2), "minus": np.array([1, -1], complex) / np.sqrt(2)}
    for name, t in targets.items():
        for u in (0.2, 0.8):
            psi = D.random_state(N, rng)
            P0 = on(np.diag([1.0 + 0j, 0]), 2, N)
            m = 0 if u < float(np.vdot(psi, P0 @ psi).real) else 1
            got = O.reset_u(psi.copy(), 2, name, N, u)
            # the state is |t> on qubit 2 times the normalised branch of outcome m on the others
            branch = psi.reshape(2, 2, 2)[:, m, :]               # axes: qubit 3, qubit 2, qubit 1
            branch = branch / np.linalg.norm(branch)
            want = np.einsum("ac,b->abc", branch, t).reshape(-1)
            assert np.max(np.abs(got - want)) < 1e-14, (name, u)
    # X-basis measurement of |+>: always 0, state unchanged; Y basis of |+i>: always 0
    plus = np.ones(2, complex) / np.sqrt(2)
    psi = plus.copy()
    out = O.apply_circuit_mcwf(psi, O.make_ops([("measure_x", [1], 0, 0.0)]), 1, np.zeros(1), 1, 5, 0)
    assert list(out) == [0] and np.max(np.abs(psi - plus)) < 1e-14
    plus_i = np.array([1, 1j]) / np.sqrt(2)
    psi = plus_i.copy()
    out = O.apply_circuit_mcwf(psi, O.make_ops([("measure_y", [1], 0, 0.0)]), 1, np.zeros(1), 1, 5, 0)
    assert list(out) == [0] and np.max(np.abs(psi - plus_i)) < 1e-14
    # feed-forward: H on qubit 1, measure it, X on qubit 2 if the outcome was 1; then
    # qubit 2 equals the outcome; a condition on a measurement not yet made never holds
    ops = O.make_ops([("h", [1], 0, 0.0), ("x", [3], 0, 0.0, 2), ("measure_z", [1], 0, 0.0),
                      ("x", [2], 0, 0.0, 1)])
    seen = set()
    for traj in range(40):
        psi = O.zero_state(N, 0)
        out = O.apply_circuit_mcwf(psi, ops, 4, np.zeros(1), N, 9, traj)
        m = int(out[0])
        seen.add(m)
        idx = m | (m << 1)
        assert abs(abs(psi[idx]) - 1) < 1e-14, (traj, m)
    assert seen == {0, 1}

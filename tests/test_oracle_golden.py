"""Pins the CPU oracle (oracle/smoq_oracle.c) before it is trusted as the checker:
(1) the known-answer checks of the reference's own demo suites and docstrings
(tests/golden/known_answers.json), (2) an independent dense kron-product
restatement of every gate and observable (tests/dense_ref.py), (3) the
Philox4x32-10 known-answer vectors of Salmon et al. (SC'11)."""
import json
import math
import os

import numpy as np
import pytest

import dense_ref as D
import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KA = json.load(open(os.path.join(GOLD, "known_answers.json")))


def c(pair_list):
    return np.array([a + 1j * b for a, b in pair_list])


# ------------------------------------------------------- known answers
def test_rotations_on_zero():
    ka = KA["rotations_on_zero"]
    for case in ka["cases"]:
        psi = O.zero_state(1)
        getattr(O, f"apply_{case['gate']}_psi")(psi, 1, case["theta"], 1)
        assert np.max(np.abs(psi - c(case["psi"]))) < ka["tol"], case


@pytest.mark.parametrize("N", KA["hadamard_all_uniform"]["N"])
def test_hadamard_all_uniform(N):
    psi = O.zero_state(N)
    for k in range(1, N + 1):
        O.apply_hadamard_psi(psi, k, N)
    u = np.full(1 << N, 1 / math.sqrt(1 << N))
    F = abs(np.vdot(u, psi)) ** 2
    assert abs(F - 1.0) < KA["hadamard_all_uniform"]["tol"]


@pytest.mark.parametrize("N", KA["ry_half_squared"]["N"])
def test_ry_half_squared(N):
    p1, p2 = O.zero_state(N), O.zero_state(N)
    for k in range(1, N + 1):
        O.apply_ry_psi(p1, k, math.pi / 2, N)
        O.apply_ry_psi(p1, k, math.pi / 2, N)
        O.apply_ry_psi(p2, k, math.pi, N)
    assert abs(abs(np.vdot(p1, p2)) ** 2 - 1) < 1e-10


def test_norm_after_ry():
    N = 16
    psi = O.zero_state(N)
    for k in range(1, N + 1):
        O.apply_ry_psi(psi, k, math.pi / 4, N)
    assert abs(math.sqrt(O.norm2(psi, N)) - 1) < 1e-10


def test_bell_and_ghz_observables():
    b = KA["bell"]
    psi = np.zeros(4, complex)
    psi[0] = psi[3] = 1 / math.sqrt(2)
    assert abs(O.expect_local(psi, 1, 2, "z") - b["z1"]) < 1e-14
    assert abs(O.expect_corr(psi, 1, 2, 2, "zz") - b["zz"]) < 1e-14
    assert abs(O.expect_corr(psi, 1, 2, 2, "xx") - b["xx"]) < 1e-14
    assert abs(O.expect_corr(psi, 1, 2, 2, "yy") - b["yy"]) < 1e-14
    g = KA["ghz3"]
    psi = np.zeros(8, complex)
    psi[0] = psi[7] = 1 / math.sqrt(2)
    assert abs(O.pauli_string(psi, ["Z", "Z", "Z"], [1, 2, 3], 3) - g["zzz"]) < 1e-14
    assert abs(O.pauli_string(psi, ["X", "Z"], [1, 2], 3) - g["x1z2"]) < 1e-14
    assert abs(O.pauli_string(psi, ["X", "X", "X"], [1, 2, 3], 3) - g["xxx"]) < 1e-14
    pp = np.full(4, 0.5 + 0j)
    assert abs(O.expect_corr(pp, 1, 2, 2, "xx") - KA["plus_plus_xx"]["xx"]) < 1e-14


def test_psi_vs_rho_observables():
    """demo_parametrized_gates.jl:1040-1057: the Z/ZZ reductions of a pure state
    equal those of its density matrix, tol 1e-12."""
    N = 6
    rng = np.random.default_rng(3)
    psi = D.random_state(N, rng)
    rho = np.asfortranarray(np.outer(psi, psi.conj()))
    for k in range(1, N + 1):
        assert abs(O.expect_local(psi, k, N, "z") - O.dm_expect_z(rho, k, N)) < 1e-12
    for k in range(1, N):
        assert abs(O.expect_corr(psi, k, k + 1, N, "zz") - O.dm_expect_zz(rho, k, k + 1, N)) < 1e-12


# --------------------------------------------- dense restatement, all gates
N_D = 5


@pytest.fixture
def st():
    return D.random_state(N_D, np.random.default_rng(11))


ANG = 0.7321


def _one_qubit_cases():
    return [("rx", lambda k: D.embed({k: D.rx(ANG)}, N_D), True), ("ry", lambda k: D.embed({k: D.ry(ANG)}, N_D), True),
            ("rz", lambda k: D.embed({k: D.rz(ANG)}, N_D), True), ("hadamard", lambda k: D.embed({k: D.H}, N_D), False),
            ("pauli_x", lambda k: D.embed({k: D.X}, N_D), False), ("pauli_y", lambda k: D.embed({k: D.Y}, N_D), False),
            ("pauli_z", lambda k: D.embed({k: D.Z}, N_D), False), ("s", lambda k: D.embed({k: D.S}, N_D), False),
            ("sdagger", lambda k: D.embed({k: D.S.conj()}, N_D), False),
            ("t", lambda k: D.embed({k: D.T}, N_D), False), ("tdagger", lambda k: D.embed({k: D.T.conj()}, N_D), False),
            ("sigma_minus", lambda k: D.embed({k: D.SM}, N_D), False),
            ("sigma_plus", lambda k: D.embed({k: D.SP}, N_D), False)]


@pytest.mark.parametrize("name,M,param", _one_qubit_cases())
def test_one_qubit_gates_vs_dense(st, name, M, param):
    for k in range(1, N_D + 1):
        psi = st.copy()
        f = getattr(O, f"apply_{name}_psi")
        f(psi, k, ANG, N_D) if param else f(psi, k, N_D)
        assert np.max(np.abs(psi - M(k) @ st)) < 1e-13, (name, k)


def test_two_three_qubit_gates_vs_dense(st):
    for a in range(1, N_D + 1):
        for b in range(1, N_D + 1):
            if a == b:
                continue
            cases = [
                (O.apply_cnot_psi, (a, b), D.controlled(D.X, a, b, N_D)),
                (O.apply_cz_psi, (a, b), D.controlled(D.Z, a, b, N_D)),
                (O.apply_cry_psi, (a, b, ANG), D.controlled(D.ry(ANG), a, b, N_D)),
                (O.apply_rxx_psi, (a, b, ANG), D.rpp(D.X, a, b, ANG, N_D)),
                (O.apply_ryy_psi, (a, b, ANG), D.rpp(D.Y, a, b, ANG, N_D)),
                (O.apply_rzz_psi, (a, b, ANG), D.rpp(D.Z, a, b, ANG, N_D)),
            ]
            for f, args, M in cases:
                psi = st.copy()
                f(psi, *args, N_D)
                assert np.max(np.abs(psi - M @ st)) < 1e-13, (f.__name__, a, b)
    psi = st.copy()
    O.apply_ccz_psi(psi, 1, 3, 5, N_D)
    assert np.max(np.abs(psi - D.ccz(1, 3, 5, N_D) @ st)) < 1e-14
    psi = st.copy()
    O.apply_toffoli_psi(psi, 4, 2, 1, N_D)
    assert np.max(np.abs(psi - D.toffoli(4, 2, 1, N_D) @ st)) < 1e-14


def test_generic_gates_vs_dense(st):
    rng = np.random.default_rng(5)
    U2 = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))[0]
    U4 = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
    SW = np.eye(4)[[0, 2, 1, 3]]
    for k in range(1, N_D + 1):
        psi = st.copy()
        O.apply_one_qubit_gate(psi, U2, k, N_D)
        assert np.max(np.abs(psi - D.embed({k: U2}, N_D) @ st)) < 1e-13
    for a, b in [(1, 2), (2, 5), (5, 1), (4, 3)]:
        lo, hi = min(a, b), max(a, b)
        psi = st.copy()
        O.apply_two_qubit_gate(psi, U4, a, b, N_D)   # Trotter convention: U's bit 0 = min(a, b)
        assert np.max(np.abs(psi - D.two_qubit_local(U4, lo, hi, N_D) @ st)) < 1e-13
        psi = st.copy()
        O.apply_2qubit_gate_ru(psi, U4, a, b, N_D)   # RandomUnitaries: U's bit 0 = a
        assert np.max(np.abs(psi - D.two_qubit_local(U4, a, b, N_D) @ st)) < 1e-13
        if a > b:
            assert np.max(np.abs(D.two_qubit_local(U4, a, b, N_D) - D.two_qubit_local(SW @ U4 @ SW, b, a, N_D))) < 1e-14


def test_observables_vs_dense(st):
    for k in range(1, N_D + 1):
        for p, M in (("x", D.X), ("y", D.Y), ("z", D.Z)):
            assert abs(O.expect_local(st, k, N_D, p) - D.expect(st, {k: M}, N_D)) < 1e-13
    for a in range(1, N_D + 1):
        for b in range(1, N_D + 1):
            if a != b:
                for p, M in (("xx", D.X), ("yy", D.Y), ("zz", D.Z)):
                    assert abs(O.expect_corr(st, a, b, N_D, p) - D.expect(st, {a: M, b: M}, N_D)) < 1e-13
    rng = np.random.default_rng(1)
    for _ in range(30):
        n = rng.integers(1, N_D + 1)
        qs = list(rng.choice(np.arange(1, N_D + 1), size=n, replace=False))
        ops = list(rng.choice(["X", "Y", "Z"], size=n))
        want = D.expect(st, {q: {"X": D.X, "Y": D.Y, "Z": D.Z}[o] for q, o in zip(qs, ops)}, N_D)
        assert abs(O.pauli_string(st, ops, [int(q) for q in qs], N_D) - want) < 1e-13
    assert abs(O.population_excited_psi(st, 2, N_D) - D.expect(st, {2: np.diag([0, 1])}, N_D)) < 1e-14


# ------------------------------------------------------------- Trotter
def test_trotter_precompute_closed_form_vs_expm():
    bonds = [(1, 2, 1.0, 1.0, 0.5), (2, 3, 0.3, -0.7, 1.1)]
    fields = [(1, 0.4, 0.0, 0.0), (2, 0.0, 0.0, -0.8), (3, 0.2, 0.5, -0.1), (1, 0.0, 0.0, 0.0)]
    dt = 0.05
    arr, n = O.precompute_trotter_gates(bonds, fields, dt)
    assert n == 5  # the all-zero field is dropped (Trotter.jl:346)
    gl = O.gates_to_list(arr, n)
    XX, YY, ZZ = np.kron(D.X, D.X), np.kron(D.Y, D.Y), np.kron(D.Z, D.Z)
    for (idx, U), (i, j, jx, jy, jz) in zip(gl[:2], bonds):
        assert idx == [i, j]
        assert np.max(np.abs(U - D.expm_herm(jx * XX + jy * YY + jz * ZZ, dt))) < 1e-14
    for (idx, U), (q, hx, hy, hz) in zip(gl[2:], fields[:3]):
        assert idx == [q]
        assert np.max(np.abs(U - D.expm_herm(hx * D.X + hy * D.Y + hz * D.Z, dt))) < 1e-14


def test_trotter_step_vs_dense():
    N = 4
    rng = np.random.default_rng(2)
    bonds = [(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)]
    fields = [(i, 0.0, 0.0, rng.uniform(-1, 1)) for i in range(1, N + 1)]
    arr, n = O.precompute_trotter_gates(bonds, fields, 0.05)
    psi = D.random_state(N, rng)
    want = psi.copy()
    for idx, U in O.gates_to_list(arr, n):
        M = D.embed({idx[0]: U}, N) if len(idx) == 1 else D.two_qubit_local(U, idx[0], idx[1], N)
        want = M @ want
    O.trotter_step(psi, arr, n, N)
    assert np.max(np.abs(psi - want)) < 1e-13


def test_dm_trotter_matches_pure():
    N = 4
    rng = np.random.default_rng(4)
    arr, n = O.precompute_trotter_gates([(i, i + 1, 1, 1, 0.5) for i in range(1, N)],
                                        [(i, 1.0, 0, 0) for i in range(1, N + 1)], 0.05)
    psi = D.random_state(N, rng)
    rho = np.asfortranarray(np.outer(psi, psi.conj()))
    O.trotter_step(psi, arr, n, N)
    O.dm_trotter_step(rho, arr, n, N)
    assert np.max(np.abs(rho - np.outer(psi, psi.conj()))) < 1e-13


# ----------------------------------------------------------- gradients
def test_parameter_shift_vs_finite_difference():
    ka = KA["ps_vs_fd"]
    N, L = 4, 2
    ops = []
    p = 1
    for _ in range(L):
        for q in range(1, N + 1):
            ops.append(("ry", [q], p, 0.0))
            p += 1
        for q in range(1, N):
            ops.append(("cz", [q, q + 1], 0, 0.0))
    for q in range(1, N + 1):
        ops.append(("ry", [q], p, 0.0))
        p += 1
    arr = O.make_ops(ops)
    theta = np.random.default_rng(0).normal(size=p - 1) * 0.1
    terms = [(1.0, {1: "Z"})]   # cost <Z_1> as in demo_VQC_base_test.jl:109-113
    ps = O.grad(arr, len(ops), theta, N, terms, method="ps")
    fd = O.grad(arr, len(ops), theta, N, terms, method="fd", eps=ka["eps"])
    assert np.max(np.abs(ps - fd)) < ka["tol"]


# ---------------------------------------------------------------- RNG
def test_philox_known_answers():
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


# ----------------------------------------------------- MCWF vs density matrix
def test_mcwf_converges_to_dm_small():
    """Statistical parity MCWF <-> density matrix (demo_quantum_channels.jl:413-456 style):
    TFIM N=3, sigma- (0.1) and sigma_z (0.05) on every qubit; trajectory mean within 5 sigma."""
    N, dt, steps, ntraj = 3, 0.01, 100, 3000
    arr, n = O.precompute_trotter_gates([(i, i + 1, 0, 0, 1.0) for i in range(1, N)],
                                        [(i, 1.0, 0, 0) for i in range(1, N + 1)], dt)
    jumps = [(0, q, 0.1) for q in range(1, N + 1)] + [(2, q, 0.05) for q in range(1, N + 1)]
    ja = O.make_jumps(jumps)
    z, zz, nj = O.mcwf_run(N, arr, n, ja, len(jumps), dt, 1234, 0, ntraj, steps, steps, init_index=(1 << N) - 1,
                           nthreads=4)
    rho = np.zeros((1 << N, 1 << N), complex, order="F")
    rho[-1, -1] = 1
    for _ in range(steps):
        O.dm_trotter_step(rho, arr, n, N)
        for j in jumps:
            O.dm_dissipator(rho, j, dt, N)
    for k in range(1, N + 1):
        m, s = z[-1, :, k - 1].mean(), z[-1, :, k - 1].std() / math.sqrt(ntraj)
        assert abs(m - O.dm_expect_z(rho, k, N)) < 5 * s + 2e-3, (k, m, O.dm_expect_z(rho, k, N), s)
    assert nj.sum() > 0


def test_oracle_born_sampling_and_measurement():
    """the oracle's Born sampling reproduces |psi|^2 (chi-square over 40k shots), its
    draws are the Philox stream (u of shot s is the first uniform of counter (s, stream)),
    and _measure_z_single! / projective_measurement_all! collapse as the reference does"""
    N = 8
    rng = np.random.default_rng(3)
    psi = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    psi /= np.linalg.norm(psi)
    p = np.abs(psi) ** 2
    shots = O.sample(psi.copy(), N, 40000, seed=99, stream=5)
    cnt = np.bincount(shots, minlength=1 << N)
    chi2 = np.sum((cnt - 40000 * p) ** 2 / (40000 * p))
    assert chi2 < (1 << N) + 6 * np.sqrt(2 * (1 << N))     # dof = 255, ~6 sigma
    # shot s is the inverse CDF of the Philox uniform of (s, stream)
    cum = np.cumsum(p)
    for s in (0, 1, 7, 1234):
        w = O.philox([s & 0xFFFFFFFF, s >> 32, 5, 0], [99, 0])
        u = ((w[0] >> 5) * 67108864 + (w[1] >> 6)) / 9007199254740992.0
        assert shots[s] == min(int(np.searchsorted(cum, u, side="left")), (1 << N) - 1)
    # single-qubit measurement: outcome by u < P(0), collapse, renormalise
    q = 3
    phi = psi.copy()
    o = O.measure_qubit(phi, q, N, seed=7, stream=2)
    bits = (np.arange(1 << N) >> (q - 1)) & 1
    want = np.where(bits == o, psi, 0)
    want /= np.linalg.norm(want)
    assert np.allclose(phi, want, atol=1e-14)
    # all-qubit measurement: a basis state
    phi = psi.copy()
    idx = O.measure_all(phi, N, seed=7, stream=2)
    assert phi[idx] == 1 and np.count_nonzero(phi) == 1


def test_dm_superoperator_algebra_matches_dense_lindblad():
    """The 4x4 (row bit, column bit) map the GPU density-matrix plan applies per jump
    equals one Euler step rho + gamma dt (L rho L^dag - {L^dag L, rho}/2) of the dense
    matrices, which the oracle's _apply_dissipator_dm! restatement also matches."""
    N, dt, gamma = 3, 0.05, 0.4
    rng = np.random.default_rng(8)
    A = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
    rho0 = A @ A.conj().T
    rho0 /= np.trace(rho0)
    Ls = {0: np.array([[0, 1], [0, 0]], complex), 1: np.array([[0, 0], [1, 0]], complex),
          2: np.diag([1.0, -1.0]).astype(complex), 3: np.array([[0, 1], [1, 0]], complex)}
    for ty, L in Ls.items():
        for q in (1, 2, 3):
            Lf = D.embed({q: L}, N)
            want = rho0 + gamma * dt * (Lf @ rho0 @ Lf.conj().T - 0.5 * (Lf.conj().T @ Lf @ rho0 + rho0 @ Lf.conj().T @ Lf))
            got = np.asfortranarray(rho0.copy())
            O.dm_dissipator(got, (ty, q, gamma), dt, N)
            assert np.max(np.abs(got - want)) < 1e-13, (ty, q)


def test_oracle_hamiltonian_apply_vs_dense_and_lanczos():
    """the oracle's restatement of apply_hamiltonian_bitwise! equals the dense
    Pauli sum (Y the Pauli Y, as construct_sparse_hamiltonian builds it,
    cpuHamiltonianBuilder.jl:297), and equals its restatement of apply_H_xxz!
    (cpuQuantumStateLanczos.jl:157) for the same chain"""
    import dense_ref as Dr
    N = 6
    rng = np.random.default_rng(9)
    psi = Dr.random_state(N, rng)
    xb = [[i, i + 1, *rng.normal(size=3)] for i in range(1, N)]
    yb = [[1, 4, 0.2, -0.6, 0.4]]
    fields = [[i, *rng.normal(size=3)] for i in range(1, N + 1)]
    Hd = np.zeros((1 << N, 1 << N), complex)
    pm = {"X": Dr.X, "Y": Dr.Y, "Z": Dr.Z}
    for i, j, jx, jy, jz in xb + yb:
        for P, c in (("X", jx), ("Y", jy), ("Z", jz)):
            Hd += c * Dr.embed({int(i): pm[P], int(j): pm[P]}, N)
    for k, hx, hy, hz in fields:
        for P, c in (("X", hx), ("Y", hy), ("Z", hz)):
            Hd += c * Dr.embed({int(k): pm[P]}, N)
    got = O.apply_hamiltonian_bitwise(psi, xb, yb, fields, N)
    assert np.max(np.abs(got - Hd @ psi)) < 1e-13
    chain = O.apply_hamiltonian_bitwise(psi, [[i, i + 1, 1.0, 0.8, 0.5] for i in range(1, N)], [],
                                        [[i, 0.3, 0.0, 0.0] for i in range(1, N + 1)], N)
    assert np.max(np.abs(chain - O.apply_H_xxz(psi, N, 1.0, 0.8, 0.5, 0.3))) < 1e-13

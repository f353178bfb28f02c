"""Oracle parity at the sizes the benchmarks measure.

The other GPU tests pin every kernel against the oracle at sizes the oracle
finishes in a second.  These run the measured configurations themselves
through the C ABI and compare with the oracle (oracle/smoq_oracle.c, its
per-state loops on all host threads):

* the Trotter configuration: XXZ chain N=28, one full Strang step (218 gates)
  from the Neel state, complex128 and complex64 (the bench's plan and engine),
  every amplitude and <Z_i>
  (apply_fast_trotter_step_cpu!, utils/cpu/cpuQuantumChannelUnitaryEvolutionTrotter.jl:150-162);
* the gradient configuration: N=24, 12 layers of [Ry all; Rz all; CZ ladder]
  (576 parameters): energy and the adjoint gradient of the first, a middle and
  the last layer's Ry and Rz against the oracle's parameter-shift rule
  (calculate_gradients_parameter_shift,
  utils/cpu/cpuVariationalQuantumCircuitGradients.jl:138-163);
* the bandwidth configuration's circuit at N=26, full depth (20 layers of
  Rx/Ry/Rz on every qubit and Rzz on a random perfect matching), both dtypes;
* the 30-32-qubit index paths (qubits 26-31, byte offsets beyond 4 GiB,
  amplitude indices beyond 2^31): H on every qubit, then entangling gates
  on qubits {1, 2, 3, N-3..N} including Rzz(1, N).  The state is the oracle's
  7-qubit state on those qubits times |+> on the others, so every amplitude
  is known; windows at the start, the end and random offsets are compared;
* the bandwidth configuration's first layer at full size (N=32 complex64,
  N=31 complex128): a product state times Rzz phases, checked on windows
  against the product of the oracle's one-qubit states.

Tolerances: complex128 relative L2 error <= 1e-12 (observables 1e-12 absolute);
complex64 relative L2 error <= 2e-5 after hundreds of gates (5e-6 on the
windows of the 30-32-qubit states), observables <= 1e-5, and the gradient
configuration's energy <= 1e-6.
"""
import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu

SEED = 42


def rel_l2(got, ref, chunk=1 << 24):
    """||got - ref|| / ||ref|| in FP64, chunked (states of several GiB)"""
    num = den = 0.0
    for s in range(0, ref.size, chunk):
        r = ref[s:s + chunk]
        d = got[s:s + chunk].astype(np.complex128) - r
        num += float(np.vdot(d, d).real)
        den += float(np.vdot(r, r).real)
    return np.sqrt(num / den)


# ---------------------------------------------------------------- Trotter, N=28
def rpp(P, t):
    return np.cos(t / 2) * np.eye(4) - 1j * np.sin(t / 2) * np.kron(P, P)


def xxz_s1_gates(N, tau, J=1.0, delta=0.5):
    """S1(tau): Rz(2 h_i tau) on every site (h_i ~ U[-1, 1], seed 42), then per bond
    Rxx(2 J tau), Ryy(2 J tau), Rzz(2 J delta tau) -- the benchmark's gate list"""
    X = np.array([[0, 1], [1, 0]], complex)
    Y = np.array([[0, -1j], [1j, 0]], complex)
    Z = np.diag([1.0 + 0j, -1.0])
    h = np.random.default_rng(SEED).uniform(-1, 1, size=N)
    g = [([i + 1], np.diag([np.exp(-1j * h[i] * tau), np.exp(1j * h[i] * tau)])) for i in range(N)]
    for i in range(1, N):
        g += [([i, i + 1], rpp(X, 2 * J * tau)), ([i, i + 1], rpp(Y, 2 * J * tau)),
              ([i, i + 1], rpp(Z, 2 * J * delta * tau))]
    return g


def test_trotter_configuration_n28_one_strang_step_vs_oracle(ctx):
    N, dt = 28, 0.05
    gl = xxz_s1_gates(N, dt / 2)
    both = gl + gl[::-1]
    assert len(both) == 218
    neel = sum(1 << (k - 1) for k in range(1, N + 1, 2))
    ref = O.zero_state(N, neel)
    with O.threads():
        O.trotter_step(ref, O.make_gates(both), len(both), N)
        z_ref = np.array([O.expect_local(ref, k, N, "z") for k in range(1, N + 1)])
    gates = [S.FastTrotterGate(idx, U) for idx, U in gl]
    for dtype, tol_psi, tol_z in ((S.C128, 1e-12, 1e-12), (S.C64, 2e-5, 1e-5)):
        plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=dtype)
        st = S.CuState(ctx, N, dtype, basis=neel)
        rec = plan.run(st, 1, 1)          # <Z_i> at t = 0 and after the step
        got = st.download()
        st.close()
        plan.close()
        err = rel_l2(got, ref)
        zerr = float(np.max(np.abs(rec[1, 0, :] - z_ref)))
        print(f"N=28 Strang step dtype={dtype}: rel L2 {err:.2e}, max |dZ| {zerr:.2e}")
        assert err <= tol_psi and zerr <= tol_z, (dtype, err, zerr)
        del got


# ---------------------------------------------------------------- gradient, N=24
def hea(N, L, seed=SEED):
    ops, idx = [], 1
    for _ in range(L):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
    theta = np.random.default_rng(seed).uniform(0, 2 * np.pi, size=idx - 1)
    return S.ParameterizedCircuit(N, ops), theta


def tfim_terms(N):
    return [(-1.0, {i: "Z", i + 1: "Z"}) for i in range(1, N)] + [(-1.0, {i: "X"}) for i in range(1, N + 1)]


def test_gradient_configuration_n24_vs_oracle_parameter_shift(ctx):
    N, L = 24, 12
    circ, theta = hea(N, L)
    assert circ.n_params == 576
    terms = tfim_terms(N)
    oo = [(op.type, op.qubits, op.param_idx, op.fixed_angle) for op in circ.operations]
    arr = O.make_ops(oo)
    # parameters: layer l holds Ry(q=1..24) at 48 l + q - 1, then Rz(q=1..24) at 48 l + 24 + q - 1
    which = np.array([0, 47, 48 * 6 + 5, 48 * 6 + 30, 48 * 11 + 23, 48 * 11 + 24])
    with O.threads():
        e_ref = O.energy(arr, len(oo), theta, N, terms)
        ps = O.grad(arr, len(oo), theta, N, terms, which=which, method="ps")
    H = S.PauliSum(terms)
    e128, g128 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    e64, g64 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C64)
    print(f"N=24 vs oracle: energy c128 {abs(e128[0] - e_ref):.2e} c64 {abs(e64[0] - e_ref):.2e}; "
          f"gradient c128 {np.max(np.abs(g128[0][which] - ps)):.2e} c64 {np.max(np.abs(g64[0][which] - ps)):.2e}")
    assert abs(e128[0] - e_ref) < 1e-11
    assert np.max(np.abs(g128[0][which] - ps)) < 1e-10
    assert abs(e64[0] - e_ref) <= 1e-6
    assert np.max(np.abs(g64[0][which] - ps)) < 1e-5


# ---------------------------------------------------------------- bandwidth circuit, N=26
def bandwidth_ops(N, layers, seed=SEED):
    """20 layers of [Rx, Ry, Rz on every qubit (seeded angles); Rzz on a seeded
    random perfect matching] -- the 32 GiB sweep's circuit at any N"""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(layers):
        for g in ("rx", "ry", "rz"):
            ops += [S.gate(g, q, angle=float(rng.uniform(0, 2 * np.pi))) for q in range(1, N + 1)]
        perm = rng.permutation(N) + 1
        ops += [S.gate("rzz", [int(perm[2 * i]), int(perm[2 * i + 1])], angle=float(rng.uniform(0, 2 * np.pi)))
                for i in range(N // 2)]
    return ops


def z_masks(N):
    return [1 << q for q in range(N)] + [3 << q for q in range(N - 1)]


def zstrings(st, masks):
    return np.concatenate([S.expect_zstrings(st, masks[i:i + 32])[0] for i in range(0, len(masks), 32)])


def test_bandwidth_circuit_n26_full_depth_vs_oracle(ctx):
    N = 26
    ops = bandwidth_ops(N, 20)
    circ = S.ParameterizedCircuit(N, ops)
    oo = [(op.type, op.qubits, op.param_idx, op.fixed_angle) for op in ops]
    ref = O.zero_state(N, 0)
    masks = z_masks(N)
    with O.threads():
        O.apply_circuit(ref, O.make_ops(oo), len(oo), np.zeros(1), N)
        obs_ref = np.array([O.expect_local(ref, k, N, "z") for k in range(1, N + 1)] +
                           [O.expect_corr(ref, k, k + 1, N, "zz") for k in range(1, N)])
    for dtype, engine, tol_psi, tol_obs in ((S.C128, -1, 1e-12, 1e-12), (S.C64, -1, 2e-5, 1e-5),
                                            (S.C64, 3, 2e-5, 1e-5)):
        c = S.Context(0)
        if engine >= 0:
            if engine == 3 and not S.jit_available():
                c.close()
                continue
            c.set_option(S._lib.OPT_ENGINE, engine)
        st = S.CuState(c, N, dtype, basis=0)
        S.apply_circuit(st, circ, np.zeros(1))
        obs = zstrings(st, masks)
        err = rel_l2(st.download(), ref)
        st.close()
        c.close()
        oerr = float(np.max(np.abs(obs - obs_ref)))
        print(f"N=26 depth 20 dtype={dtype} engine={engine}: rel L2 {err:.2e}, max |d obs| {oerr:.2e}")
        assert err <= tol_psi and oerr <= tol_obs, (dtype, engine, err, oerr)


# ---------------------------------------------------------------- 30-32 qubits
def windows(N, rng, width=1 << 18):
    dim = 1 << N
    starts = [0, dim - width, dim // 2 - width // 2] + [int(x) for x in rng.integers(0, dim - width, size=3)]
    return [(s, width) for s in starts]


def compress(idx, qubits):
    """bits of the 1-based `qubits` of each index, packed in that order"""
    c = np.zeros(idx.shape, dtype=np.int64)
    for t, q in enumerate(qubits):
        c |= ((idx >> (q - 1)) & 1) << t
    return c


@pytest.mark.parametrize("N,dtype", [(30, S.C64), (31, S.C128), (32, S.C64)])
def test_high_qubit_index_paths_vs_oracle(ctx, N, dtype):
    sub = [1, 2, 3, N - 3, N - 2, N - 1, N]
    pos = {q: t + 1 for t, q in enumerate(sub)}       # full qubit -> oracle qubit
    g = S.gate
    body = [g("rx", N, angle=0.7), g("ry", N - 1, angle=1.1), g("rz", N - 2, angle=-0.4), g("t", N - 3),
            g("rzz", [1, N], angle=0.9), g("cnot", [N, 1]), g("rxx", [2, N - 1], angle=0.5),
            g("cz", [3, N - 2]), g("ryy", [N - 3, N], angle=-1.3), g("ry", 1, angle=0.3),
            g("cnot", [2, N - 3]), g("h", N - 1), g("rzz", [N - 2, 2], angle=0.8), g("rx", 3, angle=2.1),
            g("cry", [N - 1, 3], angle=0.6)]
    ops = [g("h", q) for q in range(1, N + 1)] + body
    M = len(sub)
    chi = O.zero_state(M, 0)
    oo = [("h", [q], 0, 0.0) for q in range(1, M + 1)] + \
         [(op.type, [pos[q] for q in op.qubits], op.param_idx, op.fixed_angle) for op in body]
    O.apply_circuit(chi, O.make_ops(oo), len(oo), np.zeros(1), M)
    scale = 2.0 ** (-(N - M) / 2)
    st = S.CuState(ctx, N, dtype, basis=0)
    S.apply_circuit(st, S.ParameterizedCircuit(N, ops), np.zeros(1))
    tol = 1e-12 if dtype == S.C128 else 5e-6
    rng = np.random.default_rng(N)
    worst = 0.0
    for s, w in windows(N, rng):
        got = st.download_range(s, w).astype(np.complex128)
        want = chi[compress(np.arange(s, s + w, dtype=np.int64), sub)] * scale
        worst = max(worst, float(np.linalg.norm(got - want) / np.linalg.norm(want)))
    # Z observables: <Z_k> from chi on the entangled qubits, 0 on the |+> qubits
    masks = [1 << (q - 1) for q in sub] + [(1 << 0) | (1 << (N - 1)), 1 << 10, 0]
    obs = S.expect_zstrings(st, masks)[0]
    want_obs = [O.expect_local(chi, pos[q], M, "z") for q in sub] + [O.expect_corr(chi, 1, M, M, "zz"), 0.0, 1.0]
    oerr = float(np.max(np.abs(obs - np.array(want_obs))))
    st.close()
    print(f"N={N} dtype={dtype}: window rel L2 {worst:.2e}, max |d obs| {oerr:.2e}")
    assert worst <= tol and oerr <= (1e-12 if dtype == S.C128 else 1e-5), (worst, oerr)


@pytest.mark.parametrize("N,dtype", [(32, S.C64), (31, S.C128)])
def test_bandwidth_first_layer_full_size_vs_oracle(ctx, N, dtype):
    """the 32 GiB configurations' first layer: Rx, Ry, Rz on every qubit, then Rzz
    on a random perfect matching.  Amplitude i = prod_k phi_k[bit_k(i)] times the
    Rzz phases, phi_k = Rz Ry Rx |0> from the oracle's one-qubit gates."""
    ops = bandwidth_ops(N, 1)
    phi = np.zeros((N, 2), dtype=np.complex128)
    for k in range(N):
        v = O.zero_state(1, 0)
        for op in ops[k::N][:3]:                 # Rx, Ry, Rz of qubit k + 1
            assert op.qubits == [k + 1]
            O.apply_circuit(v, O.make_ops([(op.type, [1], 0, op.fixed_angle)]), 1, np.zeros(1), 1)
        phi[k] = v
    pairs = [(op.qubits[0], op.qubits[1], op.fixed_angle) for op in ops[3 * N:]]
    st = S.CuState(ctx, N, dtype, basis=0)
    S.apply_circuit(st, S.ParameterizedCircuit(N, ops), np.zeros(1))
    tol = 1e-12 if dtype == S.C128 else 5e-6
    rng = np.random.default_rng(N + 100)
    worst = 0.0
    for s, w in windows(N, rng):
        idx = np.arange(s, s + w, dtype=np.int64)
        want = np.ones(w, dtype=np.complex128)
        for k in range(N):
            want *= phi[k][(idx >> k) & 1]
        for a, b, th in pairs:
            same = ((idx >> (a - 1)) & 1) == ((idx >> (b - 1)) & 1)
            want *= np.where(same, np.exp(-0.5j * th), np.exp(0.5j * th))
        got = st.download_range(s, w).astype(np.complex128)
        worst = max(worst, float(np.linalg.norm(got - want) / np.linalg.norm(want)))
    # <Z_k> of the product state (the Rzz phases leave the diagonal alone); <Z_k Z_l> = <Z_k><Z_l>
    z = np.abs(phi[:, 0]) ** 2 - np.abs(phi[:, 1]) ** 2
    masks = [1 << k for k in range(24)] + [3 << k for k in range(N - 8, N - 1)]
    want_obs = np.concatenate([z[:24], [z[k] * z[k + 1] for k in range(N - 8, N - 1)]])
    obs = S.expect_zstrings(st, masks)[0]
    st.close()
    oerr = float(np.max(np.abs(obs - want_obs)))
    print(f"N={N} first layer dtype={dtype}: window rel L2 {worst:.2e}, max |d obs| {oerr:.2e}")
    assert worst <= tol and oerr <= (1e-12 if dtype == S.C128 else 1e-5), (worst, oerr)

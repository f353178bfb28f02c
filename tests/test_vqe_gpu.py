"""GPU parity of the VQE energy and the adjoint gradient.

The oracle's energy (so_energy) and its gradients -- the parameter-shift rule
(calculate_gradients_parameter_shift, cpuVariationalQuantumCircuitGradients.jl:138)
and central finite differences (calculate_gradients_finite_difference, :250) --
are the references.  The gradient configuration: TFIM H = -sum Z_i Z_{i+1} -
sum X_i, 12 layers of [Ry all; Rz all; CZ ladder] on N=24 (576 parameters),
complex64 and complex128."""
import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


def hea(N, L, seed=42):
    ops, idx = [], 1
    for _ in range(L):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
    theta = np.random.default_rng(seed).uniform(0, 2 * np.pi, size=idx - 1)
    return S.ParameterizedCircuit(N, ops), theta


def tfim_terms(N):
    return [(-1.0, {i: "Z", i + 1: "Z"}) for i in range(1, N)] + [(-1.0, {i: "X"}) for i in range(1, N + 1)]


def oracle_ops(circ):
    return [(op.type, op.qubits, op.param_idx, op.fixed_angle) for op in circ.operations]


@pytest.mark.parametrize("N,L", [(4, 2), (8, 3), (11, 2)])
def test_energy_and_adjoint_gradient_vs_oracle(ctx, N, L):
    circ, theta = hea(N, L)
    terms = tfim_terms(N)
    H = S.PauliSum(terms)
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    e_ref = O.energy(arr, len(oo), theta, N, terms)
    ps = O.grad(arr, len(oo), theta, N, terms, method="ps")
    fd = O.grad(arr, len(oo), theta, N, terms, method="fd", eps=1e-4)
    assert np.max(np.abs(ps - fd)) < 1e-6           # the two oracle gradients agree
    e, g = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    assert abs(e[0] - e_ref) < 1e-11
    assert np.max(np.abs(g[0] - ps)) < 1e-10
    e64, g64 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C64)
    assert abs(e64[0] - e_ref) < 1e-5
    assert np.max(np.abs(g64[0] - ps)) < 1e-4
    assert abs(S.energy(ctx, circ, H, theta, dtype=S.C128)[0] - e_ref) < 1e-11


def test_all_generator_types_and_shared_parameters(ctx):
    """RX, RY, RZ, RXX, RYY, RZZ, CRY with parameters (one shared by two gates),
    mixed with fixed H, CNOT, S, T, CZ; Pauli terms with X, Y and Z."""
    N = 7
    g = S.gate
    ops = [g("h", 1), g("rx", 2, param_idx=1), g("ry", 3, param_idx=2), g("cnot", [1, 4]),
           g("rz", 4, param_idx=3), g("rxx", [2, 5], param_idx=4), g("s", 6), g("ryy", [5, 6], param_idx=5),
           g("t", 7), g("rzz", [3, 7], param_idx=6), g("cry", [2, 6], param_idx=7), g("cz", [1, 7]),
           g("rx", 5, param_idx=1), g("ry", 1, param_idx=8), g("cnot", [7, 2]), g("rz", 3, param_idx=2)]
    circ = S.ParameterizedCircuit(N, ops)
    theta = np.random.default_rng(3).uniform(-2, 2, size=circ.n_params)
    terms = [(0.7, {1: "X", 2: "Y"}), (-1.1, {3: "Z", 7: "Z"}), (0.4, {4: "Y"}), (0.25, {2: "X", 5: "Z", 6: "Y"}),
             (-0.3, {1: "Z"})]
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    e_ref = O.energy(arr, len(oo), theta, N, terms)
    fd = O.grad(arr, len(oo), theta, N, terms, method="fd", eps=1e-5)
    e, gr = S.energy_and_gradient(ctx, circ, S.PauliSum(terms), theta, dtype=S.C128)
    assert abs(e[0] - e_ref) < 1e-12
    assert np.max(np.abs(gr[0] - fd)) < 1e-7


@pytest.mark.parametrize("seed", [11, 12])
def test_all_generator_types_across_tiles(ctx, seed):
    """N=14 (several tiles at both precisions): a random circuit of every
    parameterised type on random qubits in both orders, fixed gates between,
    and runs where a gate directly precedes another parameterised gate on the
    same qubits (the measurement folds the gate into its sweep); gradient
    against the oracle's central differences."""
    N = 14
    rng = np.random.default_rng(seed)
    g = S.gate
    ops, p = [], 1
    one = ["rx", "ry", "rz"]
    two = ["rxx", "ryy", "rzz", "cry"]
    fixed1, fixed2 = ["h", "s", "t", "x"], ["cnot", "cz"]
    for _ in range(60):
        kind = rng.integers(0, 6)
        q1 = int(rng.integers(1, N + 1))
        q2 = int(rng.choice([q for q in range(1, N + 1) if q != q1]))
        if kind == 0:
            ops.append(g(str(rng.choice(one)), q1, param_idx=p)); p += 1
        elif kind == 1:
            ops.append(g(str(rng.choice(two)), [q1, q2], param_idx=p)); p += 1
        elif kind == 2:   # two parameterised gates on the same qubit(s), back to back
            ops.append(g(str(rng.choice(one)), q1, param_idx=p))
            ops.append(g(str(rng.choice(one)), q1, param_idx=p + 1)); p += 2
        elif kind == 3:
            ops.append(g(str(rng.choice(two)), [q1, q2], param_idx=p))
            ops.append(g(str(rng.choice(two)), [q2, q1], param_idx=p + 1)); p += 2
        elif kind == 4:
            ops.append(g(str(rng.choice(fixed1)), q1))
        else:
            ops.append(g(str(rng.choice(fixed2)), [q1, q2]))
    circ = S.ParameterizedCircuit(N, ops)
    theta = rng.uniform(-3, 3, size=circ.n_params)
    terms = [(0.9, {1: "X", 9: "Y"}), (-0.6, {3: "Z", 14: "Z"}), (0.5, {12: "Y"}), (0.3, {2: "X", 7: "Z", 13: "Y"}),
             (-0.4, {5: "Z"})]
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    e_ref = O.energy(arr, len(oo), theta, N, terms)
    fd = O.grad(arr, len(oo), theta, N, terms, method="fd", eps=1e-5)  # (CRY has no two-term shift rule)
    e, gr = S.energy_and_gradient(ctx, circ, S.PauliSum(terms), theta, dtype=S.C128)
    assert abs(e[0] - e_ref) < 1e-11
    assert np.max(np.abs(gr[0] - fd)) < 1e-7
    e64, g64 = S.energy_and_gradient(ctx, circ, S.PauliSum(terms), theta, dtype=S.C64)
    assert abs(e64[0] - e_ref) < 1e-5
    assert np.max(np.abs(g64[0] - fd)) < 1e-4


def test_batch_of_parameter_sets(ctx):
    N, L, B = 9, 2, 4
    circ, _ = hea(N, L)
    rng = np.random.default_rng(5)
    thetas = rng.uniform(0, 2 * np.pi, size=(B, circ.n_params))
    H = S.PauliSum(tfim_terms(N))
    e, g = S.energy_and_gradient(ctx, circ, H, thetas, dtype=S.C128)
    for b in range(B):
        e1, g1 = S.energy_and_gradient(ctx, circ, H, thetas[b], dtype=S.C128)
        assert abs(e[b] - e1[0]) < 1e-13 and np.max(np.abs(g[b] - g1[0])) < 1e-13


def test_gradient_configuration_n24(ctx):
    """N=24, 12 layers, 576 parameters: the complex64 adjoint agrees with the
    complex128 adjoint, and the complex128 adjoint with a GPU complex128
    parameter-shift gradient on a fixed subset of 16 parameters."""
    N, L = 24, 12
    circ, theta = hea(N, L)
    assert circ.n_params == 576 and len(circ.operations) == 852
    H = S.PauliSum(tfim_terms(N))
    e128, g128 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    e64, g64 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C64)
    print(f"N=24 energy c64-c128 {abs(e64[0] - e128[0]):.2e}, gradient {np.max(np.abs(g64[0] - g128[0])):.2e}")
    # the batched complex64 target: energy error <= 1e-6 against complex128
    assert abs(e64[0] - e128[0]) <= 1e-6, abs(e64[0] - e128[0])
    assert np.max(np.abs(g64[0] - g128[0])) < 1e-5
    idx = np.linspace(0, 575, 16).astype(int)
    shifted = np.repeat(theta[None, :], 32, axis=0)
    for k, p in enumerate(idx):
        shifted[2 * k, p] += np.pi / 2
        shifted[2 * k + 1, p] -= np.pi / 2
    es = S.energy(ctx, circ, H, shifted, dtype=S.C128)
    ps = (es[0::2] - es[1::2]) / 2
    assert np.max(np.abs(g128[0][idx] - ps)) < 1e-9


def test_many_independent_circuits_vs_oracle(ctx):
    """a batch of different circuits (sizes 5-14, depths 1-4, own Hamiltonians and
    parameters) through smoq_energy_grad_jobs: every energy and gradient equals
    the oracle's (energy, parameter-shift gradient) for that circuit"""
    rng = np.random.default_rng(7)
    jobs, refs = [], []
    for j in range(12):
        N = int(rng.integers(5, 12)) if j < 10 else 13 + (j - 10)   # the last two span several tiles
        L = int(rng.integers(1, 5)) if j < 10 else 2
        circ, theta = hea(N, L, seed=100 + j)
        terms = tfim_terms(N)
        if j % 3 == 1:  # a different Hamiltonian for some jobs: XX bonds and Z fields
            terms = [(0.7, {i: "X", i + 1: "X"}) for i in range(1, N)] + [(-0.3, {i: "Z"}) for i in range(1, N + 1)]
        jobs.append((circ, S.PauliSum(terms), theta))
        oo = oracle_ops(circ)
        arr = O.make_ops(oo)
        refs.append((O.energy(arr, len(oo), theta, N, terms), O.grad(arr, len(oo), theta, N, terms, method="ps")))
    e, g = S.energy_and_gradient_jobs(ctx, jobs, dtype=S.C128)
    for j, (er, gr) in enumerate(refs):
        assert abs(e[j] - er) < 1e-10, j
        assert np.max(np.abs(g[j] - gr)) < 1e-9, j
    e64, g64 = S.energy_and_gradient_jobs(ctx, jobs, dtype=S.C64)
    for j, (er, gr) in enumerate(refs):
        assert abs(e64[j] - er) < 1e-4 and np.max(np.abs(g64[j] - gr)) < 1e-3


def random_circuit(N, rng, n_gates=40):
    """every parameterised type on random qubits (both orders) and fixed gates between"""
    g = S.gate
    ops, p = [], 1
    for _ in range(n_gates):
        kind = rng.integers(0, 5)
        q1 = int(rng.integers(1, N + 1))
        q2 = int(rng.choice([q for q in range(1, N + 1) if q != q1]))
        if kind == 0:
            ops.append(g(str(rng.choice(["rx", "ry", "rz"])), q1, param_idx=p)); p += 1
        elif kind == 1:
            ops.append(g(str(rng.choice(["rxx", "ryy", "rzz", "cry"])), [q1, q2], param_idx=p)); p += 1
        elif kind == 2:
            ops.append(g(str(rng.choice(["h", "s", "t", "x"])), q1))
        elif kind == 3:
            ops.append(g(str(rng.choice(["cnot", "cz"])), [q1, q2]))
        else:   # a parameter shared by two gates
            ops.append(g("ry", q1, param_idx=max(1, p - 1)))
    return S.ParameterizedCircuit(N, ops)


@pytest.mark.parametrize("dtype,tol", [(S.C128, 1e-11), (S.C64, 2e-5)])
def test_jobs_in_one_launch_equal_the_tiled_path(built, dtype, tol):
    """smoq_energy_grad_jobs runs circuits that fit one CTA's shared memory in one
    launch; the same jobs with that path switched off (every circuit through the
    tiled passes, one after another) give the same energies and gradients, and
    a job list mixing both kinds keeps every job's outputs in place"""
    rng = np.random.default_rng(21)
    jobs, raw = [], []
    for j in range(24):
        N = [1, 2, 3, 5, 8, 11, 12, 13, 14][j % 9]
        circ = random_circuit(N, rng, n_gates=int(rng.integers(1, 50))) if N > 1 else \
            S.ParameterizedCircuit(1, [S.gate("rx", 1, param_idx=1), S.gate("ry", 1, param_idx=2)])
        theta = rng.uniform(-3, 3, size=circ.n_params)
        terms = [(float(rng.normal()), {int(q): str(rng.choice(["X", "Y", "Z"]))
                                        for q in rng.choice(np.arange(1, N + 1), size=min(N, 2), replace=False)})
                 for _ in range(3)]
        jobs.append((circ, S.PauliSum(terms), theta))
        raw.append(terms)
    res = {}
    for resident in (1, 0):
        c = S.Context(0)
        c.set_option(S._lib.OPT_VQE_RESIDENT, resident)
        res[resident] = S.energy_and_gradient_jobs(c, jobs, dtype=dtype)
        e_only, _ = S.energy_and_gradient_jobs(c, jobs, dtype=dtype, gradient=False)
        assert np.max(np.abs(e_only - res[resident][0])) < tol
        c.close()
    (e1, g1), (e0, g0) = res[1], res[0]
    assert np.max(np.abs(e1 - e0)) < tol
    for a, b in zip(g1, g0):
        assert a.shape == b.shape and (a.size == 0 or np.max(np.abs(a - b)) < tol)
    # and one small job against the oracle's central differences
    circ, H, theta = jobs[4]  # N = 8
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    fd = O.grad(arr, len(oo), theta, circ.N, raw[4], method="fd", eps=1e-5)
    assert np.max(np.abs(g1[4] - fd)) < (1e-7 if dtype == S.C128 else 1e-4)


@pytest.mark.parametrize("N,seed", [(13, 21), (17, 22), (20, 23)])
def test_compiled_adjoint_matches_shared_memory_adjoint(ctx, N, seed):
    """complex64 forward and backward passes run as compiled kernels with run-time
    coefficients (engine auto) or as shared-memory sweeps (engine 0): every
    parameterised type, fixed 1-3 qubit gates (Toffoli, CCZ: single-op stages)
    between; both agree, and both agree with the oracle's complex128 gradient; a
    second parameter set reuses the compiled kernels (their source holds no angle)
    and still matches"""
    if not S.jit_available():
        pytest.skip("NVRTC not available")
    rng = np.random.default_rng(seed)
    g = S.gate
    ops, p = [], 1
    for _ in range(4 * N):
        kind = rng.integers(0, 6)
        q = [int(x) + 1 for x in rng.choice(N, 3, replace=False)]
        if kind == 0:
            ops.append(g(str(rng.choice(["rx", "ry", "rz"])), q[0], param_idx=p)); p += 1
        elif kind == 1:
            ops.append(g(str(rng.choice(["rxx", "ryy", "rzz", "cry"])), q[:2], param_idx=p)); p += 1
        elif kind == 2:
            ops.append(g(str(rng.choice(["h", "s", "t", "x"])), q[0]))
        elif kind == 3:
            ops.append(g(str(rng.choice(["cnot", "cz"])), q[:2]))
        elif kind == 4:
            ops.append(g(str(rng.choice(["toffoli", "ccz"])), q))
        else:
            ops.append(g("ry", q[0], param_idx=p))
            ops.append(g("rzz", q[:2], param_idx=p + 1)); p += 2
    circ = S.ParameterizedCircuit(N, ops)
    terms = [(0.9, {1: "X", N: "Y"}), (-0.6, {3: "Z", N - 1: "Z"}), (0.5, {N // 2: "Y"}), (-0.4, {5: "Z"})]
    H = S.PauliSum(terms)
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    for k in range(2):
        theta = rng.uniform(-3, 3, size=circ.n_params)
        ctx.set_option(S._lib.OPT_ENGINE, -1)
        ctx.reset_counters()
        e_c, g_c = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C64)
        ctx.set_option(S._lib.OPT_ENGINE, 0)
        try:
            e_s, g_s = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C64)
        finally:
            ctx.set_option(S._lib.OPT_ENGINE, -1)
        e_ref = O.energy(arr, len(oo), theta, N, terms)
        fd = O.grad(arr, len(oo), theta, N, terms, method="fd", eps=1e-5)
        print(f"N={N} set {k}: compiled vs shared-memory adjoint {np.max(np.abs(g_c[0] - g_s[0])):.2e}, "
              f"vs oracle {np.max(np.abs(g_c[0] - fd)):.2e}")
        assert abs(e_c[0] - e_s[0]) < 2e-6      # (complex64 forwards of different fusion)
        assert np.max(np.abs(g_c[0] - g_s[0])) < 2e-5
        assert abs(e_c[0] - e_ref) < 1e-5 and np.max(np.abs(g_c[0] - fd)) < 1e-4


def test_compiled_adjoint_batch_and_special_angles(ctx):
    """a batch of complex64 parameter sets through one compiled kernel per pass
    (each set equals its own call), and angles that make coefficients 0 or +-1
    (theta = 0, pi: another kernel source) against the complex128 gradient"""
    N, L = 15, 3
    circ, _ = hea(N, L)
    H = S.PauliSum(tfim_terms(N))
    rng = np.random.default_rng(9)
    thetas = rng.uniform(0, 2 * np.pi, size=(3, circ.n_params))
    thetas[2, ::3] = 0.0
    thetas[2, 1::5] = np.pi
    e, g = S.energy_and_gradient(ctx, circ, H, thetas, dtype=S.C64)
    for b in range(3):
        e1, g1 = S.energy_and_gradient(ctx, circ, H, thetas[b], dtype=S.C64)
        assert abs(e[b] - e1[0]) < 1e-9 and np.max(np.abs(g[b] - g1[0])) < 1e-9
        e2, g2 = S.energy_and_gradient(ctx, circ, H, thetas[b], dtype=S.C128)
        assert abs(e[b] - e2[0]) < 1e-5 and np.max(np.abs(g[b] - g2[0])) < 1e-4


def test_many_circuits_on_worker_streams(ctx):
    """larger circuits of the many-circuit call run on worker contexts from host
    threads, concurrently with the resident launch of the small ones: every job equals
    its own single-circuit call (complex128), and a bad job is reported by its index"""
    rng = np.random.default_rng(31)
    jobs = []
    for j in range(14):
        N = int(rng.integers(14, 17)) if j % 2 == 0 else int(rng.integers(6, 12))
        circ, theta = hea(N, int(rng.integers(1, 4)), seed=200 + j)
        jobs.append((circ, S.PauliSum(tfim_terms(N)), theta))
    e, g = S.energy_and_gradient_jobs(ctx, jobs, dtype=S.C128)
    for j, (circ, H, theta) in enumerate(jobs):
        e1, g1 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
        assert abs(e[j] - e1[0]) < 1e-11 and np.max(np.abs(g[j] - g1[0])) < 1e-10, j
    bad = list(jobs)
    circ, H, theta = bad[4]
    bad[4] = (S.ParameterizedCircuit(circ.N, circ.operations + [S.gate("ry", 1, param_idx=circ.n_params + 1)],
                                     n_params=circ.n_params), H, theta)
    with pytest.raises(S.SmoqError, match="job 4"):
        S.energy_and_gradient_jobs(ctx, bad, dtype=S.C128)
    e2, _ = S.energy_and_gradient_jobs(ctx, jobs, dtype=S.C128)   # the context still works
    assert np.max(np.abs(e2 - e)) < 1e-12

"""Circuits with noise channels, measurements, resets and classical conditions on the GPU
(smoq_apply_circuit_mcwf, the pure-state branch of apply_circuit!,
utils/cpu/cpuVariationalQuantumCircuitExecutor.jl:95-201).

* trajectory-exact: every trajectory of a batch equals the oracle's replay of the
  same op list with the same Philox draws (oracle/smoq_oracle.c
  so_apply_circuit_mcwf): the same measurement outcomes, the same state
  (complex128 <= 1e-12, complex64 <= 2e-5), on one tile and across tiles;
* the trajectory mean of |psi><psi| equals the exact channel evolution of the
  density matrix (gates U rho U^dag, the reference's Kraus channels
  cpuQuantumChannelKrausOperators.jl:84-237, measurement branches, resets,
  conditional gates per branch) within the statistical error;
* errors: a conditional measurement, a probability outside [0, 1], noise in the
  gate-only entry point.
"""
import numpy as np
import pytest

import dense_ref as D
import oracle as O
import pysmoq as S
from pysmoq import _lib as L

pytestmark = pytest.mark.gpu


def noisy_circuit(N, rng, n_ops=60):
    """every op kind on random qubits: gates (parameterised and fixed), all noise
    types, measurements in the three bases, resets to the four targets, and ops
    conditioned on earlier outcomes"""
    g = S.gate
    ops, n_meas, p = [], 0, 1
    for _ in range(n_ops):
        q1 = int(rng.integers(1, N + 1))
        q2 = int(rng.choice([q for q in range(1, N + 1) if q != q1])) if N > 1 else q1
        k = int(rng.integers(0, 12))
        cond = int(rng.integers(1, n_meas + 2)) if (n_meas and rng.random() < 0.3) else 0
        if k == 0:
            ops.append(g(str(rng.choice(["rx", "ry", "rz"])), q1, param_idx=p)); p += 1
        elif k == 1 and N > 1:
            ops.append(g(str(rng.choice(["cnot", "cz", "rxx", "rzz"])), [q1, q2], angle=float(rng.uniform(-3, 3))))
        elif k == 2:
            op = g(str(rng.choice(["h", "x", "s", "t", "y"])), q1)
            op.if_outcome = cond
            ops.append(op)
        elif k in (3, 4):
            kind = str(rng.choice(["depolarizing", "dephasing", "bit_flip", "phase_flip", "phase_damping"]))
            ops.append(S.noise(kind, q1, p=float(rng.uniform(0.05, 0.6)), if_outcome=cond))
        elif k in (5, 6):
            ops.append(S.noise("amplitude_damping", q1, p=float(rng.uniform(0.05, 0.7)), if_outcome=cond))
        elif k in (7, 8):
            ops.append(S.measure(q1, basis=str(rng.choice(["z", "x", "y"]))))
            n_meas += 1
        elif k == 9:
            ops.append(S.reset(q1, target_state=str(rng.choice(["zero", "one", "plus", "minus"])), if_outcome=cond))
        elif k == 10:
            ops.append(S.noise("thermal_relaxation", q1, p=0.3))
        else:
            ops.append(g("ry", q1, angle=float(rng.uniform(-3, 3))))
    return S.ParameterizedCircuit(N, ops)


def oracle_ops(circ):
    out = []
    for op in circ.operations:
        if op.is_gate:
            out.append((op.type, op.qubits, op.param_idx, op.fixed_angle, op.if_outcome))
        elif op.type == "reset":
            out.append(("reset", [op.qubits[0], O.RESET_TARGETS[op.target_state]], 0, 0.0, op.if_outcome))
        else:
            out.append((op.type, op.qubits, 0, op.p, op.if_outcome))
    return out


@pytest.mark.parametrize("N,dtype,tol", [(6, S.C128, 1e-12), (14, S.C128, 1e-12), (6, S.C64, 2e-5),
                                         (15, S.C64, 2e-5)])
def test_trajectories_equal_the_oracle(ctx, N, dtype, tol):
    rng = np.random.default_rng(100 + N)
    circ = noisy_circuit(N, rng)
    theta = rng.uniform(-3, 3, size=max(1, circ.n_params))
    B, seed, off = 24, 77, 1000
    st = S.CuState(ctx, N, dtype, batch=B, basis=None)
    psi0 = np.stack([D.random_state(N, rng) for _ in range(B)])
    st.upload(psi0)
    res = S.apply_circuit(st, circ, theta, seed=seed, traj_offset=off)
    got = st.download()
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    worst, n_meas = 0.0, S.count_measurements(circ.operations)
    assert res.outcomes.shape == (B, n_meas)
    for b in range(B):
        ref = psi0[b].astype(np.complex128).copy()
        out = O.apply_circuit_mcwf(ref, arr, len(oo), theta, N, seed, off + b)
        assert list(res.outcomes[b]) == list(out), b
        worst = max(worst, float(np.max(np.abs(got[b] - ref))))
    print(f"N={N} dtype={dtype}: {B} trajectories x {len(oo)} ops, {n_meas} measurements, max |d psi| {worst:.2e}")
    assert worst <= tol


def unitary_of(op, N):
    """the dense matrix of one gate op, from the oracle's gate loops on basis states"""
    cols = []
    for j in range(1 << N):
        v = O.zero_state(N, j)
        O.apply_circuit(v, O.make_ops([op[:4]]), 1, np.zeros(1), N)
        cols.append(v)
    return np.stack(cols, axis=1)


def on(M, k, N):
    out = np.array([[1.0 + 0j]])
    for q in range(N, 0, -1):
        out = np.kron(out, M if q == k else np.eye(2))
    return out


def channel_kraus(kind, p, k, N):
    X = np.array([[0, 1], [1, 0]], complex)
    Y = np.array([[0, -1j], [1j, 0]], complex)
    Z = np.diag([1.0 + 0j, -1.0])
    I2 = np.eye(2, dtype=complex)
    if kind in ("dephasing", "phase_damping"):
        q = (1 - np.sqrt(1 - p)) / 2
        return [np.sqrt(1 - q) * on(I2, k, N), np.sqrt(q) * on(Z, k, N)]
    if kind == "depolarizing":
        return [np.sqrt(1 - p) * on(I2, k, N)] + [np.sqrt(p / 3) * on(P, k, N) for P in (X, Y, Z)]
    if kind == "bit_flip":
        return [np.sqrt(1 - p) * on(I2, k, N), np.sqrt(p) * on(X, k, N)]
    if kind == "phase_flip":
        return [np.sqrt(1 - p) * on(I2, k, N), np.sqrt(p) * on(Z, k, N)]
    if kind == "amplitude_damping":
        return [on(np.array([[1, 0], [0, np.sqrt(1 - p)]], complex), k, N),
                on(np.array([[0, np.sqrt(p)], [0, 0]], complex), k, N)]
    return [on(I2, k, N)]


def exact_branches(circ, theta, rho0):
    """density-matrix evolution split by measurement history: {outcomes: unnormalised rho}"""
    N = circ.N
    H = np.array([[1, 1], [1, -1]], complex) / np.sqrt(2)
    Sd = np.diag([1, -1j])
    P = [np.diag([1.0 + 0j, 0]), np.diag([0, 1.0 + 0j])]
    br = {(): rho0}
    for op in circ.operations:
        nxt = {}
        for hist, rho in br.items():
            if op.if_outcome and (op.if_outcome > len(hist) or hist[op.if_outcome - 1] != 1):
                nxt[hist] = rho
                continue
            k = op.qubits[0]
            if op.is_gate:
                a = theta[op.param_idx - 1] if op.param_idx > 0 else op.fixed_angle
                U = unitary_of((op.type, op.qubits, 0, a), N)
                nxt[hist] = U @ rho @ U.conj().T
            elif op.type.startswith("measure"):
                pre = {"measure_z": np.eye(2), "measure_x": H, "measure_y": H @ Sd}[op.type]
                B = on(pre, k, N)
                r = B @ rho @ B.conj().T
                for m in (0, 1):
                    Pm = on(P[m], k, N)
                    nxt[hist + (m,)] = B.conj().T @ (Pm @ r @ Pm) @ B
            elif op.type == "reset":
                t = {"zero": np.array([1, 0]), "one": np.array([0, 1]), "plus": np.array([1, 1]) / np.sqrt(2),
                     "minus": np.array([1, -1]) / np.sqrt(2)}[op.target_state]
                F = [on(np.outer(t, [1, 0]), k, N), on(np.outer(t, [0, 1]), k, N)]
                nxt[hist] = sum(f @ rho @ f.conj().T for f in F)
            else:
                nxt[hist] = sum(K @ rho @ K.conj().T for K in channel_kraus(op.type, op.p, k, N))
        br = nxt
    return br


def test_trajectory_mean_equals_the_density_matrix(ctx):
    N, B = 4, 40000
    g = S.gate
    ops = [g("h", 1), g("ry", 2, param_idx=1), g("cnot", [1, 3]), S.noise("depolarizing", 2, p=0.3),
           S.noise("amplitude_damping", 3, p=0.4), g("rx", 4, angle=0.7), S.measure(1, basis="x"),
           g("x", 4, ), S.noise("dephasing", 4, p=0.5, if_outcome=1), S.reset(2, target_state="plus"),
           g("cz", [2, 4]), S.noise("bit_flip", 1, p=0.2), S.measure(3), g("ry", 1, angle=1.1),
           S.noise("phase_flip", 1, p=0.35), g("h", 2, if_outcome=0), S.reset(4, target_state="one", if_outcome=2),
           S.noise("amplitude_damping", 1, p=0.25), g("rzz", [1, 2], angle=0.9)]
    circ = S.ParameterizedCircuit(N, ops)
    theta = np.array([0.8])
    st = S.CuState(ctx, N, S.C128, batch=B, basis=0)
    res = S.apply_circuit(st, circ, theta, seed=2024)
    psi = st.download()
    rho = np.einsum("bi,bj->ij", psi, psi.conj()) / B
    rho0 = np.zeros((1 << N, 1 << N), complex)
    rho0[0, 0] = 1
    br = exact_branches(circ, theta, rho0)
    want = sum(br.values())
    err = float(np.max(np.abs(rho - want)))
    # outcome frequencies per measurement history
    freq = {h: float(np.mean([tuple(o) == h for o in res.outcomes])) for h in br}
    ferr = max(abs(freq[h] - np.trace(r).real) for h, r in br.items())
    print(f"mean over {B} trajectories: max |d rho| {err:.3f}, max |d P(history)| {ferr:.3f}")
    assert err < 0.025 and ferr < 0.025      # about 5 standard errors at 40,000 trajectories


def test_circuit_errors(ctx):
    st = S.CuState(ctx, 3, S.C128, basis=0)
    with pytest.raises(S.SmoqError) as e:
        S.apply_circuit(st, S.ParameterizedCircuit(3, [S.noise("bit_flip", 1, p=1.5)]), np.zeros(1))
    assert e.value.status == L.SMOQ_ERR_BADINPUT
    op = S.measure(1)
    op.if_outcome = 1
    with pytest.raises(S.SmoqError) as e:
        S.apply_circuit(st, S.ParameterizedCircuit(3, [S.measure(2), op]), np.zeros(1))
    assert e.value.status == L.SMOQ_ERR_UNSUPPORTED
    arr, n = S._c_ops([S.noise("dephasing", 1, p=0.1)])
    assert L.lib.smoq_apply_sequence(st.h, arr, n, None) == L.SMOQ_ERR_BADINPUT
    # a condition on a measurement that has not been made never holds (the op is skipped)
    x = S.gate("x", 2)
    x.if_outcome = 1
    S.apply_circuit(st, S.ParameterizedCircuit(3, [x, S.measure(1)]), np.zeros(1))
    assert abs(st.download()[0] - 1) < 1e-14

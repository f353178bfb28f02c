"""Adjoint gradient of noisy circuits along fixed trajectories, with checkpoints
(smoq_energy_grad_mcwf).

With the draws fixed (the Philox streams of smoq_apply_circuit_mcwf), a
trajectory's energy E(theta) = <psi_T|H|psi_T> is a smooth function of theta
between branch thresholds.  The GPU's path-wise adjoint gradient is checked
against the oracle's central finite differences of that same trajectory
(oracle/smoq_oracle.c so_apply_circuit_mcwf + so_pauli_sum_expect, eps = 1e-4,
complex128; calculate_gradients_finite_difference,
utils/cpu/cpuVariationalQuantumCircuitGradients.jl:250).  A parameter whose
two difference quotients (eps 1e-4 and 5e-5) disagree sits next to a branch
threshold and is left out; nearly all are kept.  Checkpointing every branch op
and every third one give the same gradient; a gate-only circuit gives the
noiseless adjoint gradient (smoq_energy_grad).
"""
import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu


def noisy_ansatz(N, L, rng):
    """layers of parameterised rotations and entanglers with every noise kind,
    a mid-circuit measurement with feed-forward and a reset"""
    g = S.gate
    ops, p = [], 1
    for layer in range(L):
        for q in range(1, N + 1):
            ops.append(g(str(rng.choice(["rx", "ry", "rz"])), q, param_idx=p)); p += 1
        for q in range(1, N):
            ops.append(g(str(rng.choice(["cz", "cnot"])), [q, q + 1]))
        ops.append(g(str(rng.choice(["rxx", "ryy", "rzz", "cry"])), [1 + layer % N, 1 + (layer + 2) % N],
                     param_idx=p)); p += 1
        ops.append(S.noise("depolarizing", 1 + layer % N, p=0.2))
        ops.append(S.noise("amplitude_damping", 1 + (layer + 1) % N, p=0.3))
        ops.append(S.noise("dephasing", 1 + (layer + 3) % N, p=0.4))
        if layer == 1:
            ops.append(S.measure(2, basis="x"))
            ops.append(g("ry", 3, param_idx=p, if_outcome=1)); p += 1
        if layer == 2:
            ops.append(S.reset(N, target_state="plus"))
            ops.append(S.noise("bit_flip", N - 1, p=0.25))
    return S.ParameterizedCircuit(N, ops)


def tfim_terms(N):
    return [(-1.0, {i: "Z", i + 1: "Z"}) for i in range(1, N)] + [(-0.7, {i: "X"}) for i in range(1, N + 1)]


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


@pytest.mark.parametrize("N,L", [(5, 4), (11, 3)])
def test_noisy_adjoint_gradient_vs_oracle_finite_differences(ctx, N, L):
    rng = np.random.default_rng(7 + N)
    circ = noisy_ansatz(N, L, rng)
    P = circ.n_params
    theta = rng.uniform(0, 2 * np.pi, size=P)
    terms = tfim_terms(N)
    H = S.PauliSum(terms)
    seed, off, T = 4242, 10, 3
    e, g = S.energy_and_gradient_noisy(ctx, circ, H, theta, seed=seed, traj_offset=off, n_traj=T,
                                       checkpoint_every=1)
    e3, g3 = S.energy_and_gradient_noisy(ctx, circ, H, theta, seed=seed, traj_offset=off, n_traj=T,
                                         checkpoint_every=3)
    assert np.max(np.abs(e3 - e)) < 1e-13 and np.max(np.abs(g3 - g)) < 1e-12
    oo = oracle_ops(circ)
    arr = O.make_ops(oo)
    kept, worst = 0, 0.0
    for t in range(T):
        e_ref = O.noisy_energy(arr, len(oo), theta, N, terms, seed, off + t)
        assert abs(e[t] - e_ref) < 1e-12, (t, e[t], e_ref)
        for k in range(P):
            fd = []
            for eps in (1e-4, 5e-5):
                tp, tm = theta.copy(), theta.copy()
                tp[k] += eps
                tm[k] -= eps
                fd.append((O.noisy_energy(arr, len(oo), tp, N, terms, seed, off + t) -
                           O.noisy_energy(arr, len(oo), tm, N, terms, seed, off + t)) / (2 * eps))
            if abs(fd[0] - fd[1]) > 1e-5:      # a branch threshold inside the step
                continue
            kept += 1
            worst = max(worst, abs(g[t, k] - fd[0]))
    print(f"N={N}: {T} trajectories x {P} parameters, {kept} checked, max |adjoint - FD| {worst:.2e}")
    assert kept >= 0.9 * T * P
    assert worst < 1e-6


def test_gate_only_circuit_matches_the_noiseless_adjoint(ctx):
    rng = np.random.default_rng(3)
    N, g = 7, S.gate
    ops, p = [], 1
    for _ in range(3):
        for q in range(1, N + 1):
            ops.append(g("ry", q, param_idx=p)); p += 1
        ops += [g("cz", [q, q + 1]) for q in range(1, N)]
        ops.append(g("cry", [2, 5], param_idx=p)); p += 1
    circ = S.ParameterizedCircuit(N, ops)
    theta = rng.uniform(0, 2 * np.pi, size=circ.n_params)
    H = S.PauliSum(tfim_terms(N))
    e0, g0 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    e1, g1 = S.energy_and_gradient_noisy(ctx, circ, H, theta, n_traj=1)
    assert abs(e1[0] - e0[0]) < 1e-12 and np.max(np.abs(g1[0] - g0[0])) < 1e-11
    e64, g64 = S.energy_and_gradient_noisy(ctx, circ, H, theta, n_traj=1, dtype=S.C64)
    assert abs(e64[0] - e0[0]) < 1e-5 and np.max(np.abs(g64[0] - g0[0])) < 1e-4

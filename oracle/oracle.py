"""ctypes binding of the CPU oracle (libsmoq_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker.  Never part of the product path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsmoq_oracle.so")


def _ensure_built():
    srcs = [os.path.join(HERE, f) for f in ("smoq_oracle.c", "smoq_oracle.h", "Makefile")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        subprocess.run(["make", "-C", HERE, "-B"], check=True, capture_output=True)


_ensure_built()
L = C.CDLL(LIB_PATH)

_cp = C.c_void_p
_dp = C.POINTER(C.c_double)


class TrotterGate(C.Structure):
    _fields_ = [("nq", C.c_int32), ("q", C.c_int32 * 2), ("pad", C.c_int32), ("U", C.c_double * 32)]


class Op(C.Structure):
    _fields_ = [("type", C.c_int32), ("q", C.c_int32 * 3), ("param", C.c_int32), ("pad", C.c_int32),
                ("angle", C.c_double)]


class JumpOp(C.Structure):
    _fields_ = [("type", C.c_int32), ("qubit", C.c_int32), ("gamma", C.c_double)]


(G_RX, G_RY, G_RZ, G_H, G_X, G_Y, G_Z, G_S, G_SDG, G_T, G_TDG, G_CZ, G_CNOT, G_RXX, G_RYY, G_RZZ,
 G_CRY, G_CCZ, G_TOFFOLI) = range(19)
GATE_CODES = {"rx": G_RX, "ry": G_RY, "rz": G_RZ, "h": G_H, "x": G_X, "y": G_Y, "z": G_Z, "s": G_S,
              "sdg": G_SDG, "t": G_T, "tdg": G_TDG, "cz": G_CZ, "cnot": G_CNOT, "cx": G_CNOT, "rxx": G_RXX,
              "ryy": G_RYY, "rzz": G_RZZ, "cry": G_CRY, "ccz": G_CCZ, "toffoli": G_TOFFOLI}


def _p(a):
    return a.ctypes.data_as(_cp)


def _sig(name, args, res=None):
    f = getattr(L, name)
    f.argtypes = args
    f.restype = res
    return f


for n in ["rx", "ry", "rz"]:
    _sig(f"so_apply_{n}_psi", [_cp, C.c_int, C.c_double, C.c_int])
for n in ["hadamard", "pauli_x", "pauli_y", "pauli_z", "s", "sdagger", "t", "tdagger", "sigma_minus",
          "sigma_plus"]:
    _sig(f"so_apply_{n}_psi", [_cp, C.c_int, C.c_int])
_sig("so_apply_ccz_psi", [_cp, C.c_int, C.c_int, C.c_int, C.c_int])
_sig("so_apply_toffoli_psi", [_cp, C.c_int, C.c_int, C.c_int, C.c_int])
_sig("so_apply_cnot_psi", [_cp, C.c_int, C.c_int, C.c_int])
_sig("so_apply_cz_psi", [_cp, C.c_int, C.c_int, C.c_int])
_sig("so_apply_cry_psi", [_cp, C.c_int, C.c_int, C.c_double, C.c_int])
for n in ["rxx", "ryy", "rzz"]:
    _sig(f"so_apply_{n}_psi", [_cp, C.c_int, C.c_int, C.c_double, C.c_int])
_sig("so_population_excited_psi", [_cp, C.c_int, C.c_int], C.c_double)
_sig("so_apply_one_qubit_gate", [_cp, _dp, C.c_int, C.c_int])
_sig("so_apply_two_qubit_gate", [_cp, _dp, C.c_int, C.c_int, C.c_int])
_sig("so_apply_2qubit_gate_ru", [_cp, _dp, C.c_int, C.c_int, C.c_int])
for n in ["x", "y", "z"]:
    _sig(f"so_expect_{n}", [_cp, C.c_int, C.c_int], C.c_double)
for n in ["xx", "yy", "zz"]:
    _sig(f"so_expect_{n}", [_cp, C.c_int, C.c_int, C.c_int], C.c_double)
_sig("so_expect_pauli_string", [_cp, C.c_int, C.c_char_p, C.POINTER(C.c_int), C.c_int], C.c_double)
_sig("so_norm2", [_cp, C.c_int], C.c_double)
_sig("so_precompute_trotter_gates", [_dp, C.c_int, _dp, C.c_int, C.c_double, C.POINTER(TrotterGate)], C.c_int)
_sig("so_trotter_step", [_cp, C.POINTER(TrotterGate), C.c_int, C.c_int])
_sig("so_apply_circuit", [_cp, C.POINTER(Op), C.c_int, _dp, C.c_int])
_sig("so_pauli_sum_expect", [_cp, C.c_int, _dp, C.c_char_p, C.c_int], C.c_double)
_sig("so_energy", [C.POINTER(Op), C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_char_p], C.c_double)
_sig("so_grad_parameter_shift", [C.POINTER(Op), C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_char_p,
                                 C.c_double, C.POINTER(C.c_int), C.c_int, _dp])
_sig("so_grad_finite_difference", [C.POINTER(Op), C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_char_p,
                                   C.c_double, C.POINTER(C.c_int), C.c_int, _dp])
_sig("so_philox4x32_10", [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)])
_sig("so_sample", [_cp, C.c_int, C.c_int64, C.c_uint64, C.c_uint64, C.POINTER(C.c_int64)])
_sig("so_measure_all", [_cp, C.c_int, C.c_uint64, C.c_uint64], C.c_int64)
_sig("so_measure_qubit", [_cp, C.c_int, C.c_int, C.c_uint64, C.c_uint64], C.c_int)
_sig("so_u01_from_words", [C.c_uint32, C.c_uint32], C.c_double)
_sig("so_mcwf_step", [_cp, C.c_int, C.POINTER(TrotterGate), C.c_int, C.POINTER(JumpOp), C.c_int, C.c_double,
                      C.c_uint64, C.c_uint64, C.c_uint64], C.c_int)
_sig("so_mcwf_run", [C.c_int, C.POINTER(TrotterGate), C.c_int, C.POINTER(JumpOp), C.c_int, C.c_double,
                     C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_uint64, _dp, _dp,
                     C.POINTER(C.c_int), C.c_int])
_sig("so_trotter_step_rho", [_cp, C.POINTER(TrotterGate), C.c_int, C.c_int])
_sig("so_dissipator_dm", [_cp, C.POINTER(JumpOp), C.c_double, C.c_int])
_sig("so_expect_z_rho", [_cp, C.c_int, C.c_int], C.c_double)
_sig("so_expect_zz_rho", [_cp, C.c_int, C.c_int, C.c_int], C.c_double)
_sig("so_wtime", [], C.c_double)
_sig("so_qrc_n_ops", [C.c_int, C.c_int], C.c_int)
_sig("so_measure_all_observables", [_cp, C.c_int, C.c_int, _dp])
_sig("so_qrc_window", [_dp, C.c_int, C.c_int, C.c_int, _dp])
_sig("so_qrc_encode", [_dp, C.c_int, _cp])
_sig("so_qrc_reset", [_cp, _cp, _cp, C.c_int, C.c_int, C.c_double], C.c_int)
_sig("so_qrc_run", [C.c_int, C.POINTER(TrotterGate), C.c_int, C.c_int, C.c_int, C.c_int, _cp, _dp, C.c_int, C.c_int,
                    C.c_uint64, C.c_uint64, _dp, _dp, C.c_int])
_sig("so_qrc_dm_run", [C.c_int, C.POINTER(TrotterGate), C.c_int, C.c_int, C.c_int, C.c_int, _cp, _dp, C.c_int, _dp])
_sig("so_expect_pauli_rho", [_cp, C.c_uint64, C.c_uint64, C.c_int], C.c_double)
for _n in ("dephasing", "depolarizing", "bit_flip", "phase_flip", "amplitude_damping"):
    _sig(f"so_noise_{_n}_u", [_cp, C.c_double, C.c_int, C.c_int, C.c_double])
_sig("so_measure_z_u", [_cp, C.c_int, C.c_int, C.c_double], C.c_int)
_sig("so_reset_u", [_cp, C.c_int, C.c_int, C.c_int, C.c_double])
_sig("so_circuit_draw", [C.c_uint64, C.c_uint32, C.c_uint64], C.c_double)
_sig("so_apply_circuit_mcwf", [_cp, C.POINTER(Op), C.c_int, _dp, C.c_int, C.c_uint64, C.c_uint64,
                               C.POINTER(C.c_int)], C.c_int)
_sig("so_apply_hamiltonian_bitwise", [_cp, _cp, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_int])
_sig("so_apply_H_xxz", [_cp, _cp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double])
_sig("so_set_threads", [C.c_int])
_sig("so_get_threads", [], C.c_int)


class threads:
    """with threads(n): the oracle's per-state loops use n threads inside the
    block (default 1, the reference's single-threaded loops)"""

    def __init__(self, n=None):
        self.n = n or os.cpu_count() or 1

    def __enter__(self):
        self.old = L.so_get_threads()
        L.so_set_threads(int(self.n))
        return self

    def __exit__(self, *exc):
        L.so_set_threads(self.old)
        return False


def zero_state(N, index=0):
    psi = np.zeros(1 << N, dtype=np.complex128)
    psi[index] = 1.0
    return psi


def _g1(name):
    f = getattr(L, f"so_apply_{name}_psi")

    def g(psi, k, N):
        f(_p(psi), k, N)
        return psi
    return g


def _g1t(name):
    f = getattr(L, f"so_apply_{name}_psi")

    def g(psi, k, theta, N):
        f(_p(psi), k, theta, N)
        return psi
    return g


apply_rx_psi, apply_ry_psi, apply_rz_psi = _g1t("rx"), _g1t("ry"), _g1t("rz")
apply_hadamard_psi, apply_pauli_x_psi, apply_pauli_y_psi = _g1("hadamard"), _g1("pauli_x"), _g1("pauli_y")
apply_pauli_z_psi, apply_s_psi, apply_sdagger_psi = _g1("pauli_z"), _g1("s"), _g1("sdagger")
apply_t_psi, apply_tdagger_psi = _g1("t"), _g1("tdagger")
apply_sigma_minus_psi, apply_sigma_plus_psi = _g1("sigma_minus"), _g1("sigma_plus")


def apply_ccz_psi(psi, a, b, c, N):
    L.so_apply_ccz_psi(_p(psi), a, b, c, N)
    return psi


def apply_toffoli_psi(psi, a, b, t, N):
    L.so_apply_toffoli_psi(_p(psi), a, b, t, N)
    return psi


def apply_cnot_psi(psi, c, t, N):
    L.so_apply_cnot_psi(_p(psi), c, t, N)
    return psi


def apply_cz_psi(psi, a, b, N):
    L.so_apply_cz_psi(_p(psi), a, b, N)
    return psi


def apply_cry_psi(psi, c, t, theta, N):
    L.so_apply_cry_psi(_p(psi), c, t, theta, N)
    return psi


def _rpp(name):
    f = getattr(L, f"so_apply_{name}_psi")

    def g(psi, a, b, theta, N):
        f(_p(psi), a, b, theta, N)
        return psi
    return g


apply_rxx_psi, apply_ryy_psi, apply_rzz_psi = _rpp("rxx"), _rpp("ryy"), _rpp("rzz")


def colmajor(U):
    U = np.asarray(U, dtype=np.complex128)
    return np.ascontiguousarray(U.T).view(np.float64).reshape(-1).copy()


def apply_one_qubit_gate(psi, U, q, N):
    u = colmajor(U)
    L.so_apply_one_qubit_gate(_p(psi), u.ctypes.data_as(_dp), q, N)
    return psi


def apply_two_qubit_gate(psi, U, q1, q2, N):
    u = colmajor(U)
    L.so_apply_two_qubit_gate(_p(psi), u.ctypes.data_as(_dp), q1, q2, N)
    return psi


def apply_2qubit_gate_ru(psi, U, q1, q2, N):
    u = colmajor(U)
    L.so_apply_2qubit_gate_ru(_p(psi), u.ctypes.data_as(_dp), q1, q2, N)
    return psi


def population_excited_psi(psi, k, N):
    return L.so_population_excited_psi(_p(psi), k, N)


def expect_local(psi, k, N, p):
    return getattr(L, f"so_expect_{p}")(_p(psi), k, N)


def expect_corr(psi, i, j, N, pp):
    return getattr(L, f"so_expect_{pp}")(_p(psi), i, j, N)


def pauli_string(psi, ops, qubits, N):
    qs = (C.c_int * len(qubits))(*qubits)
    return L.so_expect_pauli_string(_p(psi), len(qubits), "".join(ops).encode(), qs, N)


def norm2(psi, N):
    return L.so_norm2(_p(psi), N)


def make_gates(gates):
    """list of (indices 1-based, U ndarray) -> TrotterGate array"""
    arr = (TrotterGate * max(1, len(gates)))()
    for t, (idx, U) in enumerate(gates):
        arr[t].nq = len(idx)
        for k, q in enumerate(idx):
            arr[t].q[k] = q
        u = colmajor(U)
        for k, v in enumerate(u):
            arr[t].U[k] = v
    return arr


def precompute_trotter_gates(bonds, fields, dt):
    """bonds: rows (i, j, Jxx, Jyy, Jzz) 1-based; fields: rows (idx, hx, hy, hz). Returns (array, n)."""
    b = np.ascontiguousarray(bonds, dtype=np.float64).reshape(-1)
    f = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1)
    nb, nf = len(b) // 5, len(f) // 4
    out = (TrotterGate * max(1, nb + nf))()
    n = L.so_precompute_trotter_gates(b.ctypes.data_as(_dp), nb, f.ctypes.data_as(_dp), nf, dt, out)
    return out, n


def gates_to_list(arr, n):
    res = []
    for t in range(n):
        g = arr[t]
        dim = 2 if g.nq == 1 else 4
        u = np.array(g.U[:2 * dim * dim]).view(np.complex128).reshape(dim, dim).T.copy()
        res.append(([g.q[k] for k in range(g.nq)], u))
    return res


def trotter_step(psi, arr, n, N):
    L.so_trotter_step(_p(psi), arr, n, N)
    return psi


(N_DEPOLARIZING, N_AMPLITUDE_DAMPING, N_DEPHASING, N_BIT_FLIP, N_PHASE_FLIP, N_PHASE_DAMPING,
 N_THERMAL_RELAXATION) = range(32, 39)
M_MEASURE_Z, M_MEASURE_X, M_MEASURE_Y, R_RESET, T_TRACE_OUT, L_LINDBLAD_STEP = range(48, 54)
CIRCUIT_CODES = dict(GATE_CODES, depolarizing=N_DEPOLARIZING, amplitude_damping=N_AMPLITUDE_DAMPING,
                     dephasing=N_DEPHASING, bit_flip=N_BIT_FLIP, phase_flip=N_PHASE_FLIP,
                     phase_damping=N_PHASE_DAMPING, thermal_relaxation=N_THERMAL_RELAXATION,
                     measure_z=M_MEASURE_Z, measure_x=M_MEASURE_X, measure_y=M_MEASURE_Y, reset=R_RESET,
                     trace_out=T_TRACE_OUT, lindblad_step=L_LINDBLAD_STEP)
RESET_TARGETS = {"zero": 0, "one": 1, "plus": 2, "minus": 3}


def make_ops(ops):
    """ops: list of (name, [1-based qubits], param (1-based or 0), angle[, if_outcome]);
    noise ops carry p (gamma) in angle, a reset its target code in qubits[1]"""
    arr = (Op * max(1, len(ops)))()
    for t, op in enumerate(ops):
        name, qs, param, angle = op[:4]
        arr[t].type = CIRCUIT_CODES[name]
        for k, q in enumerate(qs):
            arr[t].q[k] = q
        arr[t].param = param
        arr[t].angle = angle
        arr[t].pad = op[4] if len(op) > 4 else 0
    return arr


def apply_circuit_mcwf(psi, ops_arr, n, theta, N, seed, traj):
    """one trajectory of a noisy circuit; returns the measurement outcomes"""
    th = np.ascontiguousarray(theta, dtype=np.float64)
    out = np.zeros(max(1, n), dtype=np.int32)
    m = L.so_apply_circuit_mcwf(_p(psi), ops_arr, n, th.ctypes.data_as(_dp), N, seed, traj,
                                out.ctypes.data_as(C.POINTER(C.c_int)))
    return out[:m]


def noisy_energy(ops_arr, n, theta, N, terms, seed, traj):
    """<psi_T|H|psi_T> of one trajectory of a noisy circuit from |0...0>"""
    coef, s = pauli_strings(terms, N)
    psi = zero_state(N, 0)
    apply_circuit_mcwf(psi, ops_arr, n, theta, N, seed, traj)
    return L.so_pauli_sum_expect(_p(psi), len(terms), coef.ctypes.data_as(_dp), s, N)


def _rows(rows, width):
    a = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(-1, width))
    return a, a.shape[0]


def apply_hamiltonian_bitwise(psi_in, x_bonds, y_bonds, fields, N):
    """out = H psi_in for bond rows (i, j, Jxx, Jyy, Jzz) and field rows (idx, hx, hy, hz), 1-based"""
    out = np.zeros_like(psi_in)
    xb, nx = _rows(x_bonds if len(x_bonds) else np.zeros((0, 5)), 5)
    yb, ny = _rows(y_bonds if len(y_bonds) else np.zeros((0, 5)), 5)
    fb, nf = _rows(fields if len(fields) else np.zeros((0, 4)), 4)
    L.so_apply_hamiltonian_bitwise(_p(out), _p(psi_in), xb.ctypes.data_as(_dp), nx, yb.ctypes.data_as(_dp), ny,
                                   fb.ctypes.data_as(_dp), nf, N)
    return out


def apply_H_xxz(psi, N, Jx, Jy, Jz, h):
    out = np.zeros_like(psi)
    L.so_apply_H_xxz(_p(psi), _p(out), N, Jx, Jy, Jz, h)
    return out


def circuit_draw(seed, op_index, traj):
    return L.so_circuit_draw(seed, op_index, traj)


def noise_u(kind, psi, p, k, N, u):
    """one noise unravelling with the draw u (kind: dephasing, depolarizing, bit_flip,
    phase_flip, amplitude_damping)"""
    getattr(L, f"so_noise_{kind}_u")(_p(psi), p, k, N, u)
    return psi


def measure_z_u(psi, k, N, u):
    return L.so_measure_z_u(_p(psi), k, N, u)


def reset_u(psi, k, target, N, u):
    L.so_reset_u(_p(psi), k, RESET_TARGETS.get(target, target), N, u)
    return psi


def apply_circuit(psi, ops_arr, n, theta, N):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    L.so_apply_circuit(_p(psi), ops_arr, n, th.ctypes.data_as(_dp), N)
    return psi


def pauli_strings(terms, N):
    """terms: list of (coef, {q(1-based): letter}) -> coef array, packed letters"""
    coef = np.array([c for c, _ in terms], dtype=np.float64)
    rows = []
    for _, ops in terms:
        r = ["I"] * N
        for q, p in ops.items():
            r[q - 1] = p
        rows.append("".join(r))
    return coef, "".join(rows).encode()


def energy(ops_arr, n, theta, N, terms):
    coef, s = pauli_strings(terms, N)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    return L.so_energy(ops_arr, n, th.ctypes.data_as(_dp), N, len(terms), coef.ctypes.data_as(_dp), s)


def grad(ops_arr, n, theta, N, terms, which=None, method="fd", eps=1e-4, shift=np.pi / 2):
    coef, s = pauli_strings(terms, N)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    P = th.size
    w = np.arange(P, dtype=np.int32) if which is None else np.ascontiguousarray(which, dtype=np.int32)
    out = np.empty(len(w))
    wp = w.ctypes.data_as(C.POINTER(C.c_int))
    if method == "fd":
        L.so_grad_finite_difference(ops_arr, n, th.ctypes.data_as(_dp), P, N, len(terms), coef.ctypes.data_as(_dp),
                                    s, eps, wp, len(w), out.ctypes.data_as(_dp))
    else:
        L.so_grad_parameter_shift(ops_arr, n, th.ctypes.data_as(_dp), P, N, len(terms), coef.ctypes.data_as(_dp),
                                  s, shift, wp, len(w), out.ctypes.data_as(_dp))
    return out


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    L.so_philox4x32_10(c, k, o)
    return list(o)


def make_jumps(jumps):
    """jumps: list of (type code, qubit 1-based, gamma)"""
    arr = (JumpOp * max(1, len(jumps)))()
    for t, (ty, q, g) in enumerate(jumps):
        arr[t].type, arr[t].qubit, arr[t].gamma = ty, q, g
    return arr


def mcwf_run(N, gates_arr, ng, jumps_arr, nj, dt, seed, t0, ntraj, steps, record_every, init_index=0,
             nthreads=1):
    nrec = steps // record_every + 1
    z = np.empty(nrec * ntraj * N)
    zz = np.empty(nrec * ntraj * max(1, N - 1))
    nj_out = np.zeros(ntraj, dtype=np.int32)
    L.so_mcwf_run(N, gates_arr, ng, jumps_arr, nj, dt, seed, t0, ntraj, steps, record_every, init_index,
                  z.ctypes.data_as(_dp), zz.ctypes.data_as(_dp), nj_out.ctypes.data_as(C.POINTER(C.c_int)), nthreads)
    return z.reshape(nrec, ntraj, N), zz.reshape(nrec, ntraj, -1)[:, :, :N - 1], nj_out


def dm_trotter_step(rho, arr, n, N):
    L.so_trotter_step_rho(_p(rho), arr, n, N)
    return rho


def dm_dissipator(rho, jump, dt, N):
    j = JumpOp(*jump)
    L.so_dissipator_dm(_p(rho), C.byref(j), dt, N)
    return rho


def dm_expect_z(rho, k, N):
    return L.so_expect_z_rho(_p(rho), k, N)


def dm_expect_zz(rho, i, j, N):
    return L.so_expect_zz_rho(_p(rho), i, j, N)


def wtime():
    return L.so_wtime()


def sample(psi, N, nshots, seed, stream=0):
    """Born sampling, shot loop of run_benchmark_smoq_Float64.jl:424-435 (Philox draws)"""
    out = np.empty(nshots, dtype=np.int64)
    L.so_sample(_p(psi), N, nshots, seed, stream, out.ctypes.data_as(C.POINTER(C.c_int64)))
    return out


def measure_all(psi, N, seed, stream=0):
    """projective_measurement_all! (cpuQuantumStateMeasurements.jl:484), in place"""
    return int(L.so_measure_all(_p(psi), N, seed, stream))


def measure_qubit(psi, k, N, seed, stream=0):
    """_measure_z_single! (cpuQuantumStateMeasurements.jl:224), in place, k 1-based"""
    return int(L.so_measure_qubit(_p(psi), k, N, seed, stream))


# ---- quantum reservoir computing (bitwise MCWF path; two rails of L qubits)
QRC_ENCODING = {"batch": 0, "batch_causal": 0, "broadcast": 1}
QRC_RESET = {"traceout_rail_1": 1, "protocol1": 1, "traceout_rail_2": 2, "protocol2": 2}


def qrc_n_ops(L, n_rails=2):
    return 3 * L * n_rails + 3 * (L - 1) * n_rails + 3 * L * (n_rails - 1)


def measure_all_observables(psi, L_, n_rails):
    out = np.empty(qrc_n_ops(L_, n_rails))
    L.so_measure_all_observables(_p(psi), L_, n_rails, out.ctypes.data_as(_dp))
    return out


def qrc_padded(inputs, L_):
    return np.concatenate([np.zeros(L_), np.asarray(inputs, dtype=np.float64)])


def qrc_run(L_, gates_arr, ng, inputs, n_traj, n_substeps=5, encoding="batch", reset="traceout_rail_1", seed=1234,
            traj_offset=0, psi0=None, per_trajectory=False, nthreads=1):
    """trajectory mean X[T, n_ops] (and, if asked, X_traj[n_traj, T, n_ops]) for the input series
    `inputs` (padded with L zeros in front, as run_mcwf_simulation does)"""
    T = len(inputs)
    u = np.ascontiguousarray(qrc_padded(inputs, L_))
    nops = qrc_n_ops(L_)
    p0 = zero_state(2 * L_) if psi0 is None else np.ascontiguousarray(psi0, dtype=np.complex128)
    X = np.empty(T * nops)
    Xt = np.empty(n_traj * T * nops) if per_trajectory else None
    L.so_qrc_run(L_, gates_arr, ng, n_substeps, QRC_ENCODING[encoding], QRC_RESET[reset], _p(p0),
                 u.ctypes.data_as(_dp), T, n_traj, seed, traj_offset, X.ctypes.data_as(_dp),
                 Xt.ctypes.data_as(_dp) if per_trajectory else None, nthreads)
    X = X.reshape(T, nops)
    return (X, Xt.reshape(n_traj, T, nops)) if per_trajectory else X


def qrc_dm_run(L_, gates_arr, ng, inputs, n_substeps=5, encoding="batch", reset="traceout_rail_1", psi0=None):
    T = len(inputs)
    u = np.ascontiguousarray(qrc_padded(inputs, L_))
    nops = qrc_n_ops(L_)
    p0 = zero_state(2 * L_) if psi0 is None else np.ascontiguousarray(psi0, dtype=np.complex128)
    X = np.empty(T * nops)
    L.so_qrc_dm_run(L_, gates_arr, ng, n_substeps, QRC_ENCODING[encoding], QRC_RESET[reset], _p(p0),
                    u.ctypes.data_as(_dp), T, X.ctypes.data_as(_dp))
    return X.reshape(T, nops)

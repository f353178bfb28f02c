"""pysmoq -- host-side mirror of SmoQ.jl's state-vector API over libsmoq_cuda.so.

Function names, argument order, 1-based qubit numbering and error behaviour
follow the Julia functions in the reference's utils/cpu modules (the `!` of
mutating Julia functions is dropped); every call runs on the GPU through the
C ABI in include/smoq_cuda.h.  `CuState` plays the role of the reference's
`ψ::Vector{ComplexF64}` and lives in HBM.

    ψ = CuState(ctx, N)                  # |0...0>, complex128
    apply_ry_psi(ψ, 1, 0.3, N)           # apply_ry_psi!(ψ, 1, 0.3, N)
    expect_local(ψ, 1, N, "z")           # expect_local(ψ, 1, N, :z)
"""
import ctypes as C
import weakref
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from ._lib import (C64, C128, SmoqError, SmoqJumpOp, SmoqOp, SmoqPauliTerm, SmoqTrotterGate, ck, dptr, lib,
                   EXPORTED, LIB_PATH)
from . import _lib

__all__ = [
    "Context", "CuState", "SmoqError", "C64", "C128",
    "apply_rx_psi", "apply_ry_psi", "apply_rz_psi", "apply_hadamard_psi", "apply_pauli_x_psi",
    "apply_pauli_y_psi", "apply_pauli_z_psi", "apply_s_psi", "apply_sdagger_psi", "apply_t_psi",
    "apply_tdagger_psi", "apply_ccz_psi", "apply_toffoli_psi", "apply_cnot_psi", "apply_cz_psi",
    "apply_cry_psi", "apply_rxx_psi", "apply_ryy_psi", "apply_rzz_psi", "apply_sigma_minus_psi",
    "apply_sigma_plus_psi", "apply_sigma_z", "population_excited_psi", "apply_one_qubit_gate_bitwise",
    "apply_two_qubit_gate_bitwise", "apply_gate", "apply_2qubit_gate", "expect_local", "expect_corr",
    "get_expectation_pauli_string", "get_norm", "normalize_state", "make_initial_psi",
    "CouplingTerm", "FieldTerm", "HamiltonianParams", "build_hamiltonian_parameters", "FastTrotterGate",
    "precompute_trotter_gates_bitwise", "TrotterPlan", "apply_fast_trotter_step", "evolve_trotter_psi",
    "CircuitOperation", "gate", "ParameterizedCircuit", "single_qubit_rotation_layer", "entangling_layer",
    "repeat_layer", "apply_circuit", "JumpOperator", "create_jump_operator", "mcwf_run", "PauliSum",
    "energy", "energy_and_gradient", "debug_plan", "run_mcwf_simulation", "qrc_n_ops",
]


# ----------------------------------------------------------------- context
class Context:
    """Owns a CUDA stream, scratch buffers and the last-error string (smoq_ctx).
    Closing it first closes the states and plans created on it (their C objects
    refer to the context)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        s = lib.smoq_ctx_create(device, C.byref(h))
        if s != 0:
            raise SmoqError(s, f"smoq_ctx_create(device={device}) failed")
        self.h = h
        self._children = weakref.WeakSet()

    def close(self):
        if self.h:
            for child in list(self._children):
                child.close()
            lib.smoq_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        ck(lib.smoq_ctx_synchronize(self.h), self.h, "synchronize")

    def set_option(self, opt: int, value: int):
        ck(lib.smoq_ctx_set_option(self.h, opt, value), self.h, "set_option")

    def counters(self):
        a, b = C.c_longlong(), C.c_longlong()
        ms, by = C.c_double(), C.c_double()
        ck(lib.smoq_ctx_counters(self.h, C.byref(a), C.byref(b), C.byref(ms), C.byref(by)), self.h)
        return {"launches": a.value, "tile_passes": b.value, "tile_ms": ms.value, "tile_bytes": by.value}

    def reset_counters(self):
        ck(lib.smoq_ctx_reset_counters(self.h), self.h)

    def tune_report(self) -> str:
        """the autotuner's per-pass variant timings (ms per launch) and choices"""
        buf = C.create_string_buffer(1 << 16)
        ck(lib.smoq_ctx_tune_report(self.h, buf, len(buf)), self.h)
        return buf.value.decode()

    @property
    def stream(self) -> int:
        return lib.smoq_ctx_stream(self.h)


# ------------------------------------------------------------------- state
class CuState:
    """`batch` state vectors of 2^N amplitudes in HBM (complex128 or complex64)."""

    def __init__(self, ctx: Context, N: int, dtype: int = C128, batch: int = 1, basis: Optional[int] = 0):
        self.ctx, self.N, self.dtype, self.batch = ctx, N, dtype, batch
        self.h = None
        h = C.c_void_p()
        ck(lib.smoq_state_create(ctx.h, N, dtype, batch, C.byref(h)), ctx.h, "smoq_state_create")
        self.h = h
        ctx._children.add(self)
        if basis is not None:
            self.set_basis(basis)

    @property
    def np_dtype(self):
        return np.complex64 if self.dtype == C64 else np.complex128

    def close(self):
        if self.h and self.ctx.h:  # a closed context has already closed this state
            lib.smoq_state_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_basis(self, index: int):
        ck(lib.smoq_state_set_basis(self.h, index), self.ctx.h, "set_basis")

    def upload(self, psi: np.ndarray):
        a = np.ascontiguousarray(psi, dtype=self.np_dtype).reshape(-1)
        if a.size != self.batch << self.N:
            raise ValueError("State dimension mismatch")
        ck(lib.smoq_state_upload(self.h, a.ctypes.data_as(C.c_void_p), a.nbytes), self.ctx.h, "upload")
        self.ctx.synchronize()

    def download(self) -> np.ndarray:
        out = np.empty(self.batch << self.N, dtype=self.np_dtype)
        ck(lib.smoq_state_download(self.h, out.ctypes.data_as(C.c_void_p), out.nbytes), self.ctx.h, "download")
        return out if self.batch == 1 else out.reshape(self.batch, -1)

    def download_range(self, first: int, count: int) -> np.ndarray:
        """amplitudes [first, first + count) of the batch (state b starts at b * 2^N)"""
        out = np.empty(count, dtype=self.np_dtype)
        ck(lib.smoq_state_download_range(self.h, first, count, out.ctypes.data_as(C.c_void_p)), self.ctx.h,
           "download_range")
        return out

    def copy_from(self, other: "CuState"):
        ck(lib.smoq_state_copy(self.h, other.h), self.ctx.h, "copy")


def _n(psi: CuState, N: int):
    if N != psi.N:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"N={N} does not match the state's N={psi.N}")


def _g1(fn):
    def f(psi: CuState, k: int, N: int):
        _n(psi, N)
        ck(fn(psi.h, k - 1), psi.ctx.h, fn.__name__)
        return psi
    return f


def _g1t(fn):
    def f(psi: CuState, k: int, theta: float, N: int):
        _n(psi, N)
        ck(fn(psi.h, k - 1, float(theta)), psi.ctx.h, fn.__name__)
        return psi
    return f


# utils/cpu/cpuQuantumChannelGates.jl
apply_rx_psi = _g1t(lib.smoq_apply_rx)
apply_ry_psi = _g1t(lib.smoq_apply_ry)
apply_rz_psi = _g1t(lib.smoq_apply_rz)
apply_hadamard_psi = _g1(lib.smoq_apply_h)
apply_pauli_x_psi = _g1(lib.smoq_apply_x)
apply_pauli_y_psi = _g1(lib.smoq_apply_y)
apply_pauli_z_psi = _g1(lib.smoq_apply_z)
apply_sigma_z = _g1(lib.smoq_apply_z)   # cpuQuantumChannelLindbladianEvolutionMonteCarloWaveFunction.jl:170
apply_s_psi = _g1(lib.smoq_apply_s)
apply_sdagger_psi = _g1(lib.smoq_apply_sdg)
apply_t_psi = _g1(lib.smoq_apply_t)
apply_tdagger_psi = _g1(lib.smoq_apply_tdg)
apply_sigma_minus_psi = _g1(lib.smoq_apply_sigma_minus)
apply_sigma_plus_psi = _g1(lib.smoq_apply_sigma_plus)


def apply_ccz_psi(psi, q1, q2, q3, N):
    _n(psi, N)
    ck(lib.smoq_apply_ccz(psi.h, q1 - 1, q2 - 1, q3 - 1), psi.ctx.h, "apply_ccz_psi")
    return psi


def apply_toffoli_psi(psi, c1, c2, t, N):
    _n(psi, N)
    ck(lib.smoq_apply_toffoli(psi.h, c1 - 1, c2 - 1, t - 1), psi.ctx.h, "apply_toffoli_psi")
    return psi


def apply_cnot_psi(psi, control, target, N):
    _n(psi, N)
    ck(lib.smoq_apply_cnot(psi.h, control - 1, target - 1), psi.ctx.h, "apply_cnot_psi")
    return psi


def apply_cz_psi(psi, qi, qj, N):
    _n(psi, N)
    ck(lib.smoq_apply_cz(psi.h, qi - 1, qj - 1), psi.ctx.h, "apply_cz_psi")
    return psi


def apply_cry_psi(psi, control, target, theta, N):
    _n(psi, N)
    ck(lib.smoq_apply_cry(psi.h, control - 1, target - 1, float(theta)), psi.ctx.h, "apply_cry_psi")
    return psi


def _rpp(fn):
    def f(psi, qi, qj, theta, N):
        _n(psi, N)
        ck(fn(psi.h, qi - 1, qj - 1, float(theta)), psi.ctx.h, fn.__name__)
        return psi
    return f


apply_rxx_psi = _rpp(lib.smoq_apply_rxx)
apply_ryy_psi = _rpp(lib.smoq_apply_ryy)
apply_rzz_psi = _rpp(lib.smoq_apply_rzz)


def _colmajor(U, n):
    U = np.asarray(U, dtype=np.complex128).reshape(n, n)
    return np.ascontiguousarray(U.T).view(np.float64).reshape(-1).copy()


def apply_one_qubit_gate_bitwise(psi, U, qubit, N):
    """apply_one_qubit_gate_bitwise_cpu! (cpuQuantumChannelUnitaryEvolutionTrotter.jl:77)"""
    _n(psi, N)
    u = _colmajor(U, 2)
    ck(lib.smoq_apply_u1(psi.h, qubit - 1, dptr(u)), psi.ctx.h, "apply_one_qubit_gate_bitwise")
    return psi


apply_gate = apply_one_qubit_gate_bitwise  # apply_gate! (cpuQuantumChannelRandomUnitaries.jl:230)


def apply_two_qubit_gate_bitwise(psi, U, q1, q2, N):
    """apply_two_qubit_gate_bitwise_cpu! (Trotter.jl:107): q1 > q2 swaps qubits, not U."""
    _n(psi, N)
    u = _colmajor(U, 4)
    ck(lib.smoq_apply_u2(psi.h, q1 - 1, q2 - 1, dptr(u), 0), psi.ctx.h, "apply_two_qubit_gate_bitwise")
    return psi


def apply_2qubit_gate(psi, U, q1, q2, N):
    """apply_2qubit_gate! (RandomUnitaries.jl:317): q1 > q2 conjugates U by SWAP."""
    _n(psi, N)
    u = _colmajor(U, 4)
    ck(lib.smoq_apply_u2(psi.h, q1 - 1, q2 - 1, dptr(u), 1), psi.ctx.h, "apply_2qubit_gate")
    return psi


# ------------------------------------------------------------ observables
def _scalar(psi, out):
    return float(out[0]) if psi.batch == 1 else out


def expect_local(psi: CuState, k: int, N: int, pauli: str):
    """expect_local (cpuQuantumStateObservables.jl:175)"""
    _n(psi, N)
    p = pauli.lower().lstrip(":")
    fn = {"z": lib.smoq_expect_z, "x": lib.smoq_expect_x, "y": lib.smoq_expect_y}.get(p)
    if fn is None:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown Pauli operator: {pauli}. Use :x, :y, or :z")
    out = np.empty(psi.batch)
    ck(fn(psi.h, k - 1, dptr(out)), psi.ctx.h, "expect_local")
    return _scalar(psi, out)


def expect_corr(psi: CuState, i: int, j: int, N: int, pauli_pair: str):
    """expect_corr (cpuQuantumStateObservables.jl:306)"""
    _n(psi, N)
    p = pauli_pair.lower().lstrip(":")
    fn = {"zz": lib.smoq_expect_zz, "xx": lib.smoq_expect_xx, "yy": lib.smoq_expect_yy}.get(p)
    if fn is None:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown Pauli pair: {pauli_pair}. Use :zz, :xx, or :yy")
    out = np.empty(psi.batch)
    ck(fn(psi.h, i - 1, j - 1, dptr(out)), psi.ctx.h, "expect_corr")
    return _scalar(psi, out)


def get_expectation_pauli_string(psi: CuState, operators: Sequence[str], qubits: Sequence[int], N: int):
    """get_expectation_pauli_string (cpuQuantumStateObservables.jl:840); full expectation for mixed strings."""
    _n(psi, N)
    if len(operators) != len(qubits):
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "operators and qubits must have same length")
    if len(operators) == 0:
        return 1.0
    ops = "".join(str(o).lstrip(":").upper() for o in operators).encode()
    qs = (C.c_int * len(qubits))(*[q - 1 for q in qubits])
    out = np.empty(psi.batch)
    ck(lib.smoq_expect_pauli_string(psi.h, len(qubits), ops, qs, dptr(out)), psi.ctx.h, "pauli_string")
    return _scalar(psi, out)


def expect_zstrings(psi: CuState, zmasks: Sequence[int]) -> np.ndarray:
    m = np.asarray(zmasks, dtype=np.uint64)
    out = np.empty(psi.batch * len(m))
    ck(lib.smoq_expect_zstrings(psi.h, m.ctypes.data_as(C.POINTER(C.c_uint64)), len(m), dptr(out)),
       psi.ctx.h, "expect_zstrings")
    return out.reshape(psi.batch, len(m))


def sample_bitstrings(psi: CuState, nshots: int, seed: int, stream: int = 0) -> np.ndarray:
    """Born-rule shots (basis indices; bit k-1 = qubit k), [batch, nshots] or [nshots]."""
    out = np.empty((psi.batch, nshots), dtype=np.int64)
    ck(lib.smoq_sample(psi.h, nshots, seed, stream, out.ctypes.data_as(C.POINTER(C.c_longlong))), psi.ctx.h,
       "sample")
    return out[0] if psi.batch == 1 else out


def projective_measurement_all(psi: CuState, N: int, seed: int, stream: int = 0):
    """projective_measurement_all!(psi, N): (bitstring per qubit, collapsed psi)."""
    _n(psi, N)
    out = np.empty(psi.batch, dtype=np.int64)
    ck(lib.smoq_measure_all(psi.h, seed, stream, out.ctypes.data_as(C.POINTER(C.c_longlong))), psi.ctx.h,
       "projective_measurement_all")
    bits = [[(int(o) >> (k - 1)) & 1 for k in range(1, N + 1)] for o in out]
    return (bits[0] if psi.batch == 1 else bits), psi


def measure_z(psi: CuState, k: int, N: int, seed: int, stream: int = 0):
    """_measure_z_single!(psi, k, N): outcome 0/1 (per state), psi collapsed."""
    _n(psi, N)
    out = np.empty(psi.batch, dtype=np.int32)
    ck(lib.smoq_measure_qubit(psi.h, k - 1, seed, stream, out.ctypes.data_as(C.POINTER(C.c_int))), psi.ctx.h,
       "measure_z")
    return int(out[0]) if psi.batch == 1 else out


def measure_all_observables_state_vector(psi: CuState, L: int, n_rails: int) -> np.ndarray:
    """measure_all_observables_state_vector_cpu(psi, L, n_rails): local X, Y, Z, then
    XX, YY, ZZ on rail bonds, then on rungs (reference order); [n_ops] or [batch, n_ops]."""
    N = L * n_rails
    n_ops = 3 * N + 3 * (L - 1) * n_rails + 3 * L * (n_rails - 1)
    out = np.empty((psi.batch, n_ops))
    ck(lib.smoq_measure_all_observables(psi.h, L, n_rails, dptr(out)), psi.ctx.h, "measure_all_observables")
    return out[0] if psi.batch == 1 else out


def population_excited_psi(psi: CuState, k: int, N: int):
    _n(psi, N)
    out = np.empty(psi.batch)
    ck(lib.smoq_population_excited(psi.h, k - 1, dptr(out)), psi.ctx.h, "population_excited_psi")
    return _scalar(psi, out)


def get_norm(psi: CuState):
    out = np.empty(psi.batch)
    ck(lib.smoq_norm2(psi.h, dptr(out)), psi.ctx.h, "get_norm")
    return _scalar(psi, np.sqrt(out))


def normalize_state(psi: CuState):
    ck(lib.smoq_normalize(psi.h), psi.ctx.h, "normalize_state")
    return psi


def make_initial_psi(ctx: Context, N: int, init_bits: Sequence[int] = (), dtype: int = C128, batch: int = 1):
    """make_initial_psi (cpuQuantumStatePreparation.jl:1211)"""
    idx = 0
    if len(init_bits):
        if len(init_bits) != N:
            raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "init_bits must have length N")
        for k, b in enumerate(init_bits):
            if b == 1:
                idx |= 1 << k
    return CuState(ctx, N, dtype, batch, basis=idx)


# ------------------------------------------------------ Hamiltonian + Trotter
@dataclass
class CouplingTerm:      # cpuHamiltonianBuilder.jl:42 (1-based sites)
    i: int
    j: int
    Jxx: float
    Jyy: float
    Jzz: float


@dataclass
class FieldTerm:         # cpuHamiltonianBuilder.jl:51
    idx: int
    hx: float
    hy: float
    hz: float


@dataclass
class HamiltonianParams:  # cpuHamiltonianBuilder.jl:69
    N: int
    x_bonds: List[CouplingTerm]
    y_bonds: List[CouplingTerm]
    fields: List[FieldTerm]


def build_hamiltonian_parameters(Nx: int, Ny: int, J_x_direction, J_y_direction, h_field) -> HamiltonianParams:
    """build_hamiltonian_parameters (cpuHamiltonianBuilder.jl:166): uniform couplings on an Nx x Ny grid."""
    N = Nx * Ny
    xb = [CouplingTerm((r - 1) * Nx + i, (r - 1) * Nx + i + 1, *J_x_direction)
          for r in range(1, Ny + 1) for i in range(1, Nx)]
    yb = []
    if Ny >= 2:
        for i in range(1, Nx + 1):
            yb.append(CouplingTerm(i, Nx + i, *J_y_direction))
        for r in range(2, Ny):
            for i in range(1, Nx + 1):
                yb.append(CouplingTerm((r - 1) * Nx + i, r * Nx + i, *J_y_direction))
    fields = [FieldTerm(i, *h_field) for i in range(1, N + 1)]
    return HamiltonianParams(N, xb, yb, fields)


@dataclass
class FastTrotterGate:   # cpuQuantumChannelUnitaryEvolutionTrotter.jl:62 (1-based indices)
    indices: List[int]
    U: np.ndarray


def _to_c_gates(gates: Sequence[FastTrotterGate]):
    arr = (SmoqTrotterGate * max(1, len(gates)))()
    for t, g in enumerate(gates):
        n = len(g.indices)
        arr[t].nq = n
        for k, q in enumerate(g.indices):
            arr[t].q[k] = q - 1
        u = _colmajor(g.U, 2 if n == 1 else 4)
        for k, v in enumerate(u):
            arr[t].U[k] = v
    return arr


def precompute_trotter_gates_bitwise(params: HamiltonianParams, dt: float) -> List[FastTrotterGate]:
    """precompute_trotter_gates_bitwise_cpu (Trotter.jl:322) via the library's closed form."""
    bonds = params.x_bonds + params.y_bonds
    b = np.array([[c.i - 1, c.j - 1, c.Jxx, c.Jyy, c.Jzz] for c in bonds], dtype=np.float64).reshape(-1)
    f = np.array([[x.idx - 1, x.hx, x.hy, x.hz] for x in params.fields], dtype=np.float64).reshape(-1)
    out = (SmoqTrotterGate * (len(bonds) + len(params.fields) + 1))()
    n = C.c_int()
    ck(lib.smoq_precompute_trotter_gates(dptr(b) if b.size else None, len(bonds), dptr(f) if f.size else None,
                                         len(params.fields), float(dt), out, C.byref(n)), None,
       "precompute_trotter_gates")
    res = []
    for t in range(n.value):
        g = out[t]
        dim = 2 if g.nq == 1 else 4
        u = np.array(g.U[:2 * dim * dim]).view(np.complex128).reshape(dim, dim).T.copy()
        res.append(FastTrotterGate([g.q[k] + 1 for k in range(g.nq)], u))
    return res


class TrotterPlan:
    """A compiled Trotter step (order 1 = the gate list; order 2 = Strang: list + reversed list)."""

    def __init__(self, ctx: Context, N: int, gates: Sequence[FastTrotterGate], order: int = 1, dtype: int = C128):
        self.ctx, self.N, self.order, self.dtype = ctx, N, order, dtype
        self.h = None
        arr = _to_c_gates(gates)
        h = C.c_void_p()
        ck(lib.smoq_trotter_plan_create(ctx.h, N, dtype, arr, len(gates), order, C.byref(h)), ctx.h,
           "trotter_plan_create")
        self.h = h
        ctx._children.add(self)

    def close(self):
        if self.h and self.ctx.h:  # a closed context has already closed this plan
            lib.smoq_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, psi: CuState, n_steps: int = 1):
        ck(lib.smoq_trotter_step(self.h, psi.h, n_steps), self.ctx.h, "trotter_step")

    def run(self, psi: CuState, steps: int, record_every: int) -> np.ndarray:
        nrec = steps // record_every + 1
        out = np.empty(nrec * psi.batch * self.N)
        ck(lib.smoq_trotter_run(self.h, psi.h, steps, record_every, dptr(out)), self.ctx.h, "trotter_run")
        return out.reshape(nrec, psi.batch, self.N)


def apply_fast_trotter_step(psi: CuState, gates, N: int):
    """apply_fast_trotter_step_cpu! (Trotter.jl:150); `gates` is a TrotterPlan or a gate list."""
    _n(psi, N)
    plan = gates if isinstance(gates, TrotterPlan) else TrotterPlan(psi.ctx, N, gates, 1, psi.dtype)
    plan.step(psi, 1)
    return psi


def evolve_trotter_psi(psi: CuState, gates, N: int, n_substeps: int = 1):
    """evolve_trotter_psi_cpu! (Trotter.jl:250)"""
    _n(psi, N)
    plan = gates if isinstance(gates, TrotterPlan) else TrotterPlan(psi.ctx, N, gates, 1, psi.dtype)
    plan.step(psi, n_substeps)
    return psi


# --------------------------------------------------------------- circuits
_GATE_CODES = {"rx": _lib.G_RX, "ry": _lib.G_RY, "rz": _lib.G_RZ, "h": _lib.G_H, "x": _lib.G_X, "y": _lib.G_Y,
               "z": _lib.G_Z, "s": _lib.G_S, "sdg": _lib.G_SDG, "t": _lib.G_T, "tdg": _lib.G_TDG,
               "cz": _lib.G_CZ, "cnot": _lib.G_CNOT, "cx": _lib.G_CNOT, "rxx": _lib.G_RXX, "ryy": _lib.G_RYY,
               "rzz": _lib.G_RZZ, "cry": _lib.G_CRY, "ccz": _lib.G_CCZ, "toffoli": _lib.G_TOFFOLI}


_NOISE_CODES = {"depolarizing": _lib.N_DEPOLARIZING, "amplitude_damping": _lib.N_AMPLITUDE_DAMPING,
                "dephasing": _lib.N_DEPHASING, "bit_flip": _lib.N_BIT_FLIP, "phase_flip": _lib.N_PHASE_FLIP,
                "phase_damping": _lib.N_PHASE_DAMPING, "thermal_relaxation": _lib.N_THERMAL_RELAXATION}
_MEASURE_CODES = {"measure_z": _lib.M_MEASURE_Z, "measure_x": _lib.M_MEASURE_X, "measure_y": _lib.M_MEASURE_Y,
                  "measure": _lib.M_MEASURE_Z}
_OTHER_CODES = {"reset": _lib.R_RESET, "trace_out": _lib.T_TRACE_OUT, "lindblad_step": _lib.L_LINDBLAD_STEP}
_RESET_TARGETS = {"zero": 0, "one": 1, "plus": 2, "minus": 3}


@dataclass
class CircuitOperation:  # cpuVariationalQuantumCircuitBuilder.jl:120
    type: str
    qubits: List[int]
    param_idx: int = 0
    fixed_angle: float = 0.0
    p: float = 0.0                 # noise probability or rate
    target_state: str = "none"     # reset target: zero, one, plus, minus
    basis: str = "z"               # measurement basis
    if_outcome: int = 0            # 0 always; k > 0 only if the trajectory's outcome k (1-based) is 1

    @property
    def is_gate(self) -> bool:
        return self.type in _GATE_CODES


def gate(type: str, qubits, param_idx: int = 0, angle: float = 0.0, if_outcome: int = 0) -> CircuitOperation:
    """gate (cpuVariationalQuantumCircuitBuilder.jl:172)"""
    t = type.lower().lstrip(":")
    if t not in _GATE_CODES:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown gate type: {type}")
    q = [qubits] if isinstance(qubits, int) else list(qubits)
    return CircuitOperation(t, q, param_idx, angle, if_outcome=if_outcome)


def noise(type: str, qubits, p: float = 0.0, if_outcome: int = 0) -> CircuitOperation:
    """noise (cpuVariationalQuantumCircuitBuilder.jl:192): a channel unravelled per trajectory"""
    t = type.lower().lstrip(":")
    if t not in _NOISE_CODES:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown noise type: {type}")
    q = [qubits] if isinstance(qubits, int) else list(qubits)
    return CircuitOperation(t, q, p=float(p), if_outcome=if_outcome)


def measure(qubits, basis: str = "z") -> CircuitOperation:
    """measure (cpuVariationalQuantumCircuitBuilder.jl:210): projective, one outcome per qubit"""
    b = basis.lower().lstrip(":")
    if b not in ("x", "y", "z"):
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown basis: {basis}. Use :z, :x, :y")
    q = [qubits] if isinstance(qubits, int) else list(qubits)
    return CircuitOperation("measure_" + b, q, basis=b)


def reset(qubits, target_state: str = "zero", if_outcome: int = 0) -> CircuitOperation:
    """reset (cpuVariationalQuantumCircuitBuilder.jl:229)"""
    t = target_state.lower().lstrip(":")
    if t not in _RESET_TARGETS:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown reset target: {target_state}")
    q = [qubits] if isinstance(qubits, int) else list(qubits)
    return CircuitOperation("reset", q, target_state=t, if_outcome=if_outcome)


def trace_out(qubits) -> CircuitOperation:
    """trace_out (cpuVariationalQuantumCircuitBuilder.jl:261): no effect on a pure state"""
    return CircuitOperation("trace_out", [qubits] if isinstance(qubits, int) else list(qubits))


def lindblad_step(qubits) -> CircuitOperation:
    """lindblad_step (cpuVariationalQuantumCircuitBuilder.jl:245): the reference's pure-state executor skips it"""
    return CircuitOperation("lindblad_step", [qubits] if isinstance(qubits, int) else list(qubits))


@dataclass
class CircuitResult:  # cpuVariationalQuantumCircuitBuilder.jl:150
    state: "CuState"
    outcomes: np.ndarray   # [outcomes] (batch 1) or [batch, outcomes]: 0/1 in execution order


@dataclass
class ParameterizedCircuit:  # cpuVariationalQuantumCircuitBuilder.jl:295
    N: int
    operations: List[CircuitOperation]
    n_params: int = field(default=-1)

    def __post_init__(self):
        if self.n_params < 0:
            self.n_params = max([op.param_idx for op in self.operations] + [0])


def single_qubit_rotation_layer(N: int, param_offset: int, gates=("ry",)):
    """single_qubit_rotation_layer (Builder.jl:337): gate-major parameter order."""
    ops, idx = [], param_offset
    for g in gates:
        for q in range(1, N + 1):
            ops.append(gate(g, [q], param_idx=idx))
            idx += 1
    return ops, idx


def entangling_layer(N: int, topology: str = "chain", gate_type: str = "cz"):
    """entangling_layer (Builder.jl:356)"""
    if topology == "chain":
        return [gate(gate_type, [q, q + 1]) for q in range(1, N)]
    if topology == "ring":
        ops = [gate(gate_type, [q, q + 1]) for q in range(1, N)]
        if N > 2:
            ops.append(gate(gate_type, [N, 1]))
        return ops
    if topology == "all":
        return [gate(gate_type, [i, j]) for i in range(1, N + 1) for j in range(i + 1, N + 1)]
    raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown topology: {topology}")


def repeat_layer(layer_fn, L: int, N: int, param_offset: int = 1):
    """repeat_layer (Builder.jl:605)"""
    all_ops, idx = [], param_offset
    for _ in range(L):
        ops, idx = layer_fn(N, idx)
        all_ops.extend(ops)
    return all_ops, idx


def _c_ops(ops: Sequence[CircuitOperation]):
    """one smoq_op per gate, and one per qubit of a noise / measure / reset op (the
    reference loops over those qubits in order)"""
    out = []
    for op in ops:
        if op.type in _GATE_CODES:
            out.append((_GATE_CODES[op.type], [q - 1 for q in op.qubits], op.param_idx - 1 if op.param_idx > 0 else -1,
                        op.fixed_angle, op.if_outcome))
            continue
        code = _NOISE_CODES.get(op.type, _MEASURE_CODES.get(op.type, _OTHER_CODES.get(op.type)))
        if code is None:
            raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown operation type: {op.type}")
        for q in op.qubits:
            qs = [q - 1, _RESET_TARGETS[op.target_state]] if op.type == "reset" else [q - 1]
            out.append((code, qs, -1, op.p, op.if_outcome))
    arr = (SmoqOp * max(1, len(out)))()
    for t, (code, qs, param, angle, cond) in enumerate(out):
        arr[t].type = code
        for k, q in enumerate(qs):
            arr[t].q[k] = q
        arr[t].param = param
        arr[t].angle = angle
        arr[t].if_outcome = cond
    return arr, len(out)


def circuit_to_c_ops(ops: Sequence[CircuitOperation]):
    return _c_ops(ops)[0]


def count_measurements(ops: Sequence[CircuitOperation]) -> int:
    return sum(len(op.qubits) for op in ops if op.type in _MEASURE_CODES)


def apply_circuit(psi: CuState, circuit: ParameterizedCircuit, theta, fused: bool = True, seed: int = 1234,
                  traj_offset: int = 0):
    """apply_circuit! (cpuVariationalQuantumCircuitExecutor.jl:95).  Gate-only circuits run as
    fused tile passes (fused=True) or one kernel per gate and return psi.  Circuits with noise,
    measurements, resets or classical conditions run every state of psi as one trajectory
    (draws from Philox4x32-10, key seed, counter (op index, 0x80000000, traj_offset + b)) and
    return a CircuitResult with the measurement outcomes."""
    if psi.N != circuit.N:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "State dimension mismatch")
    th = np.ascontiguousarray(theta, dtype=np.float64)
    if th.size < circuit.n_params:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "Not enough parameters")
    arr, n = _c_ops(circuit.operations)
    if all(op.is_gate and op.if_outcome == 0 for op in circuit.operations):
        fn = lib.smoq_apply_sequence if fused else lib.smoq_apply_sequence_unfused
        ck(fn(psi.h, arr, n, dptr(th)), psi.ctx.h, "apply_circuit")
        return psi
    nm = count_measurements(circuit.operations)
    out = np.zeros(max(1, psi.batch * nm), dtype=np.int32)
    ck(lib.smoq_apply_circuit_mcwf(psi.h, arr, n, dptr(th), seed, traj_offset,
                                   out.ctypes.data_as(C.POINTER(C.c_int32))), psi.ctx.h, "apply_circuit")
    oc = out[:psi.batch * nm].reshape(psi.batch, nm)
    return CircuitResult(psi, oc[0] if psi.batch == 1 else oc)


def _channel(kind, psi: CuState, p: float, qubits, N: int, seed: int, traj_offset: int):
    _n(psi, N)
    qs = [qubits] if isinstance(qubits, int) else list(qubits)
    circ = ParameterizedCircuit(N, [noise(kind, qs, p=p)])
    apply_circuit(psi, circ, np.zeros(1), seed=seed, traj_offset=traj_offset)
    return psi


def apply_channel_dephasing(psi, p, qubits, N, seed=1234, traj_offset=0):
    """apply_channel_dephasing! (cpuQuantumChannelKrausOperators.jl:426), pure-state unravelling"""
    return _channel("dephasing", psi, p, qubits, N, seed, traj_offset)


def apply_channel_depolarizing(psi, p, qubits, N, seed=1234, traj_offset=0):
    """apply_channel_depolarizing! (cpuQuantumChannelKrausOperators.jl:458)"""
    return _channel("depolarizing", psi, p, qubits, N, seed, traj_offset)


def apply_channel_amplitude_damping(psi, gamma, qubits, N, seed=1234, traj_offset=0):
    """apply_channel_amplitude_damping! (cpuQuantumChannelKrausOperators.jl:492)"""
    return _channel("amplitude_damping", psi, gamma, qubits, N, seed, traj_offset)


def apply_channel_bit_flip(psi, p, qubits, N, seed=1234, traj_offset=0):
    """apply_channel_bit_flip! (cpuQuantumChannelKrausOperators.jl:524)"""
    return _channel("bit_flip", psi, p, qubits, N, seed, traj_offset)


def apply_channel_phase_flip(psi, p, qubits, N, seed=1234, traj_offset=0):
    """apply_channel_phase_flip! (cpuQuantumChannelKrausOperators.jl:556)"""
    return _channel("phase_flip", psi, p, qubits, N, seed, traj_offset)


def projective_measurement(psi: CuState, qubits, basis: str, N: int, seed: int = 1234, traj_offset: int = 0):
    """projective_measurement! (cpuQuantumStateMeasurements.jl:319): (outcomes, psi)"""
    _n(psi, N)
    r = apply_circuit(psi, ParameterizedCircuit(N, [measure(qubits, basis)]), np.zeros(1), seed=seed,
                      traj_offset=traj_offset)
    return r.outcomes, psi


def reset_state(psi: CuState, qubits, targets, N: int, seed: int = 1234, traj_offset: int = 0):
    """reset_state! (cpuQuantumStateMeasurements.jl:555): targets a symbol or one per qubit"""
    _n(psi, N)
    qs = [qubits] if isinstance(qubits, int) else list(qubits)
    ts = [targets] * len(qs) if isinstance(targets, str) else list(targets)
    if len(ts) != len(qs):
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "Must specify target for each qubit")
    apply_circuit(psi, ParameterizedCircuit(N, [reset([q], t) for q, t in zip(qs, ts)]), np.zeros(1), seed=seed,
                  traj_offset=traj_offset)
    return psi


# ------------------------------------------------------------------ MCWF
_JUMP_CODES = {"sigma_minus": 0, "sigma_plus": 1, "sigma_z": 2, "sigma_x": 3}


@dataclass
class JumpOperator:      # cpuQuantumChannelLindbladianEvolution.jl:65 (bitwise types)
    type: str
    qubit: int
    gamma: float


def create_jump_operator(type: str, qubit: int = 1, gamma: float = 0.1) -> JumpOperator:
    t = type.lower().lstrip(":")
    if t not in _JUMP_CODES:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, f"Unknown jump operator type: {type}")
    return JumpOperator(t, qubit, gamma)


def mcwf_run(plan: TrotterPlan, psi: CuState, jump_ops: Sequence[JumpOperator], dt: float, seed: int,
             steps: int, record_every: int, traj_offset: int = 0, per_trajectory: bool = False):
    """Batched MCWF (evolve_mcwf_batched_trotter!, MonteCarloWaveFunction.jl:412): every state of psi is a
    trajectory.  Returns dict with z_mean [nrec, N], zz_mean [nrec, N-1], jumps [B] and, if asked,
    z_traj [nrec, B, N], zz_traj [nrec, B, N-1]."""
    N, B = psi.N, psi.batch
    nrec = steps // record_every + 1
    ops = (SmoqJumpOp * max(1, len(jump_ops)))()
    for t, o in enumerate(jump_ops):
        ops[t].type = _JUMP_CODES[o.type]
        ops[t].qubit = o.qubit - 1
        ops[t].gamma = o.gamma
    zm = np.empty(nrec * N)
    zzm = np.empty(nrec * max(1, N - 1))
    zt = np.empty(nrec * B * N) if per_trajectory else None
    zzt = np.empty(nrec * B * max(1, N - 1)) if per_trajectory else None
    jumps = np.zeros(B, dtype=np.int32)
    ck(lib.smoq_mcwf_run(plan.h, psi.h, ops, len(jump_ops), float(dt), seed, traj_offset, steps, record_every,
                         dptr(zm), dptr(zzm), dptr(zt), dptr(zzt), jumps.ctypes.data_as(C.POINTER(C.c_int))),
       psi.ctx.h, "mcwf_run")
    out = {"z_mean": zm.reshape(nrec, N), "zz_mean": zzm.reshape(nrec, -1)[:, :N - 1], "jumps": jumps}
    if per_trajectory:
        out["z_traj"] = zt.reshape(nrec, B, N)
        out["zz_traj"] = zzt.reshape(nrec, B, -1)[:, :, :N - 1]
    return out


# ------------------------------------------------------------------- VQE
class PauliSum:
    """H = sum_t coef_t P_t; terms given as (coef, {qubit(1-based): 'X'|'Y'|'Z'})."""

    def __init__(self, terms):
        self.terms = []
        for coef, ops in terms:
            x = z = 0
            for q, p in ops.items():
                b = 1 << (q - 1)
                p = p.upper()
                if p in "XY":
                    x |= b
                if p in "YZ":
                    z |= b
            self.terms.append((float(coef), x, z))

    @staticmethod
    def tfim(N: int, J: float = 1.0, h: float = 1.0) -> "PauliSum":
        """H = -J sum Z_i Z_{i+1} - h sum X_i (the VQE energy of demo_vqe_dm_vs_mcwf.jl:189-202)."""
        terms = [(-J, {i: "Z", i + 1: "Z"}) for i in range(1, N)] + [(-h, {i: "X"}) for i in range(1, N + 1)]
        return PauliSum(terms)

    def c_terms(self):
        arr = (SmoqPauliTerm * max(1, len(self.terms)))()
        for t, (c, x, z) in enumerate(self.terms):
            arr[t].coef, arr[t].xmask, arr[t].zmask = c, x, z
        return arr


def apply_pauli_sum(psi_out: CuState, psi_in: CuState, H: PauliSum):
    """psi_out = H psi_in for a Pauli sum; returns Re <psi_in|H|psi_in> (per state)."""
    e = np.empty(psi_in.batch)
    ck(lib.smoq_apply_pauli_sum(psi_in.h, psi_out.h, H.c_terms(), len(H.terms), dptr(e)), psi_in.ctx.h,
       "apply_pauli_sum")
    return e[0] if psi_in.batch == 1 else e


def apply_hamiltonian_bitwise(psi_out: CuState, psi_in: CuState, params):
    """apply_hamiltonian_bitwise!(psi_out, psi_in, params::HamiltonianParams)
    (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55): psi_out = H psi_in.  `params` is a
    HamiltonianParams (1-based sites, as the reference's), or a PauliSum (then the
    return value is Re <psi_in|H|psi_in> per state)."""
    if isinstance(params, PauliSum):
        return apply_pauli_sum(psi_out, psi_in, params)
    xb = np.array([[b.i - 1, b.j - 1, b.Jxx, b.Jyy, b.Jzz] for b in params.x_bonds], dtype=np.float64).reshape(-1)
    yb = np.array([[b.i - 1, b.j - 1, b.Jxx, b.Jyy, b.Jzz] for b in params.y_bonds], dtype=np.float64).reshape(-1)
    fb = np.array([[f.idx - 1, f.hx, f.hy, f.hz] for f in params.fields], dtype=np.float64).reshape(-1)
    ck(lib.smoq_apply_hamiltonian_bitwise(psi_out.h, psi_in.h, dptr(xb), len(params.x_bonds), dptr(yb),
                                          len(params.y_bonds), dptr(fb), len(params.fields)),
       psi_in.ctx.h, "apply_hamiltonian_bitwise")
    return psi_out


def apply_H_xxz(psi: CuState, out: CuState, N: int, Jx: float, Jy: float, Jz: float, h: float):
    """apply_H_xxz! (cpuQuantumStateLanczos.jl:157)"""
    _n(psi, N)
    ck(lib.smoq_apply_h_xxz(psi.h, out.h, Jx, Jy, Jz, h), psi.ctx.h, "apply_H_xxz")
    return out


def apply_H_ising(psi: CuState, out: CuState, N: int, J: float, h: float):
    """apply_H_ising! (cpuQuantumStateLanczos.jl:220)"""
    return apply_H_xxz(psi, out, N, 0.0, 0.0, J, h)


def energy(ctx: Context, circuit: ParameterizedCircuit, H: PauliSum, theta, dtype: int = C128):
    th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1, circuit.n_params)
    B = th.shape[0]
    ops = circuit_to_c_ops(circuit.operations)
    e = np.empty(B)
    ck(lib.smoq_energy(ctx.h, circuit.N, dtype, ops, len(circuit.operations), circuit.n_params, H.c_terms(),
                       len(H.terms), B, dptr(th), dptr(e)), ctx.h, "energy")
    return e


def energy_and_gradient(ctx: Context, circuit: ParameterizedCircuit, H: PauliSum, theta, dtype: int = C128):
    """Energy and adjoint gradient for B parameter sets (theta shape [B, P] or [P])."""
    th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1, circuit.n_params)
    B = th.shape[0]
    ops = circuit_to_c_ops(circuit.operations)
    e = np.empty(B)
    g = np.empty((B, circuit.n_params))
    ck(lib.smoq_energy_grad(ctx.h, circuit.N, dtype, ops, len(circuit.operations), circuit.n_params, H.c_terms(),
                            len(H.terms), B, dptr(th), dptr(e), dptr(g)), ctx.h, "energy_grad")
    return e, g


def energy_and_gradient_noisy(ctx: Context, circuit: ParameterizedCircuit, H: PauliSum, theta, seed: int = 1234,
                              traj_offset: int = 0, n_traj: int = 1, checkpoint_every: int = 1, dtype: int = C128,
                              gradient: bool = True):
    """Energy and path-wise adjoint gradient of a noisy circuit along the trajectories
    traj_offset .. traj_offset + n_traj - 1 (the draws of apply_circuit with the same seed),
    from |0...0>.  Returns (energies[n_traj], grads[n_traj, P])."""
    th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
    if th.size < circuit.n_params:
        raise SmoqError(_lib.SMOQ_ERR_BADINPUT, "Not enough parameters")
    arr, n = _c_ops(circuit.operations)
    e = np.empty(n_traj)
    g = np.empty((n_traj, max(1, circuit.n_params))) if gradient else None
    ck(lib.smoq_energy_grad_mcwf(ctx.h, circuit.N, dtype, arr, n, circuit.n_params, H.c_terms(), len(H.terms),
                                 dptr(th), seed, traj_offset, n_traj, checkpoint_every, dptr(e), dptr(g)),
       ctx.h, "energy_grad_mcwf")
    return e, (g[:, :circuit.n_params] if gradient else None)


def energy_and_gradient_jobs(ctx: Context, jobs, dtype: int = C128, gradient: bool = True):
    """Many independent circuits at once: jobs = [(circuit, PauliSum, theta), ...],
    each its own size and Hamiltonian.  Returns (energies[njobs], [grad arrays])."""
    keep, arr = [], (_lib.SmoqVqeJob * max(1, len(jobs)))()
    e = np.empty(len(jobs))
    grads = []
    for j, (circ, H, theta) in enumerate(jobs):
        ops = circuit_to_c_ops(circ.operations)
        terms = H.c_terms()
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        if th.size != circ.n_params:
            raise ValueError(f"job {j}: theta has {th.size} values, the circuit {circ.n_params} parameters")
        g = np.zeros(max(1, circ.n_params))
        keep += [ops, terms, th, g]
        grads.append(g[:circ.n_params])
        arr[j] = _lib.SmoqVqeJob(circ.N, C.cast(ops, C.POINTER(_lib.SmoqOp)), len(circ.operations), circ.n_params,
                                 C.cast(terms, C.POINTER(_lib.SmoqPauliTerm)), len(H.terms), dptr(th),
                                 C.cast(C.c_void_p(e.ctypes.data + 8 * j), C.POINTER(C.c_double)),
                                 dptr(g) if gradient else None)
    ck(lib.smoq_energy_grad_jobs(ctx.h, dtype, arr, len(jobs)), ctx.h, "energy_grad_jobs")
    return e, grads


# ------------------------------------------------------ planner introspection
def debug_plan(N: int, ops: Sequence[CircuitOperation], theta=None, dtype: int = C128, tile_bits: int = 12,
               low_bits: int = 4, engine: int = 0):
    """Host-only view of how smoq_apply_sequence splits `ops` into tile passes
    (as scheduled for fused-pass `engine`).
    Returns a list of passes: {"T","L","H","hb","ops":[{"kind","nq","lb","gb","perm","c"}]}."""
    arr = circuit_to_c_ops(ops)
    th = np.ascontiguousarray(theta if theta is not None else np.zeros(1), dtype=np.float64)
    npass, nops = C.c_int(), C.c_int()
    ck(lib.smoq_debug_plan_sequence(N, dtype, tile_bits, low_bits, engine, arr, len(ops), dptr(th), None, 0, None, 0,
                                    C.byref(npass), C.byref(nops)), None, "debug_plan")
    P = (_lib.SmoqPassInfo * max(1, npass.value))()
    F = (_lib.SmoqFusedOpInfo * max(1, nops.value))()
    ck(lib.smoq_debug_plan_sequence(N, dtype, tile_bits, low_bits, engine, arr, len(ops), dptr(th), P, npass.value, F,
                                    nops.value, C.byref(npass), C.byref(nops)), None, "debug_plan")
    out, k = [], 0
    for i in range(npass.value):
        p = P[i]
        d = {"T": p.T, "L": p.L, "H": p.H, "hb": list(p.hb[:p.H]), "ops": []}
        for _ in range(p.nops):
            f = F[k]
            k += 1
            d["ops"].append({"kind": f.kind, "nq": f.nq, "lb": list(f.lb), "gb": list(f.gb), "perm": list(f.perm),
                             "slot": list(f.slot), "mode": f.mode,
                             "c": np.array(f.c[:]).view(np.complex128).copy()})
        out.append(d)
    return out


def debug_compile_plan(N: int, ops: Sequence[CircuitOperation], theta=None, dtype: int = C64, tile_bits: int = 13,
                       low_bits: int = 5, verbose: bool = False, buffers: int = 1, groups: int = 2,
                       rtc: bool = False, source: bool = False, all_sources: bool = False):
    """Host-only: plan `ops` for the plan compiler (engine 3) and compile every pass
    kernel with NVRTC (no GPU, nothing loaded).  Returns (status, n_compiled, message);
    with verbose the message is the compiler's register/spill report.  rtc: the
    run-time-coefficient form (a variational forward); source: the message is the
    generated source of the first pass (nothing compiled); all_sources: the sources of
    every pass, one after another (with rtc each followed by a "//@coefs" line: the pass's
    run-time coefficient block as hex floats, re im per entry)."""
    arr = circuit_to_c_ops(ops)
    th = np.ascontiguousarray(theta if theta is not None else np.zeros(1), dtype=np.float64)
    n = C.c_int()
    source = source or all_sources
    size = 1 << (26 if all_sources else 22 if source else 16)
    msg = C.create_string_buffer(size)
    flags = (1 if verbose else 0) | (2 if buffers == 2 else 0) | (4 if rtc else 0) | (8 if groups == 1 else 0) \
        | (16 if source else 0) | (32 if all_sources else 0)
    st = lib.smoq_debug_compile_plan(N, dtype, tile_bits, low_bits, arr, len(ops), dptr(th), flags, C.byref(n),
                                     msg, size)
    return st, n.value, msg.value.decode(errors="replace")


def debug_compile_adjoint(circuit: "ParameterizedCircuit", theta, tile_bits: int = 13, low_bits: int = 5,
                          verbose: bool = False, source: bool = False):
    """Host-only: build the backward program of a variational circuit as
    energy_and_gradient does (complex64), stage-schedule its passes for the compiled
    adjoint kernel and compile those kernels with NVRTC (no GPU, nothing loaded).
    Returns (status, n_passes, n_compiled, message); with verbose the message is the
    compiler's register/spill report, with source the generated CUDA source of the first
    compiled pass (nothing compiled)."""
    arr = circuit_to_c_ops(circuit.operations)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    npass, ncomp = C.c_int(), C.c_int()
    size = 1 << 22
    msg = C.create_string_buffer(size)
    st = lib.smoq_debug_compile_adjoint(circuit.N, arr, len(circuit.operations), circuit.n_params,
                                        dptr(th), tile_bits, low_bits, (1 if verbose else 0) | (2 if source else 0),
                                        C.byref(npass), C.byref(ncomp), msg, size)
    return st, npass.value, ncomp.value, msg.value.decode(errors="replace")


def jit_available() -> bool:
    """True when the plan compiler (engine 3, NVRTC) can run in this process."""
    return bool(lib.smoq_jit_available())


# ----------------------------------------------------------- density matrices
class DensityMatrixPlan(TrotterPlan):
    """One step of the reference's density-matrix evolution on a 2N-qubit state that
    holds rho column-major: rho -> U rho U^dag for the gate list (evolve_trotter_rho_cpu!),
    then one Euler dissipator step per jump (_apply_dissipator_dm!)."""

    def __init__(self, ctx: Context, N: int, gates: Sequence[FastTrotterGate], jump_ops, dt: float,
                 dtype: int = C128):
        self.ctx, self.N, self.order, self.dtype = ctx, N, 1, dtype
        self.h = None
        arr = _to_c_gates(gates)
        ops = (SmoqJumpOp * max(1, len(jump_ops)))()
        for t, o in enumerate(jump_ops):
            ops[t].type = _JUMP_CODES[o.type]
            ops[t].qubit = o.qubit - 1
            ops[t].gamma = o.gamma
        h = C.c_void_p()
        ck(lib.smoq_dm_plan_create(ctx.h, N, dtype, arr, len(gates), ops, len(jump_ops), float(dt), C.byref(h)),
           ctx.h, "dm_plan_create")
        self.h = h
        ctx._children.add(self)


def density_matrix_state(ctx: Context, N: int, basis: int = 0, dtype: int = C128, batch: int = 1) -> CuState:
    """|basis><basis| as a 2N-qubit state (rho column-major)."""
    return CuState(ctx, 2 * N, dtype, batch, basis=basis + (basis << N))


def dm_expect_zstrings(rho: CuState, N: int, zmasks: Sequence[int]) -> np.ndarray:
    """sum_i Re rho_ii (-1)^popc(i & mask) per mask (mask 0: trace), [batch, nobs]."""
    m = np.ascontiguousarray(zmasks, dtype=np.uint64)
    out = np.empty((rho.batch, len(m)))
    ck(lib.smoq_dm_expect_zstrings(rho.h, N, m.ctypes.data_as(C.POINTER(C.c_uint64)), len(m), dptr(out)),
       rho.ctx.h, "dm_expect_zstrings")
    return out


# ----------------------------------------------------------------- quantum reservoir computing
_QRC_ENCODING = {"batch": 0, "batch_causal": 0, "broadcast": 1}
_QRC_RESET = {"traceout_rail_1": 1, "protocol1": 1, "traceout_rail_2": 2, "protocol2": 2}


def qrc_n_ops(L: int, n_rails: int = 2) -> int:
    """features per input: 3N + 3 (L-1) n_rails + 3 L (n_rails-1)"""
    return 3 * L * n_rails + 3 * (L - 1) * n_rails + 3 * L * (n_rails - 1)


def run_mcwf_simulation(psi0, H_params, gates, padded_u, L: int, n_rails: int, T: int, n_traj: int,
                        integrator_type: str = "trotter_cpu", T_evol: float = 0.0, encoding: str = "batch",
                        reset_type: str = "traceout_rail_1", n_substeps: int = 5, *, ctx: "Context" = None,
                        dtype: int = C128, seed: int = 1234, traj_offset: int = 0, per_trajectory: bool = False):
    """The bitwise run_mcwf_simulation (cpuQRCSimulationMonteCarloWaveFunction.jl:531) on the GPU:
    n_traj trajectories of the QRC loop (_run_traj_loop_bitwise! :451), each
    trajectory's state in one CTA's shared memory for the whole series.  Returns
    X[T, n_ops], the trajectory mean of the ladder features after every input
    (and X_traj[n_traj, T, n_ops] with per_trajectory=True).

    psi0: 2^N amplitudes or None (|0...0>); H_params: kept for the reference's
    signature (the evolution is `gates`); gates: a TrotterPlan on N = 2L qubits or
    a FastTrotterGate list (one Trotter step); padded_u: [zeros(L); inputs]
    (T + L values).  Only the :trotter_cpu integrator runs here.  The reset's
    rand() is the Philox draw (shot = input index, stream = trajectory id)."""
    if integrator_type != "trotter_cpu":
        raise ValueError(f"Unsupported integrator: {integrator_type}. Supported here: :trotter_cpu")
    if n_rails != 2:
        raise ValueError("the QRC reset reshapes the state as 2^L x 2^L: n_rails must be 2")
    if ctx is None:
        ctx = gates.ctx if isinstance(gates, TrotterPlan) else None
    if ctx is None:
        raise ValueError("a Context is needed (pass ctx=, or a TrotterPlan)")
    N = L * n_rails
    plan = gates if isinstance(gates, TrotterPlan) else TrotterPlan(ctx, N, gates, 1, dtype)
    u = np.ascontiguousarray(padded_u, dtype=np.float64)
    if u.size < T + L:
        raise ValueError("padded_u must hold T + L values")
    p = _lib.SmoqQrcParams(L, n_substeps, _QRC_ENCODING[encoding], _QRC_RESET[reset_type], seed, traj_offset)
    nops = qrc_n_ops(L, n_rails)
    X = np.empty(T * nops)
    Xt = np.empty(n_traj * T * nops) if per_trajectory else None
    p0 = None
    if psi0 is not None:
        p0 = np.ascontiguousarray(np.asarray(psi0, dtype=np.complex128).view(np.float64))
    ck(lib.smoq_qrc_run(plan.h, C.byref(p), dptr(p0) if p0 is not None else None, dptr(u), T, n_traj, dptr(X),
                        dptr(Xt) if per_trajectory else None), ctx.h, "qrc_run")
    X = X.reshape(T, nops)
    return (X, Xt.reshape(n_traj, T, nops)) if per_trajectory else X

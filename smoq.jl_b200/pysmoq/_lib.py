"""ctypes binding of libsmoq_cuda.so (include/smoq_cuda.h).

The library is the only compute path: if it is missing or cannot be loaded,
importing this module raises -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("SMOQ_CUDA_LIB", os.path.join(_PKG, "lib", "libsmoq_cuda.so"))

SMOQ_OK, SMOQ_ERR_BADINPUT, SMOQ_ERR_OOM, SMOQ_ERR_CUDA, SMOQ_ERR_TIMEOUT, SMOQ_ERR_UNSUPPORTED, SMOQ_ERR_NOGPU = range(7)
STATUS_NAMES = {0: "OK", 1: "BADINPUT", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "UNSUPPORTED", 6: "NOGPU"}
C64, C128 = 0, 1

(G_RX, G_RY, G_RZ, G_H, G_X, G_Y, G_Z, G_S, G_SDG, G_T, G_TDG, G_CZ, G_CNOT, G_RXX, G_RYY, G_RZZ,
 G_CRY, G_CCZ, G_TOFFOLI, G_U1, G_U2) = range(21)

(OPT_TILE_BITS_C64, OPT_TILE_BITS_C128, OPT_LOW_BITS_C64, OPT_LOW_BITS_C128, OPT_USE_GRAPHS, OPT_KERNEL_TIMING,
 OPT_ENGINE, OPT_JIT_BUFFERS) = range(1, 9)
OPT_JIT_GROUPS, OPT_VQE_RESIDENT, OPT_AUTOTUNE, OPT_FUSION_DEPTH = 10, 12, 13, 14


# operations of smoq_apply_circuit_mcwf beyond the gates (one qubit each)
(N_DEPOLARIZING, N_AMPLITUDE_DAMPING, N_DEPHASING, N_BIT_FLIP, N_PHASE_FLIP, N_PHASE_DAMPING,
 N_THERMAL_RELAXATION) = range(32, 39)
M_MEASURE_Z, M_MEASURE_X, M_MEASURE_Y, R_RESET, T_TRACE_OUT, L_LINDBLAD_STEP = range(48, 54)


class SmoqOp(C.Structure):
    _fields_ = [("type", C.c_int32), ("q", C.c_int32 * 3), ("param", C.c_int32), ("if_outcome", C.c_int32),
                ("angle", C.c_double), ("U", C.c_double * 32)]


class SmoqTrotterGate(C.Structure):
    _fields_ = [("nq", C.c_int32), ("q", C.c_int32 * 2), ("pad", C.c_int32), ("U", C.c_double * 32)]


class SmoqJumpOp(C.Structure):
    _fields_ = [("type", C.c_int32), ("qubit", C.c_int32), ("gamma", C.c_double)]


class SmoqPauliTerm(C.Structure):
    _fields_ = [("coef", C.c_double), ("xmask", C.c_uint64), ("zmask", C.c_uint64)]


class SmoqVqeJob(C.Structure):
    _fields_ = [("N", C.c_int), ("ops", C.POINTER(SmoqOp)), ("n", C.c_int), ("n_params", C.c_int),
                ("H", C.POINTER(SmoqPauliTerm)), ("nterms", C.c_int), ("theta", C.POINTER(C.c_double)),
                ("energy", C.POINTER(C.c_double)), ("grad", C.POINTER(C.c_double))]


class SmoqQrcParams(C.Structure):
    _fields_ = [("L", C.c_int32), ("n_substeps", C.c_int32), ("encoding", C.c_int32), ("reset", C.c_int32),
                ("seed", C.c_uint64), ("traj_offset", C.c_uint64)]


class SmoqPassInfo(C.Structure):
    _fields_ = [("T", C.c_int32), ("L", C.c_int32), ("H", C.c_int32), ("nops", C.c_int32), ("hb", C.c_int32 * 24)]


class SmoqFusedOpInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nq", C.c_int32), ("lb", C.c_int32 * 4), ("gb", C.c_int32 * 4),
                ("perm", C.c_int32 * 8), ("slot", C.c_int32 * 4), ("mode", C.c_int32), ("c", C.c_double * 32)]


class SmoqError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"smoq status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libsmoq_cuda.so not built at {LIB_PATH} (run smoq.jl_b200/build.py)")
    return C.CDLL(LIB_PATH)


lib = _load()

_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)

_SIGS = {
    "smoq_ctx_create": [C.c_int, C.POINTER(_vp)],
    "smoq_ctx_destroy": [_vp],
    "smoq_ctx_synchronize": [_vp],
    "smoq_ctx_set_option": [_vp, C.c_int, C.c_longlong],
    "smoq_ctx_counters": [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), _dp, _dp],
    "smoq_ctx_reset_counters": [_vp],
    "smoq_ctx_tune_report": [_vp, C.c_char_p, C.c_int],
    "smoq_debug_wait_timeout": [_vp, C.c_uint64],
    "smoq_state_create": [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)],
    "smoq_state_wrap": [_vp, _vp, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)],
    "smoq_state_destroy": [_vp],
    "smoq_state_upload": [_vp, _vp, C.c_size_t],
    "smoq_state_download": [_vp, _vp, C.c_size_t],
    "smoq_state_download_range": [_vp, C.c_uint64, C.c_uint64, _vp],
    "smoq_state_set_basis": [_vp, C.c_uint64],
    "smoq_state_copy": [_vp, _vp],
    "smoq_apply_rx": [_vp, C.c_int, C.c_double],
    "smoq_apply_ry": [_vp, C.c_int, C.c_double],
    "smoq_apply_rz": [_vp, C.c_int, C.c_double],
    "smoq_apply_h": [_vp, C.c_int],
    "smoq_apply_x": [_vp, C.c_int],
    "smoq_apply_y": [_vp, C.c_int],
    "smoq_apply_z": [_vp, C.c_int],
    "smoq_apply_s": [_vp, C.c_int],
    "smoq_apply_sdg": [_vp, C.c_int],
    "smoq_apply_t": [_vp, C.c_int],
    "smoq_apply_tdg": [_vp, C.c_int],
    "smoq_apply_ccz": [_vp, C.c_int, C.c_int, C.c_int],
    "smoq_apply_toffoli": [_vp, C.c_int, C.c_int, C.c_int],
    "smoq_apply_cnot": [_vp, C.c_int, C.c_int],
    "smoq_apply_cz": [_vp, C.c_int, C.c_int],
    "smoq_apply_cry": [_vp, C.c_int, C.c_int, C.c_double],
    "smoq_apply_rxx": [_vp, C.c_int, C.c_int, C.c_double],
    "smoq_apply_ryy": [_vp, C.c_int, C.c_int, C.c_double],
    "smoq_apply_rzz": [_vp, C.c_int, C.c_int, C.c_double],
    "smoq_apply_sigma_minus": [_vp, C.c_int],
    "smoq_apply_sigma_plus": [_vp, C.c_int],
    "smoq_apply_u1": [_vp, C.c_int, _dp],
    "smoq_apply_u2": [_vp, C.c_int, C.c_int, _dp, C.c_int],
    "smoq_apply_sequence": [_vp, C.POINTER(SmoqOp), C.c_int, _dp],
    "smoq_apply_sequence_unfused": [_vp, C.POINTER(SmoqOp), C.c_int, _dp],
    "smoq_apply_circuit_mcwf": [_vp, C.POINTER(SmoqOp), C.c_int, _dp, C.c_uint64, C.c_uint64,
                                C.POINTER(C.c_int32)],
    "smoq_expect_x": [_vp, C.c_int, _dp],
    "smoq_expect_y": [_vp, C.c_int, _dp],
    "smoq_expect_z": [_vp, C.c_int, _dp],
    "smoq_expect_xx": [_vp, C.c_int, C.c_int, _dp],
    "smoq_expect_yy": [_vp, C.c_int, C.c_int, _dp],
    "smoq_expect_zz": [_vp, C.c_int, C.c_int, _dp],
    "smoq_expect_pauli_string": [_vp, C.c_int, C.c_char_p, _ip, _dp],
    "smoq_expect_zstrings": [_vp, _u64p, C.c_int, _dp],
    "smoq_expect_zstrings_noalloc": [_vp, C.c_int, C.c_int, C.c_int, _u64p, C.c_int, _vp, _vp, C.c_char_p,
                                     C.c_size_t],
    "smoq_population_excited": [_vp, C.c_int, _dp],
    "smoq_norm2": [_vp, _dp],
    "smoq_normalize": [_vp],
    "smoq_precompute_trotter_gates": [_dp, C.c_int, _dp, C.c_int, C.c_double, C.POINTER(SmoqTrotterGate), _ip],
    "smoq_trotter_plan_create": [_vp, C.c_int, C.c_int, C.POINTER(SmoqTrotterGate), C.c_int, C.c_int,
                                 C.POINTER(_vp)],
    "smoq_plan_destroy": [_vp],
    "smoq_trotter_step": [_vp, _vp, C.c_int],
    "smoq_trotter_run": [_vp, _vp, C.c_int, C.c_int, _dp],
    "smoq_mcwf_run": [_vp, _vp, C.POINTER(SmoqJumpOp), C.c_int, C.c_double, C.c_uint64, C.c_uint64, C.c_int,
                      C.c_int, _dp, _dp, _dp, _dp, _ip],
    "smoq_energy_grad": [_vp, C.c_int, C.c_int, C.POINTER(SmoqOp), C.c_int, C.c_int, C.POINTER(SmoqPauliTerm),
                         C.c_int, C.c_int, _dp, _dp, _dp],
    "smoq_jit_available": [],
    "smoq_apply_pauli_sum": [_vp, _vp, C.POINTER(SmoqPauliTerm), C.c_int, _dp],
    "smoq_apply_hamiltonian_bitwise": [_vp, _vp, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int],
    "smoq_apply_h_xxz": [_vp, _vp, C.c_double, C.c_double, C.c_double, C.c_double],
    "smoq_dm_plan_create": [_vp, C.c_int, C.c_int, C.POINTER(SmoqTrotterGate), C.c_int, C.POINTER(SmoqJumpOp),
                            C.c_int, C.c_double, C.POINTER(C.c_void_p)],
    "smoq_dm_expect_zstrings": [_vp, C.c_int, C.POINTER(C.c_uint64), C.c_int, _dp],
    "smoq_measure_all_observables": [_vp, C.c_int, C.c_int, _dp],
    "smoq_sample": [_vp, C.c_longlong, C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_longlong)],
    "smoq_measure_all": [_vp, C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_longlong)],
    "smoq_measure_qubit": [_vp, C.c_int, C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_int)],
    "smoq_energy_grad_jobs": [_vp, C.c_int, C.POINTER(SmoqVqeJob), C.c_int],
    "smoq_qrc_run": [_vp, C.POINTER(SmoqQrcParams), _dp, _dp, C.c_int, C.c_int64, _dp, _dp],
    "smoq_debug_compile_plan": [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(SmoqOp), C.c_int, _dp, C.c_int, _ip,
                                C.c_char_p, C.c_int],
    "smoq_debug_compile_adjoint": [C.c_int, C.POINTER(SmoqOp), C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int,
                                   _ip, _ip, C.c_char_p, C.c_int],
    "smoq_debug_pick_geometry": [C.POINTER(C.c_float), C.c_int],
    "smoq_debug_plan_sequence": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(SmoqOp), C.c_int, _dp,
                                 C.POINTER(SmoqPassInfo), C.c_int, C.POINTER(SmoqFusedOpInfo), C.c_int, _ip, _ip],
    "smoq_energy": [_vp, C.c_int, C.c_int, C.POINTER(SmoqOp), C.c_int, C.c_int, C.POINTER(SmoqPauliTerm),
                    C.c_int, C.c_int, _dp, _dp],
    "smoq_energy_grad_mcwf": [_vp, C.c_int, C.c_int, C.POINTER(SmoqOp), C.c_int, C.c_int, C.POINTER(SmoqPauliTerm),
                              C.c_int, _dp, C.c_uint64, C.c_uint64, C.c_int, C.c_int, _dp, _dp],
}

for _name, _args in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = C.c_int
lib.smoq_last_error.argtypes = [_vp]
lib.smoq_last_error.restype = C.c_char_p
lib.smoq_version.argtypes = []
lib.smoq_version.restype = C.c_char_p
lib.smoq_ctx_stream.argtypes = [_vp]
lib.smoq_ctx_stream.restype = _vp
lib.smoq_state_device_ptr.argtypes = [_vp]
lib.smoq_state_device_ptr.restype = _vp

EXPORTED = sorted(list(_SIGS) + ["smoq_last_error", "smoq_version", "smoq_ctx_stream", "smoq_state_device_ptr"])


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def ck(status, ctx=None, what=""):
    if status != SMOQ_OK:
        msg = lib.smoq_last_error(ctx).decode() if ctx else ""
        raise SmoqError(status, f"{what}: {msg}")

"""CPU-side checks of the C-ABI library: it builds for sm_100a, loads, and
exports every entry point include/smoq_cuda.h declares; without a GPU the
context constructor reports the absence instead of crashing."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "smoq_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(smoq_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_exports_header(built):
    import pysmoq
    lib = ctypes.CDLL(pysmoq.LIB_PATH)
    syms = header_symbols()
    assert len(syms) > 50
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares every header symbol too
    assert sorted(set(syms) - set(pysmoq.EXPORTED)) == []


def test_version_string(built):
    import pysmoq
    assert b"sm_100a" in pysmoq.lib.smoq_version()


def test_no_gpu_is_an_error_not_a_crash(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import pysmoq
    with pytest.raises(pysmoq.SmoqError) as e:
        pysmoq.Context(0)
    assert e.value.status == 6  # SMOQ_ERR_NOGPU


def test_null_handles_are_rejected(built):
    import pysmoq
    lib = pysmoq.lib
    assert lib.smoq_ctx_destroy(None) == 1
    assert lib.smoq_state_destroy(None) == 1
    assert lib.smoq_apply_rx(None, 0, 0.1) == 1
    assert lib.smoq_expect_z(None, 0, None) == 1
    assert lib.smoq_trotter_step(None, None, 1) == 1


def test_closed_form_trotter_gates_match_oracle(built):
    """smoq_precompute_trotter_gates is host code: compare with the oracle's restatement."""
    import numpy as np
    import oracle as O
    import pysmoq
    rng = np.random.default_rng(0)
    N = 6
    params = pysmoq.HamiltonianParams(
        N, [pysmoq.CouplingTerm(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)], [],
        [pysmoq.FieldTerm(i, 0.3, 0.0, float(rng.uniform(-1, 1))) for i in range(1, N + 1)])
    g = pysmoq.precompute_trotter_gates_bitwise(params, 0.025)
    arr, n = O.precompute_trotter_gates([(c.i, c.j, c.Jxx, c.Jyy, c.Jzz) for c in params.x_bonds],
                                        [(f.idx, f.hx, f.hy, f.hz) for f in params.fields], 0.025)
    ref = O.gates_to_list(arr, n)
    assert len(g) == len(ref)
    for a, (idx, U) in zip(g, ref):
        assert a.indices == idx
        assert np.max(np.abs(a.U - U)) < 1e-15

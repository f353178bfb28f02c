"""smoq_expect_zstrings_noalloc: the Z-string batch for callers that cannot
allocate device memory when they call in (fixed-footprint hosts, callers that
hold most of HBM already, code that must not wait on the allocator).  It keeps
its partial sums in a fixed array inside the library instead of a scratch
buffer grown with cudaMalloc.

Checked through the C ABI against the existing entry point
smoq_expect_zstrings, within the tolerance the other reduction tests use
(1e-12 for complex128), on two calls in a row with different shapes so a
stale value left in the shared array by the first call would show up in the
second.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import dense_ref as D
import pysmoq as S
from pysmoq import _lib as L

pytestmark = pytest.mark.gpu


def device_out(ctx, n_doubles):
    """caller-owned device output buffer: a complex128 state holds 2 doubles per amplitude"""
    n_amp = max(2, (n_doubles + 1) // 2)
    N = int(np.ceil(np.log2(n_amp)))
    st = S.CuState(ctx, N, S.C128, 1, basis=None)
    return st, L.lib.smoq_state_device_ptr(st.h)


def read_out(st, n):
    return st.download().view(np.float64)[:n].copy()


def call_noalloc(ctx, st, masks, out_ptr):
    m = np.asarray(masks, dtype=np.uint64)
    err = C.create_string_buffer(256)
    s = L.lib.smoq_expect_zstrings_noalloc(L.lib.smoq_state_device_ptr(st.h), st.N, st.dtype, st.batch,
                                           m.ctypes.data_as(C.POINTER(C.c_uint64)), len(m), out_ptr,
                                           ctx.stream, err, 256)
    ctx.synchronize()
    return s, err.value.decode()


def test_noalloc_matches_existing_entry_point_twice(ctx):
    rng = np.random.default_rng(101)
    # call 1: complex128, 4 states of N=15, 32 observables (the per-call maximum)
    N1, B1 = 15, 4
    a = S.CuState(ctx, N1, S.C128, B1, basis=None)
    a.upload(np.stack([D.random_state(N1, rng) for _ in range(B1)]))
    masks1 = [0] + [1 << q for q in range(N1)] + [(3 << q) for q in range(N1 - 1)] + [0b101101, 0b1110000000001]
    masks1 = masks1[:32]
    want1 = S.expect_zstrings(a, masks1)
    out1, p1 = device_out(ctx, B1 * len(masks1))
    s, msg = call_noalloc(ctx, a, masks1, p1)
    assert s == 0, msg
    got1 = read_out(out1, B1 * len(masks1)).reshape(B1, -1)
    assert np.max(np.abs(got1 - want1)) < 1e-12

    # call 2, right after: a different shape (one state of N=20, 7 observables) and
    # dtype; the shared scratch must not leak anything from call 1
    N2 = 20
    b = S.CuState(ctx, N2, S.C64, 1, basis=None)
    b.upload(D.random_state(N2, rng))
    masks2 = [0, 1, 1 << 19, (1 << 19) | 1, 0b111, 0xFFFFF, 1 << 7]
    want2 = S.expect_zstrings(b, masks2)
    out2, p2 = device_out(ctx, len(masks2))
    s, msg = call_noalloc(ctx, b, masks2, p2)
    assert s == 0, msg
    got2 = read_out(out2, len(masks2)).reshape(1, -1)
    assert np.max(np.abs(got2 - want2)) < 1e-12


def test_noalloc_fills_its_fixed_scratch_exactly(ctx):
    """2048 states x 32 observables = 65536 partial sums: one block per state,
    the last partial at the array's final slot"""
    rng = np.random.default_rng(202)
    N, B = 6, 2048
    a = S.CuState(ctx, N, S.C64, B, basis=None)
    a.upload(np.stack([D.random_state(N, rng) for _ in range(B)]).astype(np.complex64))
    masks = [int(m) for m in rng.integers(0, 1 << N, size=32)]
    want = S.expect_zstrings(a, masks)
    out, p = device_out(ctx, B * len(masks))
    s, msg = call_noalloc(ctx, a, masks, p)
    assert s == 0, msg
    got = read_out(out, B * len(masks)).reshape(B, -1)
    assert np.max(np.abs(got - want)) < 1e-12


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(ctx):
    a = S.CuState(ctx, 6, S.C128, 1)
    out, p = device_out(ctx, 64)
    s, msg = call_noalloc(ctx, a, list(range(33)), p)        # more than 32 observables
    assert s == L.SMOQ_ERR_BADINPUT and "32" in msg
    s, msg = call_noalloc(ctx, a, [1 << 6], p)                 # a mask beyond N
    assert s == L.SMOQ_ERR_BADINPUT and "beyond N" in msg
    big = S.CuState(ctx, 2, S.C128, 4000, basis=0)             # 4000 states x 32 obs > 65536 partials
    s, msg = call_noalloc(ctx, big, list(range(4)) * 8, p)
    assert s == L.SMOQ_ERR_BADINPUT and "65536" in msg

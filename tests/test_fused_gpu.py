"""GPU parity of the fused tile-pass engine: gate sequences planned into
shared-memory tile passes must equal the oracle's gate-by-gate result.
Covers the reference's benchmark circuits (regenerated fixtures), the
plain-method workload (N=20 complex128 hardware-efficient circuit, 590 gates,
<Z_i> and <Z_i Z_{i+1}>), Strang Trotter sweeps and tile-width variations."""
import json
import math
import os

import numpy as np
import pytest

import dense_ref as D
import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def circuit_ops(lines):
    """benchmark circuit file lines -> (pysmoq ops, oracle ops), 1-based qubits"""
    name = {"H": "h", "X": "x", "Y": "y", "Z": "z", "S": "s", "T": "t", "RX": "rx", "RY": "ry", "RZ": "rz",
            "CNOT": "cnot", "CZ": "cz"}
    g_ops, o_ops = [], []
    for ln in lines:
        p = ln.split()
        t = name[p[0]]
        if t in ("cnot", "cz"):
            qs = [int(p[1]) + 1, int(p[2]) + 1]
            ang = 0.0
        else:
            qs = [int(p[1]) + 1]
            ang = float(p[2]) if len(p) > 2 else 0.0
        g_ops.append(S.gate(t, qs, angle=ang))
        o_ops.append((t, qs, 0, ang))
    return g_ops, o_ops


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("N", [2, 6, 10, 14, 16, 20])
def test_benchmark_circuits_fused_vs_oracle(ctx, N):
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N)]
    g_ops, o_ops = circuit_ops(lines)
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    for dtype, tol in ((S.C128, 1e-12), (S.C64, 5e-5)):
        st = S.CuState(ctx, N, dtype)
        S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
        got = st.download().astype(complex)
        assert rel(got, want) < tol, (N, dtype, rel(got, want))


@pytest.mark.parametrize("tile_bits", [3, 5, 8, 12])
def test_tile_width_variations(ctx, tile_bits):
    N = 14
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N)]
    g_ops, o_ops = circuit_ops(lines[:400])
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    ctx.set_option(S._lib.OPT_TILE_BITS_C128, tile_bits)
    ctx.set_option(S._lib.OPT_LOW_BITS_C128, min(4, tile_bits))
    try:
        st = S.CuState(ctx, N, S.C128)
        S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
        assert rel(st.download(), want) < 1e-12
    finally:
        ctx.set_option(S._lib.OPT_TILE_BITS_C128, 12)
        ctx.set_option(S._lib.OPT_LOW_BITS_C128, 4)


@pytest.mark.parametrize("engine", [0, 2])
@pytest.mark.parametrize("N,tile_bits", [(9, 8), (12, 9), (16, 10), (18, 13), (20, 11)])
def test_engines_and_tile_widths(ctx, engine, N, tile_bits):
    """shared-memory sweeps (engine 0) at every tile width and stage sweeps (engine 2,
    on the passes of tile width 12-13) give the oracle's state on a benchmark circuit"""
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N - N % 2)]
    g_ops, o_ops = circuit_ops(lines[:600])
    g_ops = [op for op in g_ops if max(op.qubits) <= N]
    o_ops = [op for op in o_ops if max(op[1]) <= N]
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    ctx.set_option(S._lib.OPT_ENGINE, engine)
    try:
        for dtype, tol, opt, default in ((S.C128, 1e-12, S._lib.OPT_TILE_BITS_C128, 12),
                                         (S.C64, 5e-5, S._lib.OPT_TILE_BITS_C64, 13)):
            ctx.set_option(opt, min(tile_bits, 13 if dtype == S.C64 else 12))
            try:
                st = S.CuState(ctx, N, dtype)
                S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
                assert rel(st.download().astype(complex), want) < tol, (engine, N, tile_bits, dtype)
            finally:
                ctx.set_option(opt, default)
    finally:
        ctx.set_option(S._lib.OPT_ENGINE, -1)


def hea_ops(N, L, theta_seed=42):
    """10 layers of [Ry all; Rz all; CZ ladder], gate-major params (Builder.jl:341-346)"""
    ops, idx = [], 1
    for _ in range(L):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
    rng = np.random.default_rng(theta_seed)
    theta = rng.uniform(0, 2 * np.pi, size=idx - 1)
    return ops, theta


def test_plain_method_small_config(ctx):
    """The plain-method configuration: N=20, complex128, 10 HEA layers (590 gates);
    <Z_i> and <Z_i Z_{i+1}> vs the oracle, relative error <= 1e-12."""
    N, L = 20, 10
    ops, theta = hea_ops(N, L)
    assert len(ops) == 590 and theta.size == 400
    o_ops = [(op.type, op.qubits, op.param_idx, 0.0) for op in ops]
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), theta, N)
    zw = np.array([O.expect_local(want, k, N, "z") for k in range(1, N + 1)])
    zzw = np.array([O.expect_corr(want, k, k + 1, N, "zz") for k in range(1, N)])
    for fused in (True, False):
        st = S.CuState(ctx, N, S.C128)
        S.apply_circuit(st, S.ParameterizedCircuit(N, ops), theta, fused=fused)
        got = st.download()
        assert rel(got, want) < 1e-12
        masks = [1 << q for q in range(N)] + [(3 << q) for q in range(N - 1)]
        v = S.expect_zstrings(st, masks)[0]
        assert np.max(np.abs(v[:N] - zw)) < 1e-12
        assert np.max(np.abs(v[N:] - zzw)) < 1e-12


def xxz_gates(N, dt, seed=42):
    rng = np.random.default_rng(seed)
    h = rng.uniform(-1, 1, size=N)
    bonds = [(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)]
    fields = [(i, 0.0, 0.0, float(h[i - 1])) for i in range(1, N + 1)]
    return bonds, fields


@pytest.mark.parametrize("N,dtype,tol", [(8, S.C128, 1e-12), (16, S.C128, 1e-12), (17, S.C64, 1e-4)])
def test_strang_trotter_vs_oracle(ctx, N, dtype, tol):
    """Second-order XXZ Trotter (gates at dt/2, list + reversed list) vs the oracle
    applying the same gates one by one; records of <Z_i> every 3 steps."""
    dt, steps, rec = 0.05, 7, 3
    bonds, fields = xxz_gates(N, dt)
    arr, n = O.precompute_trotter_gates(bonds, fields, dt / 2)
    gl = O.gates_to_list(arr, n)
    fwd = [(f, 0, 0) for f in range(n)]
    neel = sum(1 << (k - 1) for k in range(1, N + 1, 2))
    psi = O.zero_state(N, neel)
    rev = O.make_gates(gl + gl[::-1])
    want_rec = [[O.expect_local(psi, k, N, "z") for k in range(1, N + 1)]]
    for s in range(1, steps + 1):
        O.trotter_step(psi, rev, 2 * n, N)
        if s % rec == 0:
            want_rec.append([O.expect_local(psi, k, N, "z") for k in range(1, N + 1)])
    gates = [S.FastTrotterGate(idx, U) for idx, U in gl]
    plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=dtype)
    st = S.CuState(ctx, N, dtype, basis=neel)
    recs = plan.run(st, steps, rec)
    assert recs.shape == (steps // rec + 1, 1, N)
    assert np.max(np.abs(recs[:, 0, :] - np.array(want_rec))) < tol
    assert rel(st.download().astype(complex), psi) < (tol if dtype == S.C128 else 1e-4)
    assert len(fwd) == n


def test_trotter_graph_and_plain_paths_agree(ctx):
    N = 15
    bonds, fields = xxz_gates(N, 0.05)
    arr, n = O.precompute_trotter_gates(bonds, fields, 0.025)
    gates = [S.FastTrotterGate(idx, U) for idx, U in O.gates_to_list(arr, n)]
    plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=S.C128)
    a = S.CuState(ctx, N, S.C128, basis=5)
    b = S.CuState(ctx, N, S.C128, basis=5)
    plan.step(a, 23)
    ctx.set_option(S._lib.OPT_USE_GRAPHS, 0)
    try:
        plan.step(b, 23)
    finally:
        ctx.set_option(S._lib.OPT_USE_GRAPHS, 1)
    assert np.max(np.abs(a.download() - b.download())) == 0.0


def test_trotter_full_size_properties(ctx):
    """N=28 complex64 (the bench workload, 2 GiB): after 20 Strang steps the norm
    stays 1 to FP32 rounding and <Z> agrees with a complex128 GPU run of the same
    plan to 1e-5 (size-independent properties; the oracle is too slow at 2^28)."""
    N = 28
    bonds, fields = xxz_gates(N, 0.05)
    arr, n = O.precompute_trotter_gates(bonds, fields, 0.025)
    gates = [S.FastTrotterGate(idx, U) for idx, U in O.gates_to_list(arr, n)]
    neel = sum(1 << (k - 1) for k in range(1, N + 1, 2))
    res = {}
    for dtype in (S.C64, S.C128):
        plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=dtype)
        st = S.CuState(ctx, N, dtype, basis=neel)
        res[dtype] = plan.run(st, 20, 10)
        assert abs(S.get_norm(st) - 1.0) < (1e-4 if dtype == S.C64 else 1e-12)
        st.close()
        plan.close()
    assert np.max(np.abs(res[S.C64] - res[S.C128])) < 1e-5


@pytest.mark.parametrize("depth", [1, 3, 7])
def test_fusion_depth_cap_keeps_the_state(ctx, depth):
    """SMOQ_OPT_FUSION_DEPTH splits passes longer than `depth` fused ops into
    consecutive passes of the same tile: a benchmark circuit (one-shot, engine 0)
    and a Strang Trotter plan (compiled kernels) still equal the oracle"""
    N = 16
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N)]
    g_ops, o_ops = circuit_ops(lines[:400])
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    ctx.set_option(S._lib.OPT_FUSION_DEPTH, depth)
    try:
        st = S.CuState(ctx, N, S.C128)
        S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
        assert rel(st.download(), want) < 1e-12
        st.close()
        h = np.random.default_rng(5).uniform(-1, 1, size=N)
        arr, n = O.precompute_trotter_gates([(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)],
                                            [(i, 0.0, 0.0, float(h[i - 1])) for i in range(1, N + 1)], 0.025)
        gl = O.gates_to_list(arr, n)
        ref = O.zero_state(N, 0b1010101010101010)
        both = O.make_gates(gl + gl[::-1])
        for _ in range(3):
            O.trotter_step(ref, both, 2 * n, N)
        plan = S.TrotterPlan(ctx, N, [S.FastTrotterGate(i, U) for i, U in gl], order=2, dtype=S.C64)
        s2 = S.CuState(ctx, N, S.C64, basis=0b1010101010101010)
        plan.step(s2, 3)
        assert rel(s2.download().astype(complex), ref) < 1e-5
        s2.close()
        plan.close()
    finally:
        ctx.set_option(S._lib.OPT_FUSION_DEPTH, 0)


def test_autotune_modes_geometry_and_variants():
    """SMOQ_OPT_AUTOTUNE on a Trotter plan of N = 20 (compiled kernels): 1 times the
    candidate geometries and then the pass variants; 2 keeps the geometry the options
    set (here low bits 4) and tunes only the variants; both evolve to the oracle's
    state; values outside 0..2 are refused"""
    if not S.jit_available():
        pytest.skip("NVRTC not available")
    N = 20
    h = np.random.default_rng(11).uniform(-1, 1, size=N)
    arr, n = O.precompute_trotter_gates([(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)],
                                        [(i, 0.0, 0.0, float(h[i - 1])) for i in range(1, N + 1)], 0.025)
    gl = O.gates_to_list(arr, n)
    ref = O.zero_state(N, 0b10101010101010101010)
    both = O.make_gates(gl + gl[::-1])
    for _ in range(2):
        O.trotter_step(ref, both, 2 * n, N)
    reports = {}
    for mode in (1, 2):
        c = S.Context(0)
        try:
            with pytest.raises(S.SmoqError):
                c.set_option(S._lib.OPT_AUTOTUNE, 3)
            c.set_option(S._lib.OPT_AUTOTUNE, mode)
            if mode == 2:
                c.set_option(S._lib.OPT_LOW_BITS_C64, 4)
            plan = S.TrotterPlan(c, N, [S.FastTrotterGate(i, U) for i, U in gl], order=2, dtype=S.C64)
            st = S.CuState(c, N, S.C64, basis=0b10101010101010101010)
            plan.step(st, 2)
            assert rel(st.download().astype(complex), ref) < 1e-5
            reports[mode] = c.tune_report()
            st.close()
            plan.close()
        finally:
            c.close()
    assert "-> geometry" in reports[1] and reports[1].count("geometry tile") >= 2
    assert "geometry" not in reports[2] and "-> v" in reports[2]

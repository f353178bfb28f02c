"""GPU parity of the stage-sweep engine (fused-pass engine 2) and of the plan
compiler (engine 3, the same stage schedule compiled per pass with NVRTC).

The stage engine runs every fused pass of tile width 12 or 13 as 4-bit
register stages with XOR-rotated bank mapping; every other width falls back to
the shared-memory sweeps.  Engine 3 compiles each complex64 stage pass into
its own kernel (literal coefficients, compile-time addressing); complex128
passes run engine 2's kernel.  These tests switch the engine on and compare with
the oracle on the workloads that reach each op kind of a stage:
dense and parity 2-qubit ops on rotated and unrotated stage bits, 1- and
2-qubit permutations turned dense, 3-qubit permutations as plain sweeps,
diagonals on any bit, the MCWF renormalise/decay passes with their norm and
population epilogue, and the VQE forward passes."""
import json
import os

import numpy as np
import pytest

import oracle as O
import pysmoq as S

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(params=[2, 3], ids=["stage", "compiled"])
def eng(request):
    return request.param


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


class engine:
    """context manager: fused-pass engine and tile widths, restored on exit"""

    def __init__(self, ctx, e, tb64=13, tb128=12):
        self.ctx, self.e, self.tb64, self.tb128 = ctx, e, tb64, tb128

    def __enter__(self):
        self.ctx.set_option(S._lib.OPT_ENGINE, self.e)
        self.ctx.set_option(S._lib.OPT_TILE_BITS_C64, self.tb64)
        self.ctx.set_option(S._lib.OPT_TILE_BITS_C128, self.tb128)

    def __exit__(self, *a):
        self.ctx.set_option(S._lib.OPT_ENGINE, -1)
        self.ctx.set_option(S._lib.OPT_TILE_BITS_C64, 13)
        self.ctx.set_option(S._lib.OPT_TILE_BITS_C128, 12)


def bench_circuit(N, n=None):
    name = {"H": "h", "X": "x", "Y": "y", "Z": "z", "S": "s", "T": "t", "RX": "rx", "RY": "ry", "RZ": "rz",
            "CNOT": "cnot", "CZ": "cz"}
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N)]
    if n:
        lines = lines[:n]
    g_ops, o_ops = [], []
    for ln in lines:
        p = ln.split()
        t = name[p[0]]
        if t in ("cnot", "cz"):
            qs, ang = [int(p[1]) + 1, int(p[2]) + 1], 0.0
        else:
            qs, ang = [int(p[1]) + 1], (float(p[2]) if len(p) > 2 else 0.0)
        g_ops.append(S.gate(t, qs, angle=ang))
        o_ops.append((t, qs, 0, ang))
    return g_ops, o_ops


def random_circuit(N, n, seed):
    """every gate kind of the op ABI on random qubits, fixed angles"""
    rng = np.random.default_rng(seed)
    one = ["h", "x", "y", "z", "s", "t", "rx", "ry", "rz"]
    two = ["cnot", "cz", "rxx", "ryy", "rzz", "cry"]
    three = ["ccz", "toffoli"]
    g_ops, o_ops = [], []
    for _ in range(n):
        u = rng.random()
        if u < 0.4:
            t, qs = one[rng.integers(len(one))], [int(rng.integers(1, N + 1))]
        elif u < 0.9:
            t = two[rng.integers(len(two))]
            a = int(rng.integers(1, N + 1))
            b = a + 1 if (rng.random() < 0.5 and a < N) else int(rng.integers(1, N + 1))
            if b == a:
                b = a % N + 1
            qs = [a, b]
        else:
            t = three[rng.integers(len(three))]
            qs = [int(x) + 1 for x in rng.choice(N, 3, replace=False)]
        ang = float(rng.uniform(-np.pi, np.pi))
        g_ops.append(S.gate(t, qs, angle=ang))
        o_ops.append((t, qs, 0, ang))
    return g_ops, o_ops


@pytest.mark.parametrize("N", [12, 14, 16, 20])
@pytest.mark.parametrize("tb64", [12, 13])
def test_benchmark_circuits(ctx, eng, N, tb64):
    g_ops, o_ops = bench_circuit(N, 800)
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    with engine(ctx, eng, tb64=tb64):
        for dtype, tol in ((S.C128, 1e-12), (S.C64, 5e-5)):
            st = S.CuState(ctx, N, dtype)
            S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
            assert rel(st.download().astype(complex), want) < tol, (N, tb64, dtype)


@pytest.mark.parametrize("N,seed", [(12, 1), (13, 2), (15, 3), (18, 4)])
def test_random_circuits_every_gate_kind(ctx, eng, N, seed):
    # the plan compiler builds one kernel per distinct pass: a shorter circuit keeps
    # its compile time in check while still reaching every gate kind
    g_ops, o_ops = random_circuit(N, 500 if eng == 2 else 200, seed)
    rng = np.random.default_rng(seed + 100)
    psi = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    psi /= np.linalg.norm(psi)
    want = psi.copy()
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    with engine(ctx, eng):
        for dtype, tol in ((S.C128, 1e-12), (S.C64, 5e-5)):
            st = S.CuState(ctx, N, dtype, basis=None)
            st.upload(psi.astype(np.complex128 if dtype == S.C128 else np.complex64))
            S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
            assert rel(st.download().astype(complex), want) < tol, (N, seed, dtype)


def xxz(N, dt):
    rng = np.random.default_rng(42)
    h = rng.uniform(-1, 1, size=N)
    bonds = [(i, i + 1, 1.0, 1.0, 0.5) for i in range(1, N)]
    fields = [(i, 0.0, 0.0, float(h[i - 1])) for i in range(1, N + 1)]
    arr, n = O.precompute_trotter_gates(bonds, fields, dt / 2)
    return arr, n, O.gates_to_list(arr, n)


@pytest.mark.parametrize("N,dtype,tb64,tol", [(14, S.C128, 13, 1e-12), (16, S.C64, 13, 1e-4),
                                              (17, S.C64, 12, 1e-4)])
def test_strang_trotter(ctx, eng, N, dtype, tb64, tol):
    dt, steps, rec = 0.05, 6, 3
    arr, n, gl = xxz(N, dt)
    neel = sum(1 << (k - 1) for k in range(1, N + 1, 2))
    psi = O.zero_state(N, neel)
    both = O.make_gates(gl + gl[::-1])
    want_rec = [[O.expect_local(psi, k, N, "z") for k in range(1, N + 1)]]
    for s in range(1, steps + 1):
        O.trotter_step(psi, both, 2 * n, N)
        if s % rec == 0:
            want_rec.append([O.expect_local(psi, k, N, "z") for k in range(1, N + 1)])
    with engine(ctx, eng, tb64=tb64):
        plan = S.TrotterPlan(ctx, N, [S.FastTrotterGate(i, U) for i, U in gl], order=2, dtype=dtype)
        st = S.CuState(ctx, N, dtype, basis=neel)
        recs = plan.run(st, steps, rec)
        assert np.max(np.abs(recs[:, 0, :] - np.array(want_rec))) < tol
        assert rel(st.download().astype(complex), psi) < tol


def test_engines_agree_on_trotter_n22(ctx):
    """N=22 complex64 XXZ, 10 Strang steps (about 4,000 fused-op applications per
    amplitude): the shared-memory, stage and compiled engines each stay within FP32
    rounding of the complex128 result of the same plan (max |d psi| < 5e-6, relative
    L2 < 1e-5: engine 0 measured 1.7e-6 and 3.3e-6), and within 5e-6 of one another.  The compiled engine splits rotations
    and folds diagonals, so its roundings come in another order than engine 0's."""
    N = 22
    _, _, gl = xxz(N, 0.05)
    gates = [S.FastTrotterGate(i, U) for i, U in gl]
    out = {}
    for e, dt in ((0, S.C128), (0, S.C64), (2, S.C64), (3, S.C64)):
        with engine(ctx, e):
            plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=dt)
            st = S.CuState(ctx, N, dt, basis=5)
            plan.step(st, 10)
            out[(e, dt)] = st.download().astype(complex)
            st.close()
            plan.close()
    ref = out[(0, S.C128)]
    for e in (0, 2, 3):
        d = out[(e, S.C64)] - ref
        print(f"N=22 engine {e} c64 vs c128: max {np.max(np.abs(d)):.2e}, rel L2 {rel(out[(e, S.C64)], ref):.2e}")
        assert np.max(np.abs(d)) < 5e-6 and rel(out[(e, S.C64)], ref) < 1e-5
    assert np.max(np.abs(out[(0, S.C64)] - out[(2, S.C64)])) < 5e-6
    assert np.max(np.abs(out[(0, S.C64)] - out[(3, S.C64)])) < 5e-6


def test_mcwf_trajectory_exact(ctx, eng):
    """N=12 complex128 trajectories through stage passes (renormalise, decay
    table, norm/population epilogue) match the oracle's jump counts exactly"""
    N, dt, steps, rec, B, seed = 12, 0.05, 30, 5, 8, 99
    arr, n = O.precompute_trotter_gates([(i, i + 1, 0.0, 0.0, 1.0) for i in range(1, N)],
                                        [(i, 1.0, 0.0, 0.0) for i in range(1, N + 1)], dt)
    gates = [S.FastTrotterGate(idx, U) for idx, U in O.gates_to_list(arr, n)]
    gj = [S.JumpOperator("sigma_minus", q, 0.3) for q in range(1, N + 1)] + \
         [S.JumpOperator("sigma_z", q, 0.1) for q in range(1, N + 1)]
    oj = [(0, q, 0.3) for q in range(1, N + 1)] + [(2, q, 0.1) for q in range(1, N + 1)]
    idx = (1 << N) - 1
    with engine(ctx, eng):
        plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C128)
        st = S.CuState(ctx, N, S.C128, B, basis=idx)
        res = S.mcwf_run(plan, st, gj, dt, seed, steps, rec, traj_offset=3, per_trajectory=True)
    z, zz, nj = O.mcwf_run(N, arr, n, O.make_jumps(oj), len(oj), dt, seed, 3, B, steps, rec, init_index=idx,
                           nthreads=4)
    assert np.array_equal(res["jumps"], nj)
    assert nj.sum() > 0
    assert np.max(np.abs(res["z_traj"] - z)) < 1e-10
    assert np.max(np.abs(res["zz_traj"] - zz)) < 1e-10


def test_vqe_energy_and_gradient(ctx, eng):
    N, L = 13, 3
    ops, idx = [], 1
    for _ in range(L):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
    theta = np.random.default_rng(5).uniform(0, 2 * np.pi, size=idx - 1)
    circ = S.ParameterizedCircuit(N, ops)
    H = S.PauliSum.tfim(N)
    e0, g0 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    with engine(ctx, eng):
        e2, g2 = S.energy_and_gradient(ctx, circ, H, theta, dtype=S.C128)
    assert abs(e2[0] - e0[0]) < 1e-11
    assert np.max(np.abs(g2 - g0)) < 1e-10


def test_mcwf_complex64_epilogue_engines_agree(ctx, eng):
    """N=13 complex64 trajectories: the compiled passes with the norm/population
    epilogue give the stage engine's jump counts and records"""
    N, dt, steps, rec, B, seed = 13, 0.05, 20, 5, 16, 7
    arr, n = O.precompute_trotter_gates([(i, i + 1, 0.0, 0.0, 1.0) for i in range(1, N)],
                                        [(i, 1.0, 0.0, 0.0) for i in range(1, N + 1)], dt)
    gates = [S.FastTrotterGate(idx, U) for idx, U in O.gates_to_list(arr, n)]
    gj = [S.JumpOperator("sigma_minus", q, 0.3) for q in range(1, N + 1)]
    out = {}
    for e in (0, eng):
        with engine(ctx, e):
            plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C64)
            st = S.CuState(ctx, N, S.C64, B, basis=(1 << N) - 1)
            out[e] = S.mcwf_run(plan, st, gj, dt, seed, steps, rec, per_trajectory=True)
    assert np.array_equal(out[0]["jumps"], out[eng]["jumps"])
    assert np.max(np.abs(out[0]["z_traj"] - out[eng]["z_traj"])) < 1e-4


def test_engine_option_range(ctx):
    with pytest.raises(Exception):
        ctx.set_option(S._lib.OPT_ENGINE, 4)
    ctx.set_option(S._lib.OPT_ENGINE, -1)


@pytest.mark.parametrize("tb64", [12, 13])
def test_compiled_two_tile_buffers(ctx, tb64):
    """engine 3 with two tile buffers per CTA (next tile prefetched): Strang XXZ
    N=16 complex64 equals the oracle"""
    N, dt, steps = 16, 0.05, 4
    arr, n, gl = xxz(N, dt)
    neel = sum(1 << (k - 1) for k in range(1, N + 1, 2))
    psi = O.zero_state(N, neel)
    both = O.make_gates(gl + gl[::-1])
    for _ in range(steps):
        O.trotter_step(psi, both, 2 * n, N)
    ctx.set_option(S._lib.OPT_JIT_BUFFERS, 2)
    try:
        with engine(ctx, 3, tb64=tb64):
            plan = S.TrotterPlan(ctx, N, [S.FastTrotterGate(i, U) for i, U in gl], order=2, dtype=S.C64)
            st = S.CuState(ctx, N, S.C64, basis=neel)
            plan.step(st, steps)
            assert rel(st.download().astype(complex), psi) < 1e-4
    finally:
        ctx.set_option(S._lib.OPT_JIT_BUFFERS, 1)


@pytest.mark.parametrize("tb64", [12, 13])
def test_compiled_one_group_per_thread(ctx, tb64):
    """engine 3 with one 16-amplitude register group per thread (SMOQ_OPT_JIT_GROUPS 1):
    random circuit with every gate kind and a Strang XXZ sweep equal the oracle"""
    N, seed = 15, 12
    g_ops, o_ops = random_circuit(N, 200, seed)
    rng = np.random.default_rng(seed)
    psi = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    psi /= np.linalg.norm(psi)
    want = psi.copy()
    O.apply_circuit(want, O.make_ops(o_ops), len(o_ops), np.zeros(1), N)
    ctx.set_option(S._lib.OPT_JIT_GROUPS, 1)
    try:
        with engine(ctx, 3, tb64=tb64):
            st = S.CuState(ctx, N, S.C64, basis=None)
            st.upload(psi.astype(np.complex64))
            S.apply_circuit(st, S.ParameterizedCircuit(N, g_ops), np.zeros(1))
            assert rel(st.download().astype(complex), want) < 5e-5
            arr, n, gl = xxz(16, 0.05)
            neel = sum(1 << (k - 1) for k in range(1, 17, 2))
            ref = O.zero_state(16, neel)
            both = O.make_gates(gl + gl[::-1])
            for _ in range(3):
                O.trotter_step(ref, both, 2 * n, 16)
            plan = S.TrotterPlan(ctx, 16, [S.FastTrotterGate(i, U) for i, U in gl], order=2, dtype=S.C64)
            s2 = S.CuState(ctx, 16, S.C64, basis=neel)
            plan.step(s2, 3)
            assert rel(s2.download().astype(complex), ref) < 1e-4
    finally:
        ctx.set_option(S._lib.OPT_JIT_GROUPS, 2)

"""Host logic of the fused-pass planner, checked on CPU: smoq_debug_plan_sequence
returns the exact pass geometry and fused op program the GPU would run; a numpy
replay of that program must reproduce the oracle's gate-by-gate state, every
pass must be a legal tile (contiguous low segment >= 16 bytes, ops on tile
bits), and fusion must produce the op kinds the kernels specialise on."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def apply_local(psi, M, bits, N):
    """apply a 2^k x 2^k matrix whose index bit t is global qubit bits[t]"""
    k = len(bits)
    t = psi.reshape([2] * N)
    axes = [N - 1 - b for b in bits]            # C-order axis of index bit b
    t = np.moveaxis(t, axes[::-1], list(range(k)))  # axis 0 = bits[k-1] (most significant)
    sh = t.shape
    t = (M @ t.reshape(1 << k, -1)).reshape(sh)
    t = np.moveaxis(t, list(range(k)), axes[::-1])
    return t.reshape(-1)


def op_matrix(op):
    c = op["c"]
    nq = op["nq"]
    dim = 1 << nq
    k = op["kind"]
    if k == 0:
        return c[:4].reshape(2, 2)
    if k == 1:
        return c[:16].reshape(4, 4)
    if k == 2:
        M = np.zeros((4, 4), complex)
        M[0, 0], M[0, 3], M[3, 0], M[3, 3] = c[0], c[1], c[2], c[3]
        M[1, 1], M[1, 2], M[2, 1], M[2, 2] = c[4], c[5], c[6], c[7]
        return M
    if k == 3:
        M = np.zeros((dim, dim), complex)
        for r in range(dim):
            M[r, op["perm"][r]] = c[r]
        return M
    if k == 4:
        return np.diag(c[:dim])
    raise AssertionError(k)


def replay(plan, N, psi):
    for p in plan:
        for op in p["ops"]:
            if op["kind"] == 10:  # stage header: no arithmetic
                continue
            psi = apply_local(psi, op_matrix(op), op["gb"][:op["nq"]], N)
    return psi


def check_geometry(plan, N, dtype, tile_bits):
    import pysmoq as S
    for p in plan:
        assert len(p["ops"]) >= 1
        assert p["T"] <= max(tile_bits, 1) or p["T"] == N
        assert p["T"] == p["L"] + p["H"]
        if dtype == S.C64:
            assert p["L"] >= 1                 # segment >= 16 bytes
        assert all(p["L"] <= b < N for b in p["hb"]) and p["hb"] == sorted(p["hb"])
        for op in p["ops"]:
            for t in range(op["nq"]):
                g, lb = op["gb"][t], op["lb"][t]
                if lb >= 0:
                    assert (lb < p["L"] and g == lb) or (lb >= p["L"] and p["hb"][lb - p["L"]] == g)
                else:
                    assert op["kind"] == 4, "only diagonal ops may touch non-tile qubits"


def circuit(N, n=None):
    import pysmoq as S
    lines = json.load(open(os.path.join(GOLD, "circuits.json")))[str(N)]
    name = {"H": "h", "X": "x", "Y": "y", "Z": "z", "S": "s", "T": "t", "RX": "rx", "RY": "ry", "RZ": "rz",
            "CNOT": "cnot", "CZ": "cz"}
    g, o = [], []
    for ln in lines[:n]:
        p = ln.split()
        t = name[p[0]]
        qs = [int(p[1]) + 1] + ([int(p[2]) + 1] if t in ("cnot", "cz") else [])
        a = float(p[2]) if t in ("rx", "ry", "rz") else 0.0
        g.append(S.gate(t, qs, angle=a))
        o.append((t, qs, 0, a))
    return g, o


@pytest.mark.parametrize("N", [2, 4, 8, 10, 12])
@pytest.mark.parametrize("tile_bits,low_bits", [(4, 1), (6, 3), (8, 5), (12, 4), (14, 5)])
def test_replay_of_fused_plan_matches_oracle(built, N, tile_bits, low_bits):
    import pysmoq as S
    g, o = circuit(N, 300)
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o), len(o), np.zeros(1), N)
    for dtype in (S.C64, S.C128):
        tb = tile_bits if dtype == S.C64 else min(tile_bits, 13)
        plan = S.debug_plan(N, g, dtype=dtype, tile_bits=tb, low_bits=low_bits)
        check_geometry(plan, N, dtype, tb)
        got = replay(plan, N, O.zero_state(N))
        assert np.max(np.abs(got - want)) < 1e-12


def test_narrow_tiles_are_rejected_not_hung(built):
    import pysmoq as S
    g, _ = circuit(10, 50)
    with pytest.raises(S.SmoqError):
        S.debug_plan(10, g, dtype=S.C64, tile_bits=3, low_bits=3)


def test_xxz_strang_step_fuses_to_parity_ops(built):
    """A Strang step of the XXZ chain (Rz fields; Rxx, Ryy, Rzz per bond) must
    fuse every bond into one parity-block op and absorb the fields."""
    import pysmoq as S
    N = 16
    rng = np.random.default_rng(42)
    h = rng.uniform(-1, 1, size=N)
    s1 = [S.gate("rz", [i + 1], angle=2 * h[i] * 0.025) for i in range(N)]
    for i in range(1, N):
        s1 += [S.gate("rxx", [i, i + 1], angle=0.05), S.gate("ryy", [i, i + 1], angle=0.05),
               S.gate("rzz", [i, i + 1], angle=0.025)]
    ops = s1 + s1[::-1]
    plan = S.debug_plan(N, ops, dtype=S.C64, tile_bits=13, low_bits=5)
    kinds = [op["kind"] for p in plan for op in p["ops"] if op["kind"] != 8]
    assert set(kinds) <= {2, 4}, kinds
    assert len(kinds) <= 2 * (N - 1) + 2
    assert len(plan) <= 3
    # replay vs the oracle on the same gates
    o = [(op.type, op.qubits, 0, op.fixed_angle) for op in ops]
    want = O.zero_state(N, 0b0101010101010101)
    O.apply_circuit(want, O.make_ops(o), len(o), np.zeros(1), N)
    got = replay(plan, N, O.zero_state(N, 0b0101010101010101))
    assert np.max(np.abs(got - want)) < 1e-12


def test_diagonal_gates_need_no_tile_membership(built):
    """Rzz on far-apart qubits is diagonal: it rides along in the low-qubit pass."""
    import pysmoq as S
    N = 20
    ops = [S.gate("rx", [q], angle=0.1 * q) for q in range(1, 9)] + [S.gate("rzz", [1, 20], angle=0.3),
                                                                    S.gate("cz", [3, 17])]
    plan = S.debug_plan(N, ops, dtype=S.C64, tile_bits=12, low_bits=5)
    assert len(plan) == 1
    assert any(op["kind"] == 4 and -1 in op["lb"][:op["nq"]] for op in plan[0]["ops"])


def check_stages(plan, lb_bank):
    """stage-sweep schedule: every member op sits on its stage's 4 bits, 2-qubit
    members in ascending stage positions, the bank rotation uses distinct lane
    bits exactly for the stage bits below the bank boundary"""
    for p in plan:
        ops = p["ops"]
        i = 0
        while i < len(ops):
            h = ops[i]
            assert h["kind"] == 10
            i += 1
            if h["nq"] == 0:                      # single wide op, plain sweep
                assert ops[i]["nq"] == 3 and ops[i]["kind"] == 3
                i += 1
                continue
            S = h["perm"][:4]
            assert S == sorted(S) and len(set(S)) == 4 and all(0 <= b < p["T"] for b in S)
            rot = h["perm"][4:]
            free_low = sum(1 for b in range(lb_bank) if b not in S)
            lanes = [r for r in rot if r >= 0]
            assert [r >= 0 for r in rot] == [b < lb_bank for b in S]
            assert sorted(lanes) == list(range(free_low, free_low + len(lanes)))
            while i < len(ops) and ops[i]["kind"] != 10:
                op = ops[i]
                if op["kind"] not in (4, 5, 6):
                    assert op["kind"] in (0, 1, 2), "permutations of 1-2 qubits run as dense stage ops"
                    pos = op["slot"][:op["nq"]]
                    assert all(S[q] == op["lb"][t] for t, q in enumerate(pos))
                    if op["nq"] == 2:
                        assert pos[0] < pos[1]
                i += 1


@pytest.mark.parametrize("N", [12, 13, 15])
@pytest.mark.parametrize("dtype,tile_bits", [("c64", 12), ("c64", 13), ("c128", 12)])
def test_stage_schedule_replays_and_is_well_formed(built, N, dtype, tile_bits):
    import pysmoq as S
    dt = S.C64 if dtype == "c64" else S.C128
    rng = np.random.default_rng(N)
    g, o = circuit(N - N % 2, 400)
    g = [x for x in g if max(x.qubits) <= N]
    o = [x for x in o if max(x[1]) <= N]
    # permutations, parity bonds and 3-qubit ops on top of the benchmark circuit
    for _ in range(40):
        a = int(rng.integers(1, N))
        t = ["swap_like", "rxx", "ryy", "toffoli", "cnot"][int(rng.integers(5))]
        if t == "toffoli":
            qs = [int(x) + 1 for x in rng.choice(N, 3, replace=False)]
        else:
            qs = [a, a + 1]
            t = "rzz" if t == "swap_like" else t
        ang = float(rng.uniform(-3, 3))
        g.append(S.gate(t, qs, angle=ang))
        o.append((t, qs, 0, ang))
    plan = S.debug_plan(N, g, dtype=dt, tile_bits=tile_bits, low_bits=5 if dt == S.C64 else 4, engine=2)
    staged = [p for p in plan if p["T"] == 12 or (p["T"] == 13 and dt == S.C64)]
    assert staged, "no pass wide enough for the stage engine"
    check_stages(staged, 4 if dt == S.C64 else 3)
    want = O.zero_state(N)
    O.apply_circuit(want, O.make_ops(o), len(o), np.zeros(1), N)
    got = replay(plan, N, O.zero_state(N))
    assert np.max(np.abs(got - want)) < 1e-12


@pytest.mark.parametrize("N,tile_bits", [(13, 12), (16, 13), (20, 13)])
def test_plan_compiler_generates_valid_kernels(built, N, tile_bits):
    """engine 3 (host only): every complex64 stage pass of a circuit with every gate
    kind compiles with NVRTC for sm_100a, with at most a few bytes of spills"""
    import pysmoq as S
    rng = np.random.default_rng(N)
    kinds = ["h", "rx", "rz", "t", "cnot", "cz", "rxx", "ryy", "rzz", "cry", "toffoli", "ccz"]
    g = []
    for _ in range(120):
        t = kinds[int(rng.integers(len(kinds)))]
        k = 3 if t in ("toffoli", "ccz") else (2 if t in ("cnot", "cz", "rxx", "ryy", "rzz", "cry") else 1)
        qs = [int(x) + 1 for x in rng.choice(N, k, replace=False)]
        g.append(S.gate(t, qs, angle=float(rng.uniform(-3, 3))))
    st, n, msg = S.debug_compile_plan(N, g, dtype=S.C64, tile_bits=tile_bits, verbose=True)
    if st == 5:
        pytest.skip("NVRTC not available: " + msg)
    assert st == 0, msg
    assert n >= 1
    import re
    spills = [int(m) for m in re.findall(r"(\d+) bytes spill stores", msg)]
    assert len(spills) == n, msg          # one compiler report per kernel
    assert max(spills) <= 64, msg


@pytest.mark.parametrize("N", [16, 24])
def test_run_time_coefficient_forward_kernels(built, N):
    """the compiled forward passes of a variational circuit with the coefficients
    passed per launch (host only): they compile without spills beyond a few bytes,
    and a second parameter set gives the same kernel source"""
    import pysmoq as S
    import re
    rng = np.random.default_rng(N)
    ops, idx = [], 1
    for layer in range(6):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
        ops.append(S.gate("rxx", [1 + layer, N - layer], param_idx=idx)); idx += 1
        ops.append(S.gate("toffoli", [2, 5 + layer, N]))
    th = [rng.uniform(0, 2 * np.pi, size=idx - 1) for _ in range(2)]
    st, n, msg = S.debug_compile_plan(N, ops, theta=th[0], rtc=True, verbose=True)
    if st == 5:
        pytest.skip("NVRTC not available: " + msg)
    assert st == 0, msg
    spills = [int(m) for m in re.findall(r"(\d+) bytes spill stores", msg)]
    assert n >= 1 and len(spills) == n and max(spills) <= 64, msg
    srcs = [S.debug_compile_plan(N, ops, theta=t, rtc=True, source=True) for t in th]
    assert srcs[0][0] == 0 and "Coefs K" in srcs[0][2] and srcs[0][2] == srcs[1][2]
    lit = [S.debug_compile_plan(N, ops, theta=t, source=True) for t in th]
    assert "Coefs" not in lit[0][2] and lit[0][2] != lit[1][2]   # literal form: the angles are in the source


@pytest.mark.parametrize("N,L,kinds", [(24, 6, ("ry", "rz")), (16, 4, ("rx", "ry", "rz")), (14, 3, "mixed")])
def test_compiled_adjoint_kernels_compile(built, N, L, kinds):
    """the compiled adjoint kernels of smoq_energy_grad (host only): every backward pass
    of tile width 12 of a variational circuit is stage-scheduled and compiles with
    NVRTC, with at most a few bytes of spills; the angles do not enter the source"""
    import pysmoq as S
    import re
    rng = np.random.default_rng(N)
    ops, idx = [], 1
    for layer in range(L):
        if kinds == "mixed":
            for q in range(1, N + 1):
                t = str(rng.choice(["rx", "ry", "rz", "h", "t"]))
                if t in ("h", "t"):
                    ops.append(S.gate(t, q))
                else:
                    ops.append(S.gate(t, q, param_idx=idx))
                    idx += 1
            for q in range(1, N):
                t = str(rng.choice(["cz", "cnot", "rxx", "ryy", "rzz", "cry"]))
                if t in ("cz", "cnot"):
                    ops.append(S.gate(t, [q, q + 1]))
                else:
                    ops.append(S.gate(t, [q, 1 + (q + 2 * layer) % N if 1 + (q + 2 * layer) % N != q else q + 1],
                                      param_idx=idx))
                    idx += 1
        else:
            rot, idx = S.single_qubit_rotation_layer(N, idx, gates=kinds)
            ops += rot + S.entangling_layer(N, "chain", "cz")
    circ = S.ParameterizedCircuit(N, ops)
    theta = rng.uniform(0, 2 * np.pi, size=circ.n_params)
    st, npass, ncomp, msg = S.debug_compile_adjoint(circ, theta, verbose=True)
    if st == 5:
        pytest.skip("NVRTC not available: " + msg)
    assert st == 0, msg
    assert npass >= 1 and ncomp == npass, (npass, ncomp)
    # (a few spilled registers on the longest passes: that build measured fastest on the GPU)
    spills = [int(m) for m in re.findall(r"(\d+) bytes spill stores", msg)]
    assert len(spills) == ncomp and max(spills) <= 256, msg
    # another parameter set of the same circuit: the same kernel source
    srcs = [S.debug_compile_adjoint(circ, th, source=True)
            for th in (theta, rng.uniform(0, 2 * np.pi, size=circ.n_params))]
    assert srcs[0][0] == 0 and srcs[1][0] == 0
    assert "smoq_adj_e0" in srcs[0][3] and srcs[0][3] == srcs[1][3]


def xxz_strang(S, N, seed=42, dt=0.05):
    rng = np.random.default_rng(seed)
    h = rng.uniform(-1, 1, size=N)
    s1 = [S.gate("rz", [i + 1], angle=2 * h[i] * dt / 2) for i in range(N)]
    for i in range(1, N):
        s1 += [S.gate("rxx", [i, i + 1], angle=dt), S.gate("ryy", [i, i + 1], angle=dt),
               S.gate("rzz", [i, i + 1], angle=dt / 2)]
    ops = s1 + s1[::-1]
    return ops, [(op.type, op.qubits, 0, op.fixed_angle) for op in ops]


@pytest.mark.parametrize("N", [13, 16, 20])
def test_compiled_plan_splits_rotations_exactly(built, N):
    """engine 3 (literal compiled kernels): every complex 2x2 rotation block of a
    1-qubit or parity op is split into diagonal . [[c, -is], [-is, c]] . diagonal;
    the split program replays to the oracle's state (1e-12), keeps the stage
    schedule well formed, and the XXZ bonds' rotations have only real and
    imaginary coefficients"""
    import pysmoq as S
    ops, o = xxz_strang(S, N)
    g2, o2 = circuit(N - N % 2, 300)
    for gates, oo in ((ops + ops, o + o), (g2, o2)):
        plan = S.debug_plan(N, gates, dtype=S.C64, tile_bits=13, low_bits=5, engine=3)
        staged = [p for p in plan if p["T"] == 13]
        assert staged
        check_stages(staged, 4)
        want = O.zero_state(N, 0b0101010101010101 & ((1 << N) - 1))
        O.apply_circuit(want, O.make_ops(oo), len(oo), np.zeros(1), N)
        got = replay(plan, N, O.zero_state(N, 0b0101010101010101 & ((1 << N) - 1)))
        assert np.max(np.abs(got - want)) < 1e-12
    plan = S.debug_plan(N, ops, dtype=S.C64, tile_bits=13, low_bits=5, engine=3)
    par = [op for p in plan if p["T"] == 13 for op in p["ops"] if op["kind"] == 2]
    assert par
    for op in par:
        c = op["c"][:8]
        for blk in (c[0:4], c[4:8]):
            assert abs(blk[0].imag) < 1e-15 and abs(blk[3].imag) < 1e-15 and abs(blk[0] - blk[3]) < 1e-15
            assert abs(blk[1].real) < 1e-15 and abs(blk[2].real) < 1e-15 and abs(blk[1] - blk[2]) < 1e-15
    # engine 2 keeps the fused ops whole
    plan2 = S.debug_plan(N, ops, dtype=S.C64, tile_bits=13, low_bits=5, engine=2)
    assert sum(len(p["ops"]) for p in plan2) < sum(len(p["ops"]) for p in plan)


def test_autotuner_geometry_rule(built):
    """the plan autotuner keeps its default geometry (candidate 0) unless another
    candidate's timed run is faster by more than 2% (one run each: smaller
    differences are noise); unplannable candidates (< 0) never win"""
    import ctypes as C
    import pysmoq as S

    def pick(ms):
        a = (C.c_float * len(ms))(*ms)
        return S.lib.smoq_debug_pick_geometry(a, len(ms))
    assert pick([53.46, 53.12, 53.74, 65.90, 59.29]) == 0      # 0.6% faster: noise, keep the default
    assert pick([62.0, 55.0, 67.9, 77.2, 67.2]) == 1           # 11% faster: switch
    assert pick([10.0, 9.85, 9.82, 12.0]) == 0                 # within 2% of the default
    assert pick([10.0, 9.7, 9.79, 12.0]) == 1                  # 3% faster
    assert pick([-1.0, 20.0, 18.0]) == 2                       # no default run: the fastest
    assert pick([-1.0, -1.0]) == -1
    assert pick([5.0]) == 0

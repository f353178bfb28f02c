"""The plan compiler's generated arithmetic, run on the host.

A literal compiled pass kernel (engine 3) is a tile loader around straight-line stage
blocks: each thread loads its register groups of the tile, applies the stage's members
with float literals, and stores them back; a barrier separates the stages, and no thread
touches another thread's amplitudes inside a stage.  Running every stage block for every
thread index in turn, on the host, is therefore exactly what the kernel computes on one
tile.  These tests extract the stage blocks from the generated source, compile them with
g++ into one host function per pass, apply each pass to every tile of the state (gathered
and scattered on the host by the pass's geometry: the low bits and the chosen high bits,
the tile's base index for the ops that read bits off the tile), and compare the result
with the oracle's gate-by-gate complex128 evolution of the same circuit: the planner's
passes, the rotation split, the diagonal folding, members moved through the pending
phases and the phases absorbed into member rows must all be exact algebra (FP32 rounding
aside)."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from test_planner_cpu import circuit, xxz_strang

_HOST_PRELUDE = r"""
typedef unsigned int u32;
typedef unsigned long long u64;
struct cf { float x, y; };
struct HostOp { cf c[16]; };          // the coefficients a mixed diagonal reads at run time
struct HostArgs { const HostOp* ops; };
struct HostCoefs { const cf* k; };    // a run-time-coefficient kernel's parameter block
static inline cf cmul(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
static inline cf cscale(cf a, float s) { return cf{a.x * s, a.y * s}; }
"""

_STAGE = re.compile(r"\n    \{  // stage S = \{[^\n]*\n(.*?)\n    \}\n    __syncthreads\(\);", re.S)


def host_library(src, tmp_path, name):
    """one host function per generated kernel source: run_<k>(tile, ops, base, coefs)
    applies that kernel's stage blocks, thread by thread, to one tile (ops: the pass's
    fused ops' complex64 coefficients, in the pass's op order; base: the tile's first
    amplitude index; coefs: the run-time coefficient block of a run-time-coefficient
    kernel).  Returns the library and each kernel's coefficient block (or None)."""
    kernels = [s for s in src.split("\ntypedef unsigned int u32;") if "// stage S" in s]
    body = [_HOST_PRELUDE]
    blocks_k = []
    for k, ks in enumerate(kernels):
        nt = int(re.search(r"#define NT (\d+)", ks).group(1))
        blocks = _STAGE.findall(ks)
        assert blocks, "no stage blocks in a compiled pass"
        for b in blocks:  # the stage blocks use the tile, tid, literals, a.ops[m].c, K.k[i] and base
            assert len(re.findall(r"\ba\.", b)) == len(re.findall(r"\ba\.ops\[", b)), b[:200]
        m = re.search(r"//@coefs([^\n]*)", ks)
        if m:
            v = [float.fromhex(x) for x in m.group(1).split()]
            blocks_k.append(np.array(v[0::2], np.float32) + 1j * np.array(v[1::2], np.float32))
        else:
            assert "K.k[" not in ks
            blocks_k.append(None)
        body.append(f'extern "C" void run_{k}(cf* tile, const HostOp* ops, u64 base, const cf* kc) {{\n'
                    f'  const HostArgs a{{ops}};\n  const HostCoefs K{{kc}};\n  (void)base; (void)K;\n')
        for b in blocks:
            body.append(f"  for (u32 tid = 0; tid < {nt}u; ++tid) {{\n{b}\n  }}\n")
        body.append("}\n")
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text("".join(body))
    subprocess.run(["g++", "-O0", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so), str(cpp)], check=True)
    return C.CDLL(str(so)), blocks_k


def random_gates(N, n, seed):
    import pysmoq as S
    rng = np.random.default_rng(seed)
    one = ["rx", "ry", "rz", "h", "s", "t", "sdg", "x", "y", "z"]
    two = ["cnot", "cz", "rxx", "ryy", "rzz", "cry"]
    g, o = [], []
    for _ in range(n):
        u = rng.random()
        if u < 0.5:
            t = one[rng.integers(len(one))]
            qs = [int(rng.integers(N)) + 1]
        elif u < 0.92:
            t = two[rng.integers(len(two))]
            qs = [int(q) + 1 for q in rng.choice(N, 2, replace=False)]
        else:
            t = "toffoli" if rng.random() < 0.5 else "ccz"
            qs = [int(q) + 1 for q in rng.choice(N, 3, replace=False)]
        a = float(rng.uniform(0, 2 * np.pi)) if t in ("rx", "ry", "rz", "rxx", "ryy", "rzz", "cry") else 0.0
        g.append(S.gate(t, qs, angle=a))
        o.append((t, qs, 0, a))
    return g, o


def tile_offsets(N, L, hb):
    """amplitude index offsets of a tile's elements in tile order (the high bits hb
    above the low L bits), and the first index of every tile (zeros at the tile's bits)"""
    H = len(hb)
    dep = np.zeros(1 << H, dtype=np.int64)
    for m, q in enumerate(hb):
        dep |= ((np.arange(1 << H) >> m) & 1).astype(np.int64) << q
    off = (dep[:, None] | np.arange(1 << L, dtype=np.int64)[None, :]).reshape(-1)
    bases = []
    for t in range(1 << (N - L - H)):
        x = t << L
        for q in hb:  # ascending: insert a zero bit at each tile position
            x = ((x >> q) << (q + 1)) | (x & ((1 << q) - 1))
        bases.append(x)
    return off, bases


CASES = {"xxz_n13": (13, 5), "bench_circuit_n12": (12, 5), "random_n13": (13, 5),
         "xxz_n18_low5": (18, 5), "xxz_n18_low4": (18, 4), "random_n16": (16, 5)}


def replay(S, N, g, low, tmp_path, name, rtc=False, groups=2):
    """the state after every compiled pass of `g`, run on the host from a seeded random
    state (complex64), and that initial state"""
    st, n, src = S.debug_compile_plan(N, g, tile_bits=13, low_bits=low, all_sources=True, rtc=rtc, groups=groups)
    if st == 5:
        pytest.skip("NVRTC not available: " + src)
    assert st == 0 and n >= 1, src[:500]
    lib, coefs = host_library(src, tmp_path, name)
    nk = len(coefs)
    assert nk == n and all((c is not None) == rtc for c in coefs)
    rng = np.random.default_rng(3)
    psi0 = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    psi0 /= np.linalg.norm(psi0)
    # the passes' op tables (for the ops that read coefficients at run time): the
    # run-time-coefficient form schedules like engine 2 (no rotation split)
    plan = S.debug_plan(N, g, dtype=S.C64, tile_bits=13, low_bits=low, engine=2 if rtc else 3)
    assert len(plan) == nk
    psi = psi0.astype(np.complex64)
    for k, p in enumerate(plan):
        cf = np.zeros((max(1, len(p["ops"])), 16), np.complex64)
        for m, op in enumerate(p["ops"]):
            cf[m] = op["c"][:16]
        off, bases = tile_offsets(N, p["L"], p["hb"])
        assert len(off) == 1 << p["T"] and len(bases) << p["T"] == 1 << N
        run = getattr(lib, f"run_{k}")
        kc = coefs[k] if coefs[k] is not None else np.zeros(1, np.complex64)
        for base in bases:
            idx = base | off
            tile = np.ascontiguousarray(psi[idx])
            run(tile.ctypes.data_as(C.c_void_p), cf.ctypes.data_as(C.c_void_p), C.c_uint64(base),
                kc.ctypes.data_as(C.c_void_p))
            psi[idx] = tile
    return psi, psi0


def case_gates(S, case):
    N, low = CASES[case]
    if case.startswith("xxz"):
        g, o = xxz_strang(S, N)
        g, o = g + g + g, o + o + o   # three Strang steps: the merged half steps fold across
    elif case.startswith("bench"):
        g, o = circuit(N, 400)
    else:
        g, o = random_gates(N, 240, 7)
    return N, low, g, o


@pytest.mark.parametrize("rtc", [False, True], ids=["literal", "run_time_coefficients"])
@pytest.mark.parametrize("case", list(CASES))
def test_generated_stage_code_replays_on_host(built, tmp_path, case, rtc):
    """literal kernels (Trotter plans, MCWF) and the run-time-coefficient form (the
    complex64 forward of smoq_energy_grad: coefficients read from the launch's
    parameter block) of the same program"""
    import pysmoq as S
    N, low, g, o = case_gates(S, case)
    psi, psi0 = replay(S, N, g, low, tmp_path, case, rtc=rtc)
    want = psi0.astype(np.complex128).copy()
    O.apply_circuit(want, O.make_ops(o), len(o), np.zeros(1), N)
    err = np.linalg.norm(psi.astype(np.complex128) - want) / np.linalg.norm(want)
    print(case, rtc, "relative L2", err)
    assert err < 2e-6, err   # FP32 rounding over the circuit: measured 4e-7 to 6e-7


@pytest.mark.parametrize("case", ["xxz_n18_low4", "random_n16"])
def test_register_group_variants_are_bit_identical(built, tmp_path, case):
    """the autotuner's register-group variants (two 16-amplitude groups per thread, or one
    with twice the threads) apply the same literal arithmetic to every amplitude: the
    host replays of both give the same bits"""
    import pysmoq as S
    N, low, g, _ = case_gates(S, case)
    two, _ = replay(S, N, g, low, tmp_path, case + "_g2", groups=2)
    one, _ = replay(S, N, g, low, tmp_path, case + "_g1", groups=1)
    assert np.array_equal(two.view(np.uint32), one.view(np.uint32))


def test_bench_program_multiply_count(built):
    """the generated arithmetic of three Strang steps of the N=28 XXZ bench program
    (tile 13, low bits 5; 19 compiled passes): FP32 multiplies, counted as the literal
    coefficient terms of the stage code.  Flushing the pending phases before every member
    gave 23,920; moving members through the phases and absorbing the final phases into
    member rows gives 18,640.  A regression to flushing shows here, not in the parity
    tests (both forms are exact)."""
    import pysmoq as S
    g, _ = xxz_strang(S, 28)
    st, n, src = S.debug_compile_plan(28, g + g + g, tile_bits=13, low_bits=5, all_sources=True)
    if st == 5:
        pytest.skip("NVRTC not available: " + src)
    assert st == 0 and n == 19, (st, n)
    stages = "".join(_STAGE.findall(src))
    mults = len(re.findall(r"\* [vx]\d", stages))
    assert mults <= 19000, mults

"""The plan compiler's generated arithmetic, run on the host.

A literal compiled pass kernel (engine 3) is a tile loader around straight-line stage
blocks: each thread loads its register groups of the tile, applies the stage's members
with float literals, and stores them back; a barrier separates the stages, and no thread
touches another thread's amplitudes inside a stage.  When the whole state is one tile
(N = tile width), running every stage block for every thread index in turn, on the host,
is exactly what the kernel computes on the tile.  These tests extract the stage blocks
from the generated source, compile them with g++ into one host function, and compare the
result with the oracle's gate-by-gate complex128 evolution of the same circuit: the
rotation split, the diagonal folding, members moved through the pending phases and the
phases absorbed into member rows must all be exact algebra (FP32 rounding aside)."""
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
static inline cf cmul(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
static inline cf cscale(cf a, float s) { return cf{a.x * s, a.y * s}; }
"""

_STAGE = re.compile(r"\n    \{  // stage S = \{[^\n]*\n(.*?)\n    \}\n    __syncthreads\(\);", re.S)


def host_library(src, tmp_path, name):
    """one host function per generated kernel source: run_<k>(tile, ops) applies that
    kernel's stage blocks, thread by thread, to one tile (ops: the pass's fused ops'
    complex64 coefficients, in the pass's op order)"""
    kernels = [s for s in src.split("\ntypedef unsigned int u32;") if "// stage S" in s]
    body = [_HOST_PRELUDE]
    for k, ks in enumerate(kernels):
        nt = int(re.search(r"#define NT (\d+)", ks).group(1))
        blocks = _STAGE.findall(ks)
        assert blocks, "no stage blocks in a compiled pass"
        for b in blocks:  # the stage blocks use the tile, tid, literals and a.ops[m].c
            assert "base" not in b and len(re.findall(r"\ba\.", b)) == len(re.findall(r"\ba\.ops\[", b)), b[:200]
        body.append(f'extern "C" void run_{k}(cf* tile, const HostOp* ops) {{\n  const HostArgs a{{ops}};\n')
        for b in blocks:
            body.append(f"  for (u32 tid = 0; tid < {nt}u; ++tid) {{\n{b}\n  }}\n")
        body.append("}\n")
    cpp = tmp_path / f"{name}.cpp"
    so = tmp_path / f"{name}.so"
    cpp.write_text("".join(body))
    subprocess.run(["g++", "-O1", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so), str(cpp)], check=True)
    return C.CDLL(str(so)), len(kernels)


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


@pytest.mark.parametrize("case", ["xxz_n13", "bench_circuit_n12", "random_n13"])
def test_generated_stage_code_replays_on_host(built, tmp_path, case):
    import pysmoq as S
    if case == "xxz_n13":
        N = 13
        g, o = xxz_strang(S, N)
        g, o = g + g + g, o + o + o   # three Strang steps: the merged half steps fold across
    elif case == "bench_circuit_n12":
        N = 12
        g, o = circuit(N, 400)
    else:
        N = 13
        g, o = random_gates(N, 240, 7)
    st, n, src = S.debug_compile_plan(N, g, tile_bits=13, low_bits=5, all_sources=True)
    if st == 5:
        pytest.skip("NVRTC not available: " + src)
    assert st == 0 and n >= 1, src[:500]
    lib, nk = host_library(src, tmp_path, case)
    assert nk == n
    rng = np.random.default_rng(3)
    psi0 = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    psi0 /= np.linalg.norm(psi0)
    want = psi0.astype(np.complex128).copy()
    O.apply_circuit(want, O.make_ops(o), len(o), np.zeros(1), N)
    plan = S.debug_plan(N, g, dtype=S.C64, tile_bits=13, low_bits=5, engine=3)
    assert len(plan) == nk
    tile = psi0.astype(np.complex64)
    for k in range(nk):
        cf = np.zeros((max(1, len(plan[k]["ops"])), 16), np.complex64)
        for m, op in enumerate(plan[k]["ops"]):
            cf[m] = op["c"][:16]
        getattr(lib, f"run_{k}")(tile.ctypes.data_as(C.c_void_p), cf.ctypes.data_as(C.c_void_p))
    err = np.max(np.abs(tile.astype(np.complex128) - want))
    assert err < 2e-6 * max(1, len(o) // 100), err

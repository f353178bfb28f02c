// jit.cpp -- the plan compiler (fused-pass engine 3).
//
// A Trotter plan (or any reused op program) runs the same few pass programs
// hundreds of times.  Engine 3 turns each stage-scheduled pass into its own
// kernel, generated as CUDA C++ and compiled with NVRTC for sm_100a when the
// program is uploaded:
//   * the pass geometry (tile bits, segment layout), every stage's 4 bits,
//     thread->group deposit masks and register addresses are literals, so a
//     shared-memory access is one load/store with an immediate offset;
//   * every op's matrix is written out as straight-line complex FMAs with
//     the coefficients as float literals; zero entries are dropped, so
//     parity-preserving and permutation matrices cost only their nonzeros,
//     and there is no per-op dispatch, decode or coefficient load;
//   * stages on bank-selecting bits read through the same per-thread XOR
//     rotation as engine 2, then put the registers back in canonical order
//     with selects, so the coefficients stay literal;
//   * diagonals on bits outside the stage, per-state scales and decay tables
//     read their runtime data from the pass's DevOp array, as in engine 2.
// Kernels are cached by source text for the life of the process.  NVRTC is
// loaded with dlopen on first use: without it, engine 3 reports
// SMOQ_ERR_UNSUPPORTED and engines 0-2 are unaffected.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <stddef.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "smoq_internal.h"

namespace smoq {

namespace {

// ------------------------------------------------------------------ NVRTC
struct Nvrtc {
    bool tried = false, ok = false;
    std::string why;
    decltype(&::nvrtcCreateProgram) create = nullptr;
    decltype(&::nvrtcCompileProgram) compile = nullptr;
    decltype(&::nvrtcGetProgramLogSize) logsize = nullptr;
    decltype(&::nvrtcGetProgramLog) log = nullptr;
    decltype(&::nvrtcGetCUBINSize) cubinsize = nullptr;
    decltype(&::nvrtcGetCUBIN) cubin = nullptr;
    decltype(&::nvrtcDestroyProgram) destroy = nullptr;
};

Nvrtc load_nvrtc() {
    Nvrtc n;
    n.tried = true;
    const char* names[] = {"libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so"};
    void* h = nullptr;
    for (const char* nm : names)
        if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
        n.why = "NVRTC (libnvrtc.so.12) not found";
        return n;
    }
#define SYM(f, s)                                                 \
    n.f = reinterpret_cast<decltype(n.f)>(dlsym(h, s));           \
    if (!n.f) {                                                   \
        n.why = std::string("NVRTC symbol missing: ") + s;         \
        return n;                                                 \
    }
    SYM(create, "nvrtcCreateProgram")
    SYM(compile, "nvrtcCompileProgram")
    SYM(logsize, "nvrtcGetProgramLogSize")
    SYM(log, "nvrtcGetProgramLog")
    SYM(cubinsize, "nvrtcGetCUBINSize")
    SYM(cubin, "nvrtcGetCUBIN")
    SYM(destroy, "nvrtcDestroyProgram")
#undef SYM
    n.ok = true;
    return n;
}

Nvrtc& nvrtc() {
    static Nvrtc n = load_nvrtc();  // thread-safe one-time load
    return n;
}

// --------------------------------------------------------------- prelude
// Device-side definitions every generated kernel starts with.  The structs
// mirror DevOp / TileArgs member for member (same order and types; the
// generated static_asserts check their sizes against the host's).
const char* kPrelude = R"PRE(
typedef unsigned int u32;
typedef unsigned long long u64;
typedef long long i64;
struct __align__(8) cf { float x, y; };
struct __align__(16) cd2 { double x, y; };
struct __align__(16) DevOp {
    int kind, nq, lb[4], gb[4], slot[4], mode, flags, pad0[2], perm[8];
    const void* aux;
    i64 aux2;
    cd2 cd[16];
    cf c[16];
};
struct TileGeom { int N, T, L, H; int hb[24]; };
struct Epilogue { double* partials; int npop; int popq[40]; };
struct TileArgs {
    void* psi;
    i64 state_len, tiles_per_state, ntiles;
    const DevOp* ops;
    int nops;
    int* err;
    TileGeom g;
    Epilogue ep;
};
__device__ __forceinline__ cf cmul(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cf cscale(cf a, float s) { return cf{a.x * s, a.y * s}; }
__device__ __forceinline__ double cabs2d(cf a) { return (double)a.x * a.x + (double)a.y * a.y; }
__device__ __forceinline__ u64 ins0(u64 x, int p) { return ((x >> p) << (p + 1)) | (x & ((1ull << p) - 1)); }
__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(u64* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64* bar, u32 parity) {
    u32 ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ u64 globaltimer_ns() { u64 t; asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t)); return t; }
// bounded wait: 2 s of wall time or 2^22 polls, then the error word and false
__device__ __forceinline__ bool mbar_wait_bounded(u64* bar, u32 parity, int* err) {
    const u64 t0 = globaltimer_ns();
    for (int it = 0; it < (1 << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63 && globaltimer_ns() - t0 > 2000000000ull) break;
    }
    if (err) atomicExch(err, 1);
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, u32 bytes, u64* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, u32 bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
)PRE";

// ------------------------------------------------------------ code helpers
std::string flit(float v) {
    char b[64];
    std::snprintf(b, sizeof b, "%a", (double)v);
    return std::string("(") + b + "f)";
}

// deposit of thread-index bits around the sorted stage bits S: segment masks
struct Deposit {
    uint32_t m[6];  // segment k of the thread index moves up by k (K + 1 segments)
};
Deposit deposit_masks(const int* S, int K) {
    Deposit d;
    int lo = 0;
    for (int k = 0; k <= K; ++k) {
        const int hi = k < K ? S[k] - k : 32;
        uint32_t mask = 0;
        for (int b = lo; b < hi && b < 32; ++b) mask |= 1u << b;
        d.m[k] = mask;
        lo = hi;
    }
    return d;
}
uint32_t deposit_value(const int* S, int K, uint32_t g) {
    uint32_t x = g;
    for (int k = 0; k < K; ++k) {
        const uint32_t lo = x & ((1u << S[k]) - 1);
        x = ((x >> S[k]) << (S[k] + 1)) | lo;
    }
    return x;
}
std::string deposit_expr(const int* S, int K, const char* g) {
    const Deposit d = deposit_masks(S, K);
    std::ostringstream o;
    o << "((" << g << " & " << d.m[0] << "u)";
    for (int k = 1; k <= K; ++k)
        if (d.m[k]) o << " | ((" << g << " & " << d.m[k] << "u) << " << k << ")";
    o << ")";
    return o.str();
}

struct CplxF {
    float re, im;
};

// dense matrix (row-major, dim x dim) of a non-diagonal op, in float
std::vector<CplxF> op_matrix_f(const DevOp& op) {
    const int dim = 1 << op.nq;
    std::vector<CplxF> M(dim * dim, CplxF{0.f, 0.f});
    auto c = [&](int i) { return CplxF{op.cf[i].x, op.cf[i].y}; };
    switch (op.kind) {
        case OPK_DENSE1:
        case OPK_DENSE2:
            for (int k = 0; k < dim * dim; ++k) M[k] = c(k);
            break;
        case OPK_PARITY2:
            M[0 * 4 + 0] = c(0), M[0 * 4 + 3] = c(1), M[3 * 4 + 0] = c(2), M[3 * 4 + 3] = c(3);
            M[1 * 4 + 1] = c(4), M[1 * 4 + 2] = c(5), M[2 * 4 + 1] = c(6), M[2 * 4 + 2] = c(7);
            break;
        case OPK_MONO:
            for (int r = 0; r < dim; ++r) M[r * dim + op.perm[r]] = c(r);
            break;
        default: break;
    }
    return M;
}

// "a*x + ..." real part and imaginary part of sum_c M[c] * x_c
void cmac_terms(const std::vector<std::pair<CplxF, std::string>>& terms, std::string& re, std::string& im) {
    std::ostringstream r, i;
    bool fr = true, fi = true;
    auto add = [](std::ostringstream& o, bool& first, float k, const std::string& v) {
        if (k == 0.f) return;
        if (!first) o << " + ";
        first = false;
        if (k == 1.f) o << v;
        else if (k == -1.f) o << "(-" << v << ")";
        else o << flit(k) << " * " << v;
    };
    for (const auto& t : terms) {
        add(r, fr, t.first.re, t.second + ".x");
        add(r, fr, -t.first.im, t.second + ".y");
        add(i, fi, t.first.re, t.second + ".y");
        add(i, fi, t.first.im, t.second + ".x");
    }
    re = fr ? "0.f" : r.str();
    im = fi ? "0.f" : i.str();
}

struct Gen {
    const Pass& p;
    int G, NT;
    std::ostringstream o;
    explicit Gen(const Pass& pass, int g, int nt) : p(pass), G(g), NT(nt) {}

    std::string v(int i) { return "v" + std::to_string(i); }

    // one stage: S sorted 4 tile bits, rl[q] lane bit of the rotation at stage
    // position q (-1 none), members = indices into p.ops
    // current stage: KB bits, GS register groups of 2^KB amplitudes per thread
    int KB = 4, GS = 2;

    // one stage: S sorted KB tile bits, rl[q] lane bit of the rotation at stage
    // position q (-1 none), members = indices into p.ops
    void stage(const int* S, int k_bits, const int* rl, const std::vector<int>& members) {
        KB = k_bits;
        GS = (G << 4) >> KB;  // the thread's 16 G amplitudes as GS groups of 2^KB
        const int R = 1 << KB;
        const uint32_t gstep = GS > 1 ? deposit_value(S, KB, (uint32_t)NT) : 0u;
        uint32_t off[32];
        for (int r = 0; r < R; ++r) {
            off[r] = 0;
            for (int q = 0; q < KB; ++q)
                if ((r >> q) & 1) off[r] |= 1u << S[q];
        }
        bool rotated = false;
        for (int q = 0; q < KB; ++q) rotated |= rl[q] >= 0;
        o << "    {  // stage S = {";
        for (int q = 0; q < KB; ++q) o << (q ? "," : "") << S[q];
        o << "}\n";
        o << "        const u32 g0 = " << deposit_expr(S, KB, "tid") << ";\n";
        if (rotated) {
            o << "        const u32 ga = g0";
            for (int q = 0; q < KB; ++q)
                if (rl[q] >= 0) o << " ^ (((tid >> " << rl[q] << ") & 1u) << " << S[q] << ")";
            o << ";\n";
        }
        const int nreg = GS * R;
        for (int i = 0; i < nreg; ++i) {
            const uint32_t c = off[i & (R - 1)] | ((i >> KB) ? gstep : 0u);
            if (rotated) o << "        cf " << v(i) << " = tile[ga ^ " << c << "u];\n";
            else o << "        cf " << v(i) << " = tile[g0 + " << c << "u];\n";
        }
        if (rotated) unrotate(rl);
        bool scal = false;
        for (int m : members) scal |= member(m, S, gstep, scal);
        if (scal)
            for (int i = 0; i < nreg; ++i) o << "        " << v(i) << " = cmul(sc, " << v(i) << ");\n";
        if (rotated) unrotate(rl);  // conditional swaps are involutions
        for (int i = 0; i < nreg; ++i) {
            const uint32_t c = off[i & (R - 1)] | ((i >> KB) ? gstep : 0u);
            if (rotated) o << "        tile[ga ^ " << c << "u] = " << v(i) << ";\n";
            else o << "        tile[g0 + " << c << "u] = " << v(i) << ";\n";
        }
        o << "    }\n    __syncthreads();\n";
    }

    // registers loaded at stage bits r ^ rot -> canonical order (and back)
    void unrotate(const int* rl) {
        for (int q = 0; q < KB; ++q) {
            if (rl[q] < 0) continue;
            o << "        { const bool s = (tid >> " << rl[q] << ") & 1u;\n";
            for (int i = 0; i < (GS << KB); ++i) {
                if ((i >> q) & 1) continue;
                const int k = i | (1 << q);
                o << "          { const cf t = s ? " << v(k) << " : " << v(i) << "; " << v(k) << " = s ? " << v(i)
                  << " : " << v(k) << "; " << v(i) << " = t; }\n";
            }
            o << "        }\n";
        }
    }

    // emits one member op; returns true when it multiplied into the stage scalar
    bool member(int m, const int* S, uint32_t gstep, bool have_scal) {
        const DevOp& op = p.ops[m];
        auto spos = [&](int lb) {
            for (int q = 0; q < KB; ++q)
                if (S[q] == lb) return q;
            return -1;
        };
        auto open_scal = [&]() {
            if (!have_scal) o << "        cf sc = cf{1.f, 0.f};\n";
        };
        if (op.kind == OPK_STATESCALE) {
            open_scal();
            o << "        sc = cscale(sc, (float)((const double*)a.ops[" << m << "].aux)[b]);\n";
            return true;
        }
        if (op.kind == OPK_REALTAB) {
            for (int i = 0; i < (GS << KB); ++i) {
                uint32_t c = (i >> KB) ? gstep : 0u;
                for (int q = 0; q < KB; ++q)
                    if ((i >> q) & 1) c |= 1u << S[q];
                o << "        " << v(i) << " = cscale(" << v(i) << ", realtab(a.ops[" << m << "], base, g0 | " << c
                  << "u));\n";
            }
            return false;
        }
        if (op.kind == OPK_DIAG) {
            int pos[4] = {-1, -1, -1, -1};
            bool any_tile_nonstage = false, any_off = false;
            for (int t = 0; t < op.nq; ++t) {
                if (op.lb[t] >= 0) {
                    pos[t] = spos(op.lb[t]);
                    if (pos[t] < 0) any_tile_nonstage = true;
                } else {
                    any_off = true;
                }
            }
            bool any_stage = false;
            for (int t = 0; t < op.nq; ++t) any_stage |= pos[t] >= 0;
            // runtime part of the diagonal index: off-tile bits from the tile base
            std::ostringstream rt;
            rt << "0u";
            for (int t = 0; t < op.nq; ++t)
                if (op.lb[t] < 0) rt << " | ((u32)((base >> " << op.gb[t] << ") & 1ull) << " << t << ")";
            if (!any_stage && !any_tile_nonstage) {
                open_scal();
                o << "        sc = cmul(sc, a.ops[" << m << "].c[" << rt.str() << "]);\n";
                return true;
            }
            if (!any_tile_nonstage && !any_off) {
                // every qubit on a stage bit: literal factor per register
                for (int i = 0; i < (GS << KB); ++i) {
                    int mi = 0;
                    for (int t = 0; t < op.nq; ++t) mi |= ((i >> pos[t]) & 1) << t;
                    const float re = op.cf[mi].x, im = op.cf[mi].y;
                    if (re == 1.f && im == 0.f) continue;
                    std::string r, q;
                    cmac_terms({{CplxF{re, im}, v(i)}}, r, q);
                    o << "        " << v(i) << " = cf{" << r << ", " << q << "};\n";
                }
                return false;
            }
            // mixed: runtime index from non-stage tile bits (per group) and off-tile bits
            for (int j = 0; j < GS; ++j) {
                o << "        { const u32 gj = g0 | " << (j ? gstep : 0u) << "u; const u32 mr = " << rt.str();
                for (int t = 0; t < op.nq; ++t)
                    if (op.lb[t] >= 0 && pos[t] < 0) o << " | (((gj >> " << op.lb[t] << ") & 1u) << " << t << ")";
                o << ";\n";
                for (int r = 0; r < (1 << KB); ++r) {
                    int mi = 0;
                    for (int t = 0; t < op.nq; ++t)
                        if (pos[t] >= 0) mi |= ((r >> pos[t]) & 1) << t;
                    o << "          " << v((j << KB) + r) << " = cmul(a.ops[" << m << "].c[mr | " << mi << "u], "
                      << v((j << KB) + r) << ");\n";
                }
                o << "        }\n";
            }
            return false;
        }
        // matrix op on stage positions
        int pos[3] = {-1, -1, -1};
        for (int t = 0; t < op.nq; ++t) pos[t] = spos(op.lb[t]);
        const int dim = 1 << op.nq;
        const std::vector<CplxF> M = op_matrix_f(op);
        int pmask = 0;
        for (int t = 0; t < op.nq; ++t) pmask |= 1 << pos[t];
        for (int j = 0; j < GS; ++j) {
            for (int e = 0; e < (1 << KB); ++e) {
                if (e & pmask) continue;
                int ix[8];
                for (int c = 0; c < dim; ++c) {
                    int r = e;
                    for (int t = 0; t < op.nq; ++t)
                        if ((c >> t) & 1) r |= 1 << pos[t];
                    ix[c] = (j << KB) + r;
                }
                o << "        {";
                for (int c = 0; c < dim; ++c) o << " const cf x" << c << " = " << v(ix[c]) << ";";
                o << "\n";
                for (int r = 0; r < dim; ++r) {
                    std::vector<std::pair<CplxF, std::string>> terms;
                    for (int c = 0; c < dim; ++c) {
                        const CplxF k = M[r * dim + c];
                        if (k.re != 0.f || k.im != 0.f) terms.push_back({k, "x" + std::to_string(c)});
                    }
                    std::string re, im;
                    cmac_terms(terms, re, im);
                    o << "          " << v(ix[r]) << " = cf{" << re << ", " << im << "};\n";
                }
                o << "        }\n";
            }
        }
        return false;
    }
};

// full source of the kernels for one pass
std::string generate(const Pass& p, bool need_epi, int nbuf, int groups, int minb_add, std::string& err) {
    const int N = p.g.N;
    const TileGeom& g = p.g;
    const int T = g.T;
    // G register groups of 16 amplitudes per thread, NT = 2^(T-4) / G threads
    // register budget: 128 per thread with two groups, 64 with one; minb_add asks
    // for that many more CTAs per SM (a tighter register cap, at most 32 a thread)
    const int G = groups, NT = 1 << (T - 4 - (G - 1));
    const int MINB = std::min(65536 / (NT * (G == 2 ? 128 : 64)) + std::max(0, minb_add), 65536 / (NT * 32));
    Gen gen(p, G, NT);
    std::ostringstream& o = gen.o;
    o << kPrelude;
    o << "static_assert(sizeof(DevOp) == " << sizeof(DevOp) << ", \"DevOp layout\");\n";
    o << "static_assert(sizeof(TileArgs) == " << sizeof(TileArgs) << ", \"TileArgs layout\");\n";
    o << "#define NT " << NT << "\n#define TB " << T << "\n#define LB " << g.L << "\n#define HB " << g.H << "\n";
    o << "#define NSHIFT " << (N - T) << "\n";
    // tile geometry as literals
    o << "__device__ __forceinline__ u64 tile_base(i64 t, i64& b) {\n"
         "    b = t >> NSHIFT;\n"
         "    u64 base = (u64)(t & ((1ll << NSHIFT) - 1)) << LB;\n";
    for (int m = 0; m < g.H; ++m) o << "    base = ins0(base, " << g.hb[m] << ");\n";
    o << "    return base;\n}\n";
    o << "__device__ __forceinline__ u64 seg_off(u64 base, u32 s) {\n    u64 off = base;\n";
    for (int m = 0; m < g.H; ++m) o << "    off |= (u64)((s >> " << m << ") & 1u) << " << g.hb[m] << ";\n";
    o << "    return off;\n}\n";
    o << "__device__ __forceinline__ float realtab(const DevOp& op, u64 base, u32 j) {\n"
         "    u64 gi = base | (j & ((1u << LB) - 1));\n"
         "    const u32 h = j >> LB;\n";
    for (int m = 0; m < g.H; ++m) o << "    gi |= (u64)((h >> " << m << ") & 1u) << " << g.hb[m] << ";\n";
    o << "    const double* tab = (const double*)op.aux;\n"
         "    double f = 1.0;\n"
         "    for (int k = 0; k < (int)op.aux2; ++k) f *= tab[k * 256 + ((gi >> (8 * k)) & 255)];\n"
         "    return (float)f;\n}\n";
    // the body
    // tile loop: one buffer (load, run, store), or two with the next tile's
    // bulk load issued before the current tile's stages run
    o << "__device__ __forceinline__ void issue_load(const TileArgs& a, i64 t, cf* buf, u64* bar) {\n"
         "    i64 b;\n"
         "    const u64 base = tile_base(t, b);\n"
         "    const cf* gs = (const cf*)a.psi + b * a.state_len;\n"
         "    if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, 8u << TB);\n"
         "    for (u32 s = threadIdx.x; s < (1u << HB); s += NT)\n"
         "        bulk_g2s(buf + ((u64)s << LB), gs + seg_off(base, s), 8u << LB, bar);\n"
         "}\n";
    o << "template <bool EPI>\n__device__ __forceinline__ void body(const TileArgs& a) {\n"
         "    extern __shared__ __align__(128) unsigned char smem_raw[];\n"
         "    cf* const buf0 = (cf*)smem_raw;\n"
         "    __shared__ __align__(8) u64 bars[2];\n"
         "    __shared__ double red[NT / 32][16];\n"
         "    const u32 tid = threadIdx.x;\n"
         "    const u32 seg_bytes = 8u << LB;\n"
         "    if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); fence_mbar_init(); }\n"
         "    __syncthreads();\n"
         "    u32 phases = 0;\n";
    if (nbuf == 2)
        o << "    cf* const buf1 = buf0 + (1u << TB);\n"
             "    if ((i64)blockIdx.x < a.ntiles) issue_load(a, blockIdx.x, buf0, &bars[0]);\n";
    o << "    int k = 0;\n"
         "    for (i64 t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++k) {\n"
         "    i64 b;\n"
         "    const u64 base = tile_base(t, b);\n"
         "    cf* gs = (cf*)a.psi + b * a.state_len;\n";
    if (nbuf == 2)
        o << "    const int cur = k & 1;\n"
             "    cf* const tile = cur ? buf1 : buf0;\n"
             "    const bool have_next = t + gridDim.x < a.ntiles;\n"
             "    if (have_next) issue_load(a, t + gridDim.x, cur ? buf0 : buf1, &bars[cur ^ 1]);\n"
             "    const bool ok = mbar_wait_bounded(&bars[cur], (phases >> cur) & 1, a.err);\n"
             "    if (!__syncthreads_and(ok)) {\n"
             "        mbar_wait_bounded(&bars[cur], (phases >> cur) & 1, nullptr);\n"
             "        if (have_next) mbar_wait_bounded(&bars[cur ^ 1], (phases >> (cur ^ 1)) & 1, nullptr);\n"
             "        return;\n"
             "    }\n"
             "    phases ^= 1u << cur;\n";
    else
        o << "    const int cur = 0;\n"
             "    cf* const tile = buf0;\n"
             "    issue_load(a, t, tile, &bars[0]);\n"
             "    const bool ok = mbar_wait_bounded(&bars[0], phases & 1, a.err);\n"
             "    if (!__syncthreads_and(ok)) { mbar_wait_bounded(&bars[0], phases & 1, nullptr); return; }\n"
             "    phases ^= 1;\n"
             "    (void)cur; (void)k;\n";
    // stages
    const int LBk = 4;  // complex64 bank boundary
    size_t o_i = 0;
    while (o_i < p.ops.size()) {
        const DevOp& h = p.ops[o_i];
        if (h.kind != OPK_STAGE) {
            err = "jit: pass program is not stage-scheduled";
            return "";
        }
        std::vector<int> members;
        int S[5], rl[5] = {-1, -1, -1, -1, -1}, kb = 4;
        if (h.nq == 0) {
            // one wide op: its 3 bits + one pad bit (bank-neutral first)
            const DevOp& op = p.ops[o_i + 1];
            std::vector<int> s;
            for (int t = 0; t < op.nq; ++t) s.push_back(op.lb[t]);
            for (int bb = LBk; (int)s.size() < 4 && bb < T; ++bb)
                if (std::find(s.begin(), s.end(), bb) == s.end()) s.push_back(bb);
            for (int bb = 0; (int)s.size() < 4 && bb < T; ++bb)
                if (std::find(s.begin(), s.end(), bb) == s.end()) s.push_back(bb);
            std::sort(s.begin(), s.end());
            int cfree = 0;
            for (int bb = 0; bb < LBk; ++bb)
                if (std::find(s.begin(), s.end(), bb) == s.end()) ++cfree;
            int a = 0;
            for (int q = 0; q < 4; ++q) {
                S[q] = s[q];
                rl[q] = s[q] < LBk ? cfree + a++ : -1;
            }
            members.push_back((int)o_i + 1);
            o_i += 2;
        } else {
            for (int q = 0; q < 4; ++q) S[q] = h.perm[q], rl[q] = h.perm[4 + q];
            for (int k = 1; k <= (int)h.aux2; ++k) members.push_back((int)(o_i + k));
            o_i += 1 + (size_t)h.aux2;
        }
        gen.stage(S, kb, rl, members);
    }
    o << "    if (EPI) {\n"
         "        constexpr int nb = NT == 128 ? 7 : NT == 256 ? 8 : 9;\n"
         "        double acc[16];\n"
         "#pragma unroll\n"
         "        for (int q = 0; q < 16; ++q) acc[q] = 0.0;\n"
         "        for (u32 j = tid; j < (1u << TB); j += NT) {\n"
         "            const double pr = cabs2d(tile[j]);\n"
         "            acc[0] += pr;\n"
         "#pragma unroll\n"
         "            for (int l = nb; l < 15; ++l) if (l < TB && ((j >> l) & 1)) acc[1 + l] += pr;\n"
         "        }\n"
         "#pragma unroll\n"
         "        for (int l = 0; l < nb; ++l) acc[1 + l] = ((tid >> l) & 1) ? acc[0] : 0.0;\n"
         "#pragma unroll\n"
         "        for (int q = 0; q < 16; ++q) {\n"
         "            double x = acc[q];\n"
         "            for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);\n"
         "            if ((tid & 31) == 0) red[tid >> 5][q] = x;\n"
         "        }\n"
         "        __syncthreads();\n"
         "        if (tid < 16) { double s = 0; for (int w = 0; w < NT / 32; ++w) s += red[w][tid]; red[0][tid] = s; }\n"
         "        __syncthreads();\n"
         "        if (tid == 0) {\n"
         "            double* out = a.ep.partials + (u64)t * (1 + a.ep.npop);\n"
         "            out[0] = red[0][0];\n"
         "            for (int q = 0; q < a.ep.npop; ++q) {\n"
         "                const int qq = a.ep.popq[q];\n"
         "                int l = -1;\n"
         "                if (qq < LB) l = qq;\n";
    for (int m = 0; m < g.H; ++m) o << "                if (qq == " << g.hb[m] << ") l = LB + " << m << ";\n";
    o << "                out[1 + q] = (l >= 0) ? red[0][1 + l] : (((base >> qq) & 1) ? red[0][0] : 0.0);\n"
         "            }\n"
         "        }\n"
         "        __syncthreads();\n"
         "    }\n"
         "    fence_proxy_async_smem();\n"
         "    __syncthreads();\n"
         "    for (u32 s = tid; s < (1u << HB); s += NT) bulk_s2g(gs + seg_off(base, s), tile + ((u64)s << LB), seg_bytes);\n"
         "    bulk_commit();\n"
         "    bulk_wait_read0();\n"
         "    __syncthreads();\n"
         "    }\n"
         "    bulk_wait0();\n"
         "}\n";
    o << "extern \"C\" __global__ void __launch_bounds__(NT, " << MINB
      << ") smoq_pass_e0(const TileArgs a) { body<false>(a); }\n";
    if (need_epi)
        o << "extern \"C\" __global__ void __launch_bounds__(NT, " << MINB
          << ") smoq_pass_e1(const TileArgs a) { body<true>(a); }\n";
    return o.str();
}

std::mutex g_mu;
std::map<std::string, std::unique_ptr<JitKernel>> g_cache;

// FNV-1a of a kernel source: the key of a pass program in the tuning cache
uint64_t fnv1a(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
    return h;
}

}  // namespace

namespace {
// NVRTC: source -> sm_100a cubin (no GPU needed)
bool compile_cubin(const std::string& src, std::vector<char>& cubin, std::string& err, std::string* info = nullptr) {
    Nvrtc& nv = nvrtc();
    if (!nv.ok) {
        err = nv.why;
        return false;
    }
    nvrtcProgram prog = nullptr;
    if (nv.create(&prog, src.c_str(), "smoq_pass.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        err = "nvrtcCreateProgram failed";
        return false;
    }
    const char* opts[] = {"-arch=sm_100a", "-std=c++17", "-default-device", "-diag-suppress=177",
                          "--ptxas-options=-v"};
    const nvrtcResult rc = nv.compile(prog, info ? 5 : 4, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t n = 0;
        nv.logsize(prog, &n);
        std::string log(n, '\0');
        if (n) nv.log(prog, &log[0]);
        err = "NVRTC compile failed: " + log.substr(0, 2000);
        nv.destroy(&prog);
        return false;
    }
    if (info) {
        size_t n = 0;
        nv.logsize(prog, &n);
        info->assign(n, '\0');
        if (n) nv.log(prog, &(*info)[0]);
        while (!info->empty() && info->back() == '\0') info->pop_back();
    }
    size_t n = 0;
    nv.cubinsize(prog, &n);
    cubin.assign(n, 0);
    nv.cubin(prog, cubin.data());
    nv.destroy(&prog);
    return true;
}
}  // namespace

// Generate and compile a staged complex64 pass without loading it (host only);
// `info` (optional) receives the compiler's resource report.
bool jit_check_pass(const Pass& p, int nbuf, int groups, std::string& err, size_t* cubin_bytes,
                    std::string* info) {
    if (!p.staged || (p.g.T != 12 && p.g.T != 13)) {
        err = "jit: only stage-scheduled passes of tile width 12-13";
        return false;
    }
    const std::string src = generate(p, p.epilogue, nbuf, groups, 0, err);
    if (src.empty()) return false;
    std::vector<char> cubin;
    if (!compile_cubin(src, cubin, err, info)) return false;
    if (cubin_bytes) *cubin_bytes = cubin.size();
    return true;
}

// Compile (or fetch) the kernel of a stage-scheduled complex64 pass and load
// it into the current device.  Returns nullptr and fills `err` on failure.
const JitKernel* jit_pass_kernel(const Pass& p, int nbuf, int groups, std::string& err, int minb_add) {
    if (!p.staged || (p.g.T != 12 && p.g.T != 13)) {
        err = "jit: only stage-scheduled passes of tile width 12-13";
        return nullptr;
    }
    std::string src = generate(p, p.epilogue, nbuf, groups, minb_add, err);
    if (src.empty()) return nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(src);
        if (it != g_cache.end()) return it->second.get();
    }
    // compile outside the lock: several host threads may compile different passes at once
    std::vector<char> cubin;
    if (!compile_cubin(src, cubin, err)) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(src);
    if (it != g_cache.end()) return it->second.get();
    std::unique_ptr<JitKernel> k(new JitKernel());
    cudaLibrary_t lib = nullptr;
    cudaError_t e = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) {
        err = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e);
        return nullptr;
    }
    k->threads = 1 << (p.g.T - 4 - (groups - 1));
    k->smem = (size_t)(nbuf == 2 ? 16 : 8) << p.g.T;
    const char* names[2] = {"smoq_pass_e0", "smoq_pass_e1"};
    for (int v = 0; v < (p.epilogue ? 2 : 1); ++v) {
        cudaKernel_t kern = nullptr;
        if ((e = cudaLibraryGetKernel(&kern, lib, names[v])) != cudaSuccess) {
            err = std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(e);
            return nullptr;
        }
        const void* fn = reinterpret_cast<const void*>(kern);
        if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k->smem)) !=
            cudaSuccess) {
            err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return nullptr;
        }
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, k->threads, k->smem)) != cudaSuccess) {
            err = std::string("occupancy query: ") + cudaGetErrorString(e);
            return nullptr;
        }
        k->fn[v] = fn;
        k->per_sm[v] = per_sm < 1 ? 1 : per_sm;
    }
    const JitKernel* out = k.get();
    g_cache.emplace(std::move(src), std::move(k));
    return out;
}

bool jit_available() { return nvrtc().ok; }

uint64_t jit_pass_key(const Pass& p, int nbuf) {
    std::string err;
    const std::string src = generate(p, p.epilogue, nbuf, 2, 0, err);
    return src.empty() ? 0 : fnv1a(src);
}

cudaError_t launch_jit(smoq_ctx* ctx, const TileArgs& a, const JitKernel* k, bool epi) {
    const void* fn = k->fn[epi ? 1 : 0];
    if (!fn) return cudaErrorInvalidValue;
    int64_t grid = (int64_t)ctx->num_sms * k->per_sm[epi ? 1 : 0];
    if (grid > a.ntiles) grid = a.ntiles;
    TileArgs args = a;
    void* params[] = {&args};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)k->threads), params, k->smem, ctx->stream);
}

}  // namespace smoq

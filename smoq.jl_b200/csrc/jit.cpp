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
#include <atomic>
#include <set>
#include <thread>
#include <cmath>
#include <complex>
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

// dense matrix (row-major, dim x dim) of a non-diagonal op, in float; idx[k] = the
// op's coefficient slot of entry k (-1: a zero of the op kind's structure)
std::vector<CplxF> op_matrix_f(const DevOp& op, std::vector<int>* idx = nullptr) {
    const int dim = 1 << op.nq;
    std::vector<CplxF> M(dim * dim, CplxF{0.f, 0.f});
    std::vector<int> I(dim * dim, -1);
    auto set = [&](int k, int i) { M[k] = CplxF{op.cf[i].x, op.cf[i].y}, I[k] = i; };
    switch (op.kind) {
        case OPK_DENSE1:
        case OPK_DENSE2:
            for (int k = 0; k < dim * dim; ++k) set(k, k);
            break;
        case OPK_PARITY2:
            set(0 * 4 + 0, 0), set(0 * 4 + 3, 1), set(3 * 4 + 0, 2), set(3 * 4 + 3, 3);
            set(1 * 4 + 1, 4), set(1 * 4 + 2, 5), set(2 * 4 + 1, 6), set(2 * 4 + 2, 7);
            break;
        case OPK_MONO:
            for (int r = 0; r < dim; ++r) set(r * dim + op.perm[r], r);
            break;
        default: break;
    }
    if (idx) idx->swap(I);
    return M;
}

// 0, +-1 and +-i: coefficients a compiled kernel keeps as literals even when it
// reads the others at run time (the entries a gate's structure fixes: CZ, CNOT, X)
bool trivial_coef(CplxF k) {
    const bool re01 = k.re == 0.f || k.re == 1.f || k.re == -1.f;
    const bool im01 = k.im == 0.f || k.im == 1.f || k.im == -1.f;
    return re01 && im01 && (k.re == 0.f || k.im == 0.f);
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

// ------------------------------------------------------ run-time coefficients
// With p.rtc, the op coefficients other than 0, +-1, +-i travel as a kernel
// parameter block (one complex64 per (op, coefficient slot) pair, in this order);
// the compiled code reads them as constant-bank operands.  The kernel source then
// depends on the circuit's gates and qubits, not on its angles, and one compiled
// kernel serves every parameter set of a variational circuit.
std::vector<std::pair<int, int>> rtc_list(const Pass& p) {
    std::vector<std::pair<int, int>> out;
    for (size_t m = 0; m < p.ops.size(); ++m) {
        const DevOp& op = p.ops[m];
        std::set<int> need;
        if (op.kind == OPK_DIAG) {
            bool on_tile = true;
            for (int t = 0; t < op.nq; ++t) on_tile &= op.lb[t] >= 0;
            if (!on_tile) continue;  // the mixed and off-tile forms index a.ops[m].c at run time
            for (int k = 0; k < (1 << op.nq); ++k)
                if (!trivial_coef(CplxF{op.cf[k].x, op.cf[k].y})) need.insert(k);
        } else if (op.kind == OPK_DENSE1 || op.kind == OPK_DENSE2 || op.kind == OPK_PARITY2 || op.kind == OPK_MONO) {
            std::vector<int> I;
            const std::vector<CplxF> M = op_matrix_f(op, &I);
            for (size_t k = 0; k < M.size(); ++k)
                if (I[k] >= 0 && !trivial_coef(M[k])) need.insert(I[k]);
        }
        for (int i : need) out.push_back({(int)m, i});
    }
    return out;
}

struct Gen {
    const Pass& p;
    int G, NT;
    std::ostringstream o;
    std::map<std::pair<int, int>, int> kslot;  // run-time coefficient (op, slot) -> parameter index
    explicit Gen(const Pass& pass, int g, int nt) : p(pass), G(g), NT(nt) {
        if (p.rtc) {
            const auto l = rtc_list(p);
            for (size_t k = 0; k < l.size(); ++k) kslot[l[k]] = (int)k;
        }
    }

    // register names: v<i> for the single-state kernels and phi of the adjoint
    // kernels, w<i> for lambda; scn: the stage scalar of that register set
    std::string vp = "v", scn = "sc";
    std::string v(int i) { return vp + std::to_string(i); }

    // one stage: S sorted 4 tile bits, rl[q] lane bit of the rotation at stage
    // position q (-1 none), members = indices into p.ops
    // current stage: KB bits, GS register groups of 2^KB amplitudes per thread
    int KB = 4, GS = 2;

    // What the dry run of a stage's members learns: per stage pattern the position of
    // the last member that mixes it (-2: a member that flushes) and the phases pending
    // at the stage's end; the emitting run marks the patterns whose final phase went into
    // a member row (taken), which the end of the stage then skips.
    struct Absorb {
        bool dry = true;
        std::vector<int> last;
        std::vector<std::complex<double>> fin;
        std::vector<bool> taken;
    };

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
        // Literal diagonals whose qubits are stage bits fold into one pending phase per
        // stage pattern (computed here in FP64); it commutes with every diagonal member
        // and with matrix members on other stage bits, and is applied before a matrix
        // member on its bits and at the stage's end.  (Run-time coefficients: no folding.)
        // A matrix member leaves alone the stage patterns whose local index k has row and
        // column e_k (an identity row: the even rows of a split XXZ rotation): only the
        // other patterns take their pending phase before it.
        const std::complex<double> one(1.0, 0.0);
        std::vector<std::complex<double>> pend(R, one);
        auto flush_where = [&](const std::vector<bool>& need) {
            for (int i = 0; i < nreg; ++i) {
                const int r = i & (R - 1);
                if (!need[r] || pend[r] == one) continue;
                const std::complex<double> z = pend[r];
                std::string re, im;
                cmac_terms({{CplxF{(float)z.real(), (float)z.imag()}, v(i)}}, re, im);
                o << "        " << v(i) << " = cf{" << re << ", " << im << "};\n";
            }
            for (int r = 0; r < R; ++r)
                if (need[r]) pend[r] = one;
        };
        auto stage_pos = [&](int lb) {
            for (int q = 0; q < KB; ++q)
                if (S[q] == lb) return q;
            return -1;
        };
        // The phase a pattern still has pending at the stage's end goes, where that costs
        // less, into the row of the last member that mixes the pattern instead of a flush
        // at the end: a dry run of the members (its code discarded) finds those members
        // and the final phases; the second run emits.
        Absorb ab;
        ab.last.assign(R, -1);
        ab.taken.assign(R, false);
        std::ostringstream kept = std::move(o);
        for (int run = 0; run < 2; ++run) {
            ab.dry = run == 0;
            if (ab.dry) o = std::ostringstream();
            else o = std::move(kept);
            std::fill(pend.begin(), pend.end(), one);
            scal = false;
            for (size_t at = 0; at < members.size(); ++at) {
                const int m = members[at];
                const DevOp& op = p.ops[m];
                int pm = 0;
                bool on_stage = op.nq >= 1;
                for (int t = 0; t < op.nq; ++t) {
                    const int q = op.lb[t] >= 0 ? stage_pos(op.lb[t]) : -1;
                    if (q < 0) on_stage = false;
                    else pm |= 1 << q;
                }
                if (!p.rtc && op.kind == OPK_DIAG && on_stage) {
                    for (int r = 0; r < R; ++r) {
                        int mi = 0;
                        for (int t = 0; t < op.nq; ++t) mi |= ((r >> stage_pos(op.lb[t])) & 1) << t;
                        pend[r] *= std::complex<double>(op.cd[mi].x, op.cd[mi].y);
                    }
                    continue;
                }
                const bool diagonal =
                    op.kind == OPK_DIAG || op.kind == OPK_STATESCALE || op.kind == OPK_REALTAB;
                if (!diagonal && !p.rtc && on_stage) {
                    member_through(m, (int)at, S, gstep, pend, ab);
                    continue;
                }
                // any other matrix member takes every pending phase first (with run-time
                // coefficients nothing is pending), and nothing it mixes is absorbed
                if (!diagonal && pm) {
                    if (ab.dry) std::fill(ab.last.begin(), ab.last.end(), -2);
                    flush_where(std::vector<bool>(R, true));
                }
                scal |= member(m, S, gstep, scal);
            }
            if (ab.dry) ab.fin = pend;
        }
        {
            std::vector<bool> rest(R);
            for (int r = 0; r < R; ++r) rest[r] = !ab.taken[r];
            flush_where(rest);
        }
        if (scal)
            for (int i = 0; i < nreg; ++i) o << "        " << v(i) << " = cmul(" << scn << ", " << v(i) << ");\n";
        if (rotated) unrotate(rl);  // conditional swaps are involutions
        for (int i = 0; i < nreg; ++i) {
            const uint32_t c = off[i & (R - 1)] | ((i >> KB) ? gstep : 0u);
            if (rotated) o << "        tile[ga ^ " << c << "u] = " << v(i) << ";\n";
            else o << "        tile[g0 + " << c << "u] = " << v(i) << ";\n";
        }
        o << "    }\n    __syncthreads();\n";
    }

    // FP32 multiplies one coefficient costs per output amplitude: none for 0, +-1, +-i
    // (a copy or a swap of parts), 2 for a real or imaginary one, 4 for a general one
    static int coef_cost(CplxF k) {
        if (trivial_coef(k)) return 0;
        return (k.re == 0.f || k.im == 0.f) ? 2 : 4;
    }

    // A literal matrix member on stage bits under the stage's pending phases P (one per
    // stage pattern).  For each pattern of the other stage bits (the "rest") it takes the
    // cheaper of two exact forms: apply the pending phases of the member's non-identity
    // rows first (a flush), then M; or leave every phase pending and apply P^-1 M P, the
    // member moved through the phases (entry (r, c) times p_c / p_r: M's diagonal stays as
    // it is, so a split rotation's real cosines stay real, and the flush disappears).
    // Where this member is the last to mix a pattern, the pattern's phase at the stage's
    // end may go into the member's row for it (row times that phase) instead of a flush
    // at the end, when the row costs less than the row plus the flush.  Coefficients are
    // formed in FP64 and rounded once.
    void member_through(int m, int at, const int* S, uint32_t gstep, std::vector<std::complex<double>>& pend,
                        Absorb& ab) {
        using cd = std::complex<double>;
        const DevOp& op = p.ops[m];
        const int dim = 1 << op.nq, R = 1 << KB;
        int pos[3] = {-1, -1, -1}, pmask = 0;
        for (int t = 0; t < op.nq; ++t) {
            for (int q = 0; q < KB; ++q)
                if (S[q] == op.lb[t]) pos[t] = q;
            pmask |= 1 << pos[t];
        }
        const std::vector<CplxF> M = op_matrix_f(op);
        const cd one(1.0, 0.0);
        auto rnd = [](cd z) { return CplxF{(float)z.real(), (float)z.imag()}; };
        std::vector<bool> iso(dim, false);  // rows and columns e_k: the member leaves pattern k alone
        for (int k = 0; k < dim; ++k) {
            bool e = M[k * dim + k].re == 1.f && M[k * dim + k].im == 0.f;
            for (int j = 0; j < dim && e; ++j)
                if (j != k) {
                    const CplxF a = M[k * dim + j], b = M[j * dim + k];
                    e = a.re == 0.f && a.im == 0.f && b.re == 0.f && b.im == 0.f;
                }
            iso[k] = e;
        }
        for (int e = 0; e < R; ++e) {
            if (e & pmask) continue;
            int pat[8];
            for (int c = 0; c < dim; ++c) {
                pat[c] = e;
                for (int t = 0; t < op.nq; ++t)
                    if ((c >> t) & 1) pat[c] |= 1 << pos[t];
            }
            // the moved-through member, its cost, and the flush form's cost
            std::vector<cd> Mt(dim * dim);
            int cost_through = 0, cost_flush = 0;
            // a zero pending factor (a projector) has no P^-1; near-zero ones take the
            // flush form too (no FP32 coefficients scaled by their inverse)
            bool invertible = true;
            for (int c = 0; c < dim; ++c) invertible &= std::abs(pend[pat[c]]) > 1e-6;
            for (int r = 0; r < dim && invertible; ++r)
                for (int c = 0; c < dim; ++c) {
                    const CplxF k = M[r * dim + c];
                    cost_flush += coef_cost(k);
                    cd ratio = pend[pat[c]] / pend[pat[r]];
                    if (std::abs(ratio - one) < 1e-15) ratio = one;
                    Mt[r * dim + c] = cd(k.re, k.im) * ratio;
                    cost_through += coef_cost(rnd(Mt[r * dim + c]));
                }
            for (int c = 0; c < dim; ++c)
                if (!iso[c] && pend[pat[c]] != one) cost_flush += coef_cost(rnd(pend[pat[c]]));
            if (!invertible) cost_through = cost_flush + 1;  // the flush form
            const bool through = cost_through <= cost_flush;
            // the rows to emit (FP64), with the final phases of the patterns this member
            // mixes last folded in where that is cheaper
            std::vector<cd> A(dim * dim);
            for (int k = 0; k < dim * dim; ++k) A[k] = through ? Mt[k] : cd(M[k].re, M[k].im);
            for (int r = 0; r < dim; ++r) {
                if (iso[r]) continue;
                if (ab.dry) {
                    ab.last[pat[r]] = at;
                    continue;
                }
                const cd f = ab.fin[pat[r]];
                if (ab.last[pat[r]] != at || f == one) continue;
                int cost_row = coef_cost(rnd(f)), cost_abs = 0;
                for (int c = 0; c < dim; ++c) {
                    cost_row += coef_cost(rnd(A[r * dim + c]));
                    cost_abs += coef_cost(rnd(A[r * dim + c] * f));
                }
                if (cost_abs > cost_row) continue;
                for (int c = 0; c < dim; ++c) A[r * dim + c] *= f;
                ab.taken[pat[r]] = true;
            }
            for (int j = 0; j < GS; ++j) {
                int ix[8];
                for (int c = 0; c < dim; ++c) ix[c] = (j << KB) + pat[c];
                if (!through)
                    for (int c = 0; c < dim; ++c) {
                        const cd z = pend[pat[c]];
                        if (iso[c] || z == one) continue;
                        std::string re, im;
                        cmac_terms({{rnd(z), v(ix[c])}}, re, im);
                        o << "        " << v(ix[c]) << " = cf{" << re << ", " << im << "};\n";
                    }
                o << "        {";
                for (int c = 0; c < dim; ++c) o << " const cf x" << c << " = " << v(ix[c]) << ";";
                o << "\n";
                for (int r = 0; r < dim; ++r) {
                    std::vector<std::pair<CplxF, std::string>> terms;
                    for (int c = 0; c < dim; ++c) {
                        const CplxF k = rnd(A[r * dim + c]);
                        if (k.re != 0.f || k.im != 0.f) terms.push_back({k, "x" + std::to_string(c)});
                    }
                    std::string re, im;
                    cmac_terms(terms, re, im);
                    o << "          " << v(ix[r]) << " = cf{" << re << ", " << im << "};\n";
                }
                o << "        }\n";
            }
            if (!through)
                for (int c = 0; c < dim; ++c)
                    if (!iso[c]) pend[pat[c]] = one;
        }
    }

    // registers loaded at stage bits r ^ rot -> canonical order (and back)
    void unrotate(const int* rl) {
        for (int q = 0; q < KB; ++q) {
            if (rl[q] < 0) continue;
            o << "        { const bool s = (tid >> " << rl[q] << ") & 1u;\n";
            for (int i = 0; i < (GS << KB); ++i) {
                if ((i >> q) & 1) continue;
                const int k = i | (1 << q);
                o << "          { const auto t = s ? " << v(k) << " : " << v(i) << "; " << v(k) << " = s ? " << v(i)
                  << " : " << v(k) << "; " << v(i) << " = t; }\n";
            }
            o << "        }\n";
        }
    }

    // ------------------------------------------------------------ adjoint (dual)
    // One stage of the compiled adjoint kernel: the same 16-amplitude groups of
    // phi (tile, registers v<i>) and lambda (tlam, w<i>).  U^dag members act on
    // both register sets (the same literal code twice); an OPK_INNER member adds
    // Im<lambda|G|phi> over the thread's registers, at its place in the op order,
    // to its warp's row of the partials.
    void stage_dual(const int* S, const int* rl, const std::vector<int>& members) {
        KB = 4;
        GS = (G << 4) >> KB;
        const int R = 1 << KB;
        const uint32_t gstep = GS > 1 ? deposit_value(S, KB, (uint32_t)NT) : 0u;
        uint32_t off[16];
        for (int r = 0; r < R; ++r) {
            off[r] = 0;
            for (int q = 0; q < KB; ++q)
                if ((r >> q) & 1) off[r] |= 1u << S[q];
        }
        bool rotated = false;
        for (int q = 0; q < KB; ++q) rotated |= rl[q] >= 0;
        o << "    {  // stage S = {" << S[0] << "," << S[1] << "," << S[2] << "," << S[3] << "}, phi and lambda\n";
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
            const std::string at = std::string(rotated ? "[ga ^ " : "[g0 + ") + std::to_string(c) + "u]";
            o << "        float2 P" << i << ", Q" << i << ";\n        { const cf f = tile" << at << ", l = tlam" << at
              << "; P" << i << " = make_float2(f.x, l.x); Q" << i << " = make_float2(f.y, l.y); }\n";
        }
        if (rotated)
            for (const char* pre : {"P", "Q"}) {
                vp = pre;
                unrotate(rl);
            }
        bool scal = false;
        o << "        cf sc = cf{1.f, 0.f};\n";
        std::vector<int> cols;  // the stage's measurements, reduced together at its end
        bool writes = false;
        size_t reduced = 0;  // measurements [0, reduced) are summed already
        for (int m : members) {
            if (p.ops[m].kind == OPK_INNER) {
                inner(m, S, (int)cols.size());
                cols.push_back(p.ops[m].perm[0]);
                // a group of kMeasGroup is reduced at once: at most that many FP32
                // accumulators stay live beside the two register sets
                if (cols.size() - reduced == (size_t)kMeasGroup) {
                    reduce_measurements(cols, reduced, cols.size());
                    reduced = cols.size();
                }
                continue;
            }
            writes = true;
            scal |= member_packed(m, S);
        }
        if (reduced < cols.size()) reduce_measurements(cols, reduced, cols.size());
        // after a stage that only read (no barrier at its end), other threads may
        // still be reading what this stage's stores overwrite
        if (writes && pending_reads) o << "        __syncthreads();\n";
        if (writes) {
            if (scal)
                for (int i = 0; i < nreg; ++i)
                    emit_pmul("P" + std::to_string(i), "Q" + std::to_string(i), "sc.x", false, "sc.y", "        ");
            if (rotated)
                for (const char* pre : {"P", "Q"}) {
                    vp = pre;
                    unrotate(rl);
                }
            for (int i = 0; i < nreg; ++i) {
                const uint32_t c = off[i & (R - 1)] | ((i >> KB) ? gstep : 0u);
                const std::string at = std::string(rotated ? "[ga ^ " : "[g0 + ") + std::to_string(c) + "u]";
                o << "        tile" << at << " = cf{P" << i << ".x, Q" << i << ".x}; tlam" << at << " = cf{P" << i
                  << ".y, Q" << i << ".y};\n";
            }
        }
        vp = "v";
        scn = "sc";
        // a stage that only measured leaves the tiles as they were: the next stage
        // may read them without a barrier (a writing stage waits before its stores)
        o << (writes ? "    }\n    __syncthreads();\n" : "    }\n");
        pending_reads = !writes;
    }
    bool pending_reads = false;
    static constexpr int kMeasGroup = 4;

    // ------------------------------------------------- packed adjoint registers
    // The adjoint stage keeps both states in float2 pairs: P<i> = (phi_i.x, lambda_i.x),
    // Q<i> = (phi_i.y, lambda_i.y).  A U^dag op multiplies both states by the same
    // coefficients, so each real multiply-add is one packed __ffma2_rn for the two.
    static std::string splat(const std::string& e) { return "make_float2(" + e + ", " + e + ")"; }
    struct PTerm {
        std::string c;  // scalar coefficient expression
        bool one;       // the coefficient is exactly 1 (no multiply)
        std::string x;  // float2 operand
    };
    static std::string chain(const std::vector<PTerm>& t) {
        if (t.empty()) return "make_float2(0.f, 0.f)";
        std::string acc = t[0].one ? t[0].x : "__fmul2_rn(" + splat(t[0].c) + ", " + t[0].x + ")";
        for (size_t i = 1; i < t.size(); ++i) acc = "__ffma2_rn(" + splat(t[i].c) + ", " + t[i].x + ", " + acc + ")";
        return acc;
    }
    // (P, Q) of a register times the complex k = (re, im) given as expressions
    // (empty: a zero part; re_one: re is exactly 1)
    void emit_pmul(const std::string& P, const std::string& Q, const std::string& re, bool re_one,
                   const std::string& im, const std::string& ind) {
        std::vector<PTerm> tp, tq;
        if (!re.empty()) tp.push_back({re, re_one, "pa"}), tq.push_back({re, re_one, "qa"});
        if (!im.empty()) tp.push_back({"-(" + im + ")", false, "qa"}), tq.push_back({im, false, "pa"});
        o << ind << "{ const float2 pa = " << P << ", qa = " << Q << "; " << P << " = " << chain(tp) << "; " << Q
          << " = " << chain(tq) << "; }\n";
    }
    // coefficient parts of entry k (op m, coefficient slot idx): literals, or the
    // parameter block under run-time coefficients
    void coef_parts(int m, int idx, CplxF k, std::string& re, bool& re_one, std::string& im) {
        re_one = false;
        if (p.rtc && !trivial_coef(k)) {
            const std::string kn = kname(m, idx);
            re = k.re == 0.f ? "" : kn + ".x";
            im = k.im == 0.f ? "" : kn + ".y";
            return;
        }
        re = k.re == 0.f ? "" : flit(k.re);
        im = k.im == 0.f ? "" : flit(k.im);
        re_one = k.re == 1.f;
    }
    // one U^dag member of the adjoint stage on the packed registers; returns true when
    // it multiplied into the stage scalar sc (a phase on off-tile bits, both states)
    bool member_packed(int m, const int* S) {
        const DevOp& op = p.ops[m];
        const int R = 1 << KB;
        auto spos = [&](int lb) {
            for (int q = 0; q < KB; ++q)
                if (S[q] == lb) return q;
            return -1;
        };
        auto P = [](int i) { return "P" + std::to_string(i); };
        auto Q = [](int i) { return "Q" + std::to_string(i); };
        if (op.kind == OPK_DIAG) {
            int pos[4] = {-1, -1, -1, -1};
            bool any_tile_nonstage = false, any_off = false, any_stage = false;
            for (int t = 0; t < op.nq; ++t) {
                if (op.lb[t] >= 0) {
                    pos[t] = spos(op.lb[t]);
                    if (pos[t] < 0) any_tile_nonstage = true;
                    else any_stage = true;
                } else {
                    any_off = true;
                }
            }
            std::ostringstream rt;
            rt << "0u";
            for (int t = 0; t < op.nq; ++t)
                if (op.lb[t] < 0) rt << " | ((u32)((base >> " << op.gb[t] << ") & 1ull) << " << t << ")";
            if (!any_stage && !any_tile_nonstage) {
                o << "        sc = cmul(sc, a.ops[" << m << "].c[" << rt.str() << "]);\n";
                return true;
            }
            if (!any_tile_nonstage && !any_off) {
                for (int i = 0; i < (GS << KB); ++i) {
                    int mi = 0;
                    for (int t = 0; t < op.nq; ++t) mi |= ((i >> pos[t]) & 1) << t;
                    const CplxF k{op.cf[mi].x, op.cf[mi].y};
                    if (k.re == 1.f && k.im == 0.f) continue;
                    std::string re, im;
                    bool one;
                    coef_parts(m, mi, k, re, one, im);
                    emit_pmul(P(i), Q(i), re, one, im, "        ");
                }
                return false;
            }
            for (int j = 0; j < GS; ++j) {
                o << "        { const u32 gj = g0 | " << (j ? deposit_value(S, KB, (uint32_t)NT) : 0u)
                  << "u; (void)gj; const u32 mr = " << rt.str();
                for (int t = 0; t < op.nq; ++t)
                    if (op.lb[t] >= 0 && pos[t] < 0) o << " | (((gj >> " << op.lb[t] << ") & 1u) << " << t << ")";
                o << ";\n";
                for (int r = 0; r < R; ++r) {
                    int mi = 0;
                    for (int t = 0; t < op.nq; ++t)
                        if (pos[t] >= 0) mi |= ((r >> pos[t]) & 1) << t;
                    o << "          { const cf z = a.ops[" << m << "].c[mr | " << mi << "u];\n";
                    emit_pmul(P((j << KB) + r), Q((j << KB) + r), "z.x", false, "z.y", "            ");
                    o << "          }\n";
                }
                o << "        }\n";
            }
            return false;
        }
        // matrix op on stage positions
        int pos[3] = {-1, -1, -1};
        for (int t = 0; t < op.nq; ++t) pos[t] = spos(op.lb[t]);
        const int dim = 1 << op.nq;
        std::vector<int> I;
        const std::vector<CplxF> M = op_matrix_f(op, &I);
        int pmask = 0;
        for (int t = 0; t < op.nq; ++t) pmask |= 1 << pos[t];
        for (int j = 0; j < GS; ++j)
            for (int e = 0; e < R; ++e) {
                if (e & pmask) continue;
                int ix[8];
                for (int c = 0; c < dim; ++c) {
                    int r = e;
                    for (int t = 0; t < op.nq; ++t)
                        if ((c >> t) & 1) r |= 1 << pos[t];
                    ix[c] = (j << KB) + r;
                }
                o << "        {";
                for (int c = 0; c < dim; ++c)
                    o << " const float2 xp" << c << " = " << P(ix[c]) << ", xq" << c << " = " << Q(ix[c]) << ";";
                o << "\n";
                for (int r = 0; r < dim; ++r) {
                    std::vector<PTerm> tp, tq;
                    for (int c = 0; c < dim; ++c) {
                        const CplxF k = M[r * dim + c];
                        if (k.re == 0.f && k.im == 0.f) continue;
                        std::string re, im;
                        bool one;
                        coef_parts(m, I[r * dim + c], k, re, one, im);
                        const std::string xp = "xp" + std::to_string(c), xq = "xq" + std::to_string(c);
                        if (!re.empty()) tp.push_back({re, one, xp}), tq.push_back({re, one, xq});
                        if (!im.empty()) tp.push_back({"-(" + im + ")", false, xq}), tq.push_back({im, false, xp});
                    }
                    o << "          " << P(ix[r]) << " = " << chain(tp) << "; " << Q(ix[r]) << " = " << chain(tq)
                      << ";\n";
                }
                o << "        }\n";
            }
        return false;
    }

    // warp sums of measurements cols[c0..c1) (at most 8, accumulators m<c0>..): a
    // transposed butterfly -- each exchange step halves the values a lane carries
    // and doubles the lanes it sums over -- then a plain butterfly; lane L ends with
    // the sum of value ((L >> 4) & 1) * h0 + ((L >> 3) & 1) * h1 + ..., and the
    // lanes with the remaining low bits 0 add it to the warp's row of the partials
    // (with s transposed steps: value (L >> (5 - s)) & (2^s - 1))
    void reduce_measurements(const std::vector<int>& cols, size_t c0, size_t c1) {
        const int n = (int)(c1 - c0);
        int P = 1, steps = 0;
        while (P < n) P <<= 1, ++steps;
        o << "        {  // warp sums of " << n << " measurements\n";
        o << "          const u32 lane = tid & 31u;\n";
        for (int i = 0; i < P; ++i)
            o << "          float r" << i << " = " << (i < n ? "m" + std::to_string(c0 + i) : std::string("0.f")) << ";\n";
        int count = P, d = 16;
        for (int s = 0; s < steps; ++s, d >>= 1) {
            const int half = count >> 1;
            o << "          { const bool up = (lane & " << d << "u) != 0;\n";
            for (int i = 0; i < half; ++i)
                o << "            { const float snd = up ? r" << i << " : r" << (i + half) << "; r" << i << " = (up ? r"
                  << (i + half) << " : r" << i << ") + __shfl_xor_sync(0xffffffffu, snd, " << d << "); }\n";
            o << "          }\n";
            count = half;
        }
        for (; d > 0; d >>= 1) o << "          r0 += __shfl_xor_sync(0xffffffffu, r0, " << d << ");\n";
        // lane bits 4, 3, ... (one per transposed step) name the value it holds
        const int low = 5 - steps;
        o << "          if ((lane & " << ((1u << low) - 1) << "u) == 0u) {\n";
        o << "            const u32 k = (lane >> " << low << ") & " << (P - 1) << "u;\n";
        o << "            const int col = ";
        for (int i = 0; i < n; ++i) o << "k == " << i << "u ? " << cols[c0 + i] << " : ";
        o << "-1;\n";
        o << "            const i64 row = (i64)blockIdx.x * (NT / 32) + (tid >> 5);\n"
             "            if (col >= 0 && row < A.n_rows && col < A.n_cols) atomicAdd(&A.partials[row * A.n_cols + col], (double)r0);\n"
             "          }\n"
             "        }\n";
    }

    // Im<lambda|G|phi> of one measurement over the thread's registers: row r of the
    // signed monomial G holds i^slot[r] at column perm[1 + r] (INNER_ZERO: a zero row);
    // with conj(l) p = a + i b, Im(i^k conj(l) p) = b, a, -b, -a for k = 0..3
    void inner(int m, const int* S, int idx) {
        const DevOp& op = p.ops[m];
        int pos[2] = {-1, -1};
        int pmask = 0;
        for (int t = 0; t < op.nq; ++t) {
            for (int q = 0; q < KB; ++q)
                if (S[q] == op.lb[t]) pos[t] = q;
            pmask |= 1 << pos[t];
        }
        const int dim = 1 << op.nq;
        auto reg_of = [&](int j, int e, int loc) {
            int r = e;
            for (int t = 0; t < op.nq; ++t)
                if ((loc >> t) & 1) r |= 1 << pos[t];
            return (j << KB) + r;
        };
        const std::string acc = "m" + std::to_string(idx);
        o << "        float " << acc << " = 0.f;  // measurement column " << op.perm[0] << "\n";
        for (int j = 0; j < GS; ++j)
            for (int e = 0; e < (1 << KB); ++e) {
                if (e & pmask) continue;
                for (int r = 0; r < dim; ++r) {
                    const int code = op.slot[r];
                    if (code == INNER_ZERO) continue;
                    // lambda = (P.y, Q.y), phi = (P.x, Q.x) of the packed registers
                    const std::string li = std::to_string(reg_of(j, e, r));
                    const std::string qi = std::to_string(reg_of(j, e, op.perm[1 + r]));
                    const std::string lx = "P" + li + ".y", ly = "Q" + li + ".y";
                    const std::string qx = "P" + qi + ".x", qy = "Q" + qi + ".x";
                    const std::string a = "(" + lx + " * " + qx + " + " + ly + " * " + qy + ")";
                    const std::string b = "(" + lx + " * " + qy + " - " + ly + " * " + qx + ")";
                    o << "        " << acc << ((code & 2) ? " -= " : " += ") << ((code & 1) ? a : b) << ";\n";
                }
            }
    }

    // the parameter-block operand of op m's coefficient slot i
    std::string kname(int m, int i) const {
        const auto it = kslot.find({m, i});
        if (it == kslot.end()) throw std::logic_error("jit: coefficient not in the parameter block");
        return "K.k[" + std::to_string(it->second) + "]";
    }

    // row r of op m's matrix times x0..x(dim-1): literals for the trivial entries,
    // named coefficient registers for the rest (real-only when the entry is real)
    void cmac_rt(int m, const std::vector<int>& I, int r, int dim, const std::vector<CplxF>& M, std::string& re,
                 std::string& im) {
        std::vector<std::pair<CplxF, std::string>> lit;
        std::ostringstream rr, ii;
        bool first = true;
        for (int c = 0; c < dim; ++c) {
            const CplxF k = M[r * dim + c];
            const std::string x = "x" + std::to_string(c);
            if (k.re == 0.f && k.im == 0.f) continue;
            if (trivial_coef(k)) {
                lit.push_back({k, x});
                continue;
            }
            const std::string kn = kname(m, I[r * dim + c]);
            if (!first) rr << " + ", ii << " + ";
            first = false;
            if (k.im == 0.f) {
                rr << kn << ".x * " << x << ".x";
                ii << kn << ".x * " << x << ".y";
            } else {
                rr << "(" << kn << ".x * " << x << ".x - " << kn << ".y * " << x << ".y)";
                ii << "(" << kn << ".x * " << x << ".y + " << kn << ".y * " << x << ".x)";
            }
        }
        std::string lr, li;
        cmac_terms(lit, lr, li);
        if (first) {
            re = lr, im = li;
            return;
        }
        re = rr.str() + (lr == "0.f" ? "" : " + " + lr);
        im = ii.str() + (li == "0.f" ? "" : " + " + li);
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
            if (!have_scal) o << "        cf " << scn << " = cf{1.f, 0.f};\n";
        };
        if (op.kind == OPK_STATESCALE) {
            open_scal();
            o << "        " << scn << " = cscale(" << scn << ", (float)((const double*)a.ops[" << m << "].aux)[b]);\n";
            return true;
        }
        if (op.kind == OPK_REALTAB) {
            if (op.aux2 == 0) return false;  // no tables: a marker op (the epilogue's anchor)
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
                o << "        " << scn << " = cmul(" << scn << ", a.ops[" << m << "].c[" << rt.str() << "]);\n";
                return true;
            }
            if (!any_tile_nonstage && !any_off) {
                // every qubit on a stage bit: literal factor per register
                for (int i = 0; i < (GS << KB); ++i) {
                    int mi = 0;
                    for (int t = 0; t < op.nq; ++t) mi |= ((i >> pos[t]) & 1) << t;
                    const float re = op.cf[mi].x, im = op.cf[mi].y;
                    if (re == 1.f && im == 0.f) continue;
                    if (p.rtc && !trivial_coef(CplxF{re, im})) {
                        o << "        " << v(i) << " = cmul(" << kname(m, mi) << ", " << v(i) << ");\n";
                        continue;
                    }
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
        std::vector<int> I;
        const std::vector<CplxF> M = op_matrix_f(op, &I);
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
                    if (p.rtc) cmac_rt(m, I, r, dim, M, re, im);
                    else cmac_terms(terms, re, im);
                    o << "          " << v(ix[r]) << " = cf{" << re << ", " << im << "};\n";
                }
                o << "        }\n";
            }
        }
        return false;
    }
};

// The tile's high qubits hb[0..H) (ascending) as runs of consecutive bit positions:
// the generated address code moves a run with one shift and mask instead of one
// bit at a time.
std::vector<std::pair<int, int>> high_runs(const TileGeom& g) {  // (first m, length)
    std::vector<std::pair<int, int>> runs;
    for (int m = 0; m < g.H; ++m) {
        if (!runs.empty() && g.hb[m] == g.hb[runs.back().first] + runs.back().second) ++runs.back().second;
        else runs.push_back({m, 1});
    }
    return runs;
}
// "var |= bits of src deposited at the high positions" lines
std::string deposit_high(const TileGeom& g, const char* var, const char* src) {
    std::ostringstream o;
    for (const auto& r : high_runs(g))
        o << "    " << var << " |= (u64)((" << src << " >> " << r.first << ") & " << ((1u << r.second) - 1)
          << "u) << " << g.hb[r.first] << ";\n";
    return o.str();
}
// "base = base with zero bits inserted at the high positions" lines (ascending runs)
std::string insert_high_zeros(const TileGeom& g) {
    std::ostringstream o;
    for (const auto& r : high_runs(g)) {
        const int p = g.hb[r.first], k = r.second;
        o << "    base = ((base >> " << p << ") << " << (p + k) << ") | (base & ((1ull << " << p << ") - 1));\n";
    }
    return o.str();
}

// full source of the kernels for one pass
std::string generate_impl(const Pass& p, bool need_epi, int nbuf, int groups, int minb_add, std::string& err) {
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
    if (p.rtc) {  // the run-time coefficients: a second kernel parameter
        const size_t nk = std::max<size_t>(1, gen.kslot.size());
        if (sizeof(TileArgs) + 8 * nk > kMaxKernelParamBytes) {
            err = "jit: the pass has more run-time coefficients than a kernel parameter block holds";
            return "";
        }
        o << "struct Coefs { cf k[" << nk << "]; };\n";
    }
    o << "#define NT " << NT << "\n#define TB " << T << "\n#define LB " << g.L << "\n#define HB " << g.H << "\n";
    o << "#define NSHIFT " << (N - T) << "\n";
    // tile geometry as literals
    o << "__device__ __forceinline__ u64 tile_base(i64 t, i64& b) {\n"
         "    b = t >> NSHIFT;\n"
         "    u64 base = (u64)(t & ((1ll << NSHIFT) - 1)) << LB;\n";
    o << insert_high_zeros(g);
    o << "    return base;\n}\n";
    o << "__device__ __forceinline__ u64 seg_off(u64 base, u32 s) {\n    u64 off = base;\n";
    o << deposit_high(g, "off", "s");
    o << "    return off;\n}\n";
    o << "__device__ __forceinline__ float realtab(const DevOp& op, u64 base, u32 j) {\n"
         "    u64 gi = base | (j & ((1u << LB) - 1));\n"
         "    const u32 h = j >> LB;\n";
    o << deposit_high(g, "gi", "h");
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
    // a hint to bring tile t's segments into L2 while the current tile's stages run
    // (the one-buffer kernels: the next bulk load then reads L2); t is a valid tile,
    // so every segment lies inside the state, 16-byte aligned, a multiple of 16 bytes
    o << "__device__ __forceinline__ void prefetch_tile(const TileArgs& a, i64 t) {\n"
         "    i64 b;\n"
         "    const u64 base = tile_base(t, b);\n"
         "    const cf* gs = (const cf*)a.psi + b * a.state_len;\n"
         "    for (u32 s = threadIdx.x; s < (1u << HB); s += NT)\n"
         "        asm volatile(\"cp.async.bulk.prefetch.L2.global [%0], %1;\" ::\"l\"(gs + seg_off(base, s)), "
         "\"r\"(8u << LB) : \"memory\");\n"
         "}\n";
    o << "template <bool EPI>\n__device__ __forceinline__ void body(const TileArgs& a"
      << (p.rtc ? ", const Coefs& K" : "") << ") {\n"
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
             "    if (t + gridDim.x < a.ntiles) prefetch_tile(a, t + gridDim.x);\n"
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
    const char* params = p.rtc ? "(const TileArgs a, const Coefs K)" : "(const TileArgs a)";
    const char* args = p.rtc ? "(a, K)" : "(a)";
    o << "extern \"C\" __global__ void __launch_bounds__(NT, " << MINB << ") smoq_pass_e0" << params
      << " { body<false>" << args << "; }\n";
    if (need_epi)
        o << "extern \"C\" __global__ void __launch_bounds__(NT, " << MINB << ") smoq_pass_e1" << params
          << " { body<true>" << args << "; }\n";
    return o.str();
}

// full source of the compiled adjoint kernel of one backward pass: the tile pair
// (phi, lambda) in shared memory by bulk copy, then the pass's stages on both
// register sets, measurements added to the warps' partial rows, then both tiles back
std::string generate_adjoint_impl(const Pass& p, std::string& err) {
    const int N = p.g.N;
    const TileGeom& g = p.g;
    const int T = g.T;
    // one 16-amplitude group of each state per thread; 2 CTAs per SM (128 registers
    // a thread: the two register sets plus a stage's run-time coefficients)
    const int G = 1, NT = 1 << (T - 4);
    const int MINB = std::max(1, 65536 / (NT * 128));
    for (const DevOp& op : p.ops)
        if (op.kind == OPK_REALTAB || op.kind == OPK_STATESCALE || op.kind == OPK_JUMP) {
            err = "jit: op kind not supported by the adjoint kernel";
            return "";
        }
    Gen gen(p, G, NT);
    std::ostringstream& o = gen.o;
    o << kPrelude;
    o << "static_assert(sizeof(DevOp) == " << sizeof(DevOp) << ", \"DevOp layout\");\n";
    o << "static_assert(sizeof(TileArgs) == " << sizeof(TileArgs) << ", \"TileArgs layout\");\n";
    o << "struct AdjArgs { TileArgs a; void* lam; double* partials; i64 n_rows; int n_cols; };\n";
    o << "static_assert(sizeof(AdjArgs) == " << sizeof(AdjArgs) << ", \"AdjArgs layout\");\n";
    const size_t nk = gen.kslot.size();
    if (sizeof(AdjArgs) + 8 * std::max<size_t>(1, nk) > kMaxKernelParamBytes) {
        err = "jit: the pass has more run-time coefficients than a kernel parameter block holds";
        return "";
    }
    o << "struct Coefs { cf k[" << std::max<size_t>(1, nk) << "]; };\n";
    o << "#define NT " << NT << "\n#define TB " << T << "\n#define LB " << g.L << "\n#define HB " << g.H << "\n";
    o << "#define NSHIFT " << (N - T) << "\n";
    o << "__device__ __forceinline__ u64 tile_base(i64 t, i64& b) {\n"
         "    b = t >> NSHIFT;\n"
         "    u64 base = (u64)(t & ((1ll << NSHIFT) - 1)) << LB;\n";
    o << insert_high_zeros(g);
    o << "    return base;\n}\n";
    o << "__device__ __forceinline__ u64 seg_off(u64 base, u32 s) {\n    u64 off = base;\n";
    o << deposit_high(g, "off", "s");
    o << "    return off;\n}\n";
    o << "extern \"C\" __global__ void __launch_bounds__(NT, " << MINB << ") smoq_adj_e0(const AdjArgs A, const Coefs K) {\n"
         "    const TileArgs& a = A.a;\n"
         "    extern __shared__ __align__(128) unsigned char smem_raw[];\n"
         "    cf* const tile = (cf*)smem_raw;\n"
         "    cf* const tlam = tile + (1u << TB);\n"
         "    __shared__ __align__(8) u64 bar;\n"
         "    const u32 tid = threadIdx.x;\n"
         "    const u32 seg_bytes = 8u << LB;\n"
         "    if (tid == 0) { mbar_init(&bar, 1); fence_mbar_init(); }\n"
         "    __syncthreads();\n"
         "    u32 phase = 0;\n"
         "    for (i64 t = blockIdx.x; t < a.ntiles; t += gridDim.x) {\n"
         "    i64 b;\n"
         "    const u64 base = tile_base(t, b);\n"
         "    cf* gs = (cf*)a.psi + b * a.state_len;\n"
         "    cf* gl = (cf*)A.lam + b * a.state_len;\n"
         "    if (tid == 0) mbar_arrive_expect_tx(&bar, 16u << TB);\n"
         "    for (u32 s = tid; s < (1u << HB); s += NT) {\n"
         "        bulk_g2s(tile + ((u64)s << LB), gs + seg_off(base, s), seg_bytes, &bar);\n"
         "        bulk_g2s(tlam + ((u64)s << LB), gl + seg_off(base, s), seg_bytes, &bar);\n"
         "    }\n"
         "    const bool ok = mbar_wait_bounded(&bar, phase, a.err);\n"
         "    if (!__syncthreads_and(ok)) { mbar_wait_bounded(&bar, phase, nullptr); return; }\n"
         "    phase ^= 1;\n";
    const int LBk = 4;
    size_t o_i = 0;
    while (o_i < p.ops.size()) {
        const DevOp& h = p.ops[o_i];
        if (h.kind != OPK_STAGE) {
            err = "jit: adjoint pass program is not stage-scheduled";
            return "";
        }
        std::vector<int> members;
        int S[4], rl[4] = {-1, -1, -1, -1};
        if (h.nq == 0) {
            // one wide op: its 3 bits + one pad bit (bank-neutral first)
            const DevOp& op = p.ops[o_i + 1];
            std::vector<int> sv;
            for (int t = 0; t < op.nq; ++t) sv.push_back(op.lb[t]);
            for (int bb = LBk; (int)sv.size() < 4 && bb < T; ++bb)
                if (std::find(sv.begin(), sv.end(), bb) == sv.end()) sv.push_back(bb);
            for (int bb = 0; (int)sv.size() < 4 && bb < T; ++bb)
                if (std::find(sv.begin(), sv.end(), bb) == sv.end()) sv.push_back(bb);
            std::sort(sv.begin(), sv.end());
            int cfree = 0;
            for (int bb = 0; bb < LBk; ++bb)
                if (std::find(sv.begin(), sv.end(), bb) == sv.end()) ++cfree;
            int aa = 0;
            for (int q = 0; q < 4; ++q) {
                S[q] = sv[q];
                rl[q] = sv[q] < LBk ? cfree + aa++ : -1;
            }
            members.push_back((int)o_i + 1);
            o_i += 2;
        } else {
            for (int q = 0; q < 4; ++q) S[q] = h.perm[q], rl[q] = h.perm[4 + q];
            for (int k = 1; k <= (int)h.aux2; ++k) members.push_back((int)(o_i + k));
            o_i += 1 + (size_t)h.aux2;
        }
        gen.stage_dual(S, rl, members);
    }
    o << "    fence_proxy_async_smem();\n"
         "    __syncthreads();\n"
         "    for (u32 s = tid; s < (1u << HB); s += NT) {\n"
         "        bulk_s2g(gs + seg_off(base, s), tile + ((u64)s << LB), seg_bytes);\n"
         "        bulk_s2g(gl + seg_off(base, s), tlam + ((u64)s << LB), seg_bytes);\n"
         "    }\n"
         "    bulk_commit();\n"
         "    bulk_wait_read0();\n"
         "    __syncthreads();\n"
         "    }\n"
         "    bulk_wait0();\n"
         "}\n";
    return o.str();
}

// the generators' failures (an inconsistent pass program) come back as errors,
// never as exceptions through the C ABI
std::string generate(const Pass& p, bool need_epi, int nbuf, int groups, int minb_add, std::string& err) {
    try {
        return generate_impl(p, need_epi, nbuf, groups, minb_add, err);
    } catch (const std::exception& ex) {
        err = ex.what();
        return std::string();
    }
}
std::string generate_adjoint(const Pass& p, std::string& err) {
    try {
        return generate_adjoint_impl(p, err);
    } catch (const std::exception& ex) {
        err = ex.what();
        return std::string();
    }
}

std::mutex g_mu;
std::map<std::string, std::unique_ptr<JitKernel>> g_cache;   // loaded kernels, by source
std::map<std::string, std::vector<char>> g_cubins;           // compiled, not loaded yet
// loaded run-time-coefficient kernels by pass signature (+ kernel variant)
std::map<std::vector<int32_t>, const JitKernel*> g_by_sig;

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

const JitKernel* jit_pass_find(const Pass& p, int nbuf, int groups, int minb_add) {
    if (!p.rtc || !p.staged) return nullptr;
    std::vector<int32_t> key = jit_pass_signature(p);
    key.insert(key.end(), {-2, nbuf, groups, minb_add});
    return jit_sig_find(key);
}

bool jit_pass_source(const Pass& p, int nbuf, int groups, std::string& src, std::string& err) {
    if (!p.staged || (p.g.T != 12 && p.g.T != 13)) {
        err = "jit: only stage-scheduled passes of tile width 12-13";
        return false;
    }
    src = generate(p, p.epilogue, nbuf, groups, 0, err);
    return !src.empty();
}

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

namespace {
// the loaded kernel of a generated source: from the process cache, from a cubin
// that jit_precompile left, or compiled here; then loaded into the current device
const JitKernel* load_source(const std::string& src, int threads, size_t smem, int nfn, const char* const* names,
                             std::string& err) {
    std::vector<char> cubin;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(src);
        if (it != g_cache.end()) return it->second.get();
        auto ct = g_cubins.find(src);  // compiled ahead by jit_precompile
        if (ct != g_cubins.end()) {
            cubin.swap(ct->second);
            g_cubins.erase(ct);
        }
    }
    if (cubin.empty() && !compile_cubin(src, cubin, err)) return nullptr;
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
    k->threads = threads;
    k->smem = smem;
    for (int v = 0; v < nfn; ++v) {
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
    g_cache.emplace(src, std::move(k));
    return out;
}
}  // namespace

// Compile (or fetch) the kernel of a stage-scheduled complex64 pass and load
// it into the current device.  Returns nullptr and fills `err` on failure.  A
// run-time-coefficient pass is looked up by its signature first (no source is
// generated for a later parameter set of the same circuit).
const JitKernel* jit_pass_kernel(const Pass& p, int nbuf, int groups, std::string& err, int minb_add) {
    if (!p.staged || (p.g.T != 12 && p.g.T != 13)) {
        err = "jit: only stage-scheduled passes of tile width 12-13";
        return nullptr;
    }
    std::vector<int32_t> key;
    if (p.rtc) {
        key = jit_pass_signature(p);
        key.insert(key.end(), {-2, nbuf, groups, minb_add});
        if (const JitKernel* k = jit_sig_find(key)) return k;
    }
    std::string src = generate(p, p.epilogue, nbuf, groups, minb_add, err);
    if (src.empty()) return nullptr;
    static const char* const names[2] = {"smoq_pass_e0", "smoq_pass_e1"};
    const JitKernel* k = load_source(src, 1 << (p.g.T - 4 - (groups - 1)), (size_t)(nbuf == 2 ? 16 : 8) << p.g.T,
                                     p.epilogue ? 2 : 1, names, err);
    if (k && p.rtc) {
        const_cast<JitKernel*>(k)->rtc = true;
        std::lock_guard<std::mutex> lk(g_mu);
        g_by_sig.emplace(key, k);
    }
    return k;
}

// the adjoint kernel of a staged backward pass (tile width 12: two 32 KB tiles)
static bool adjoint_ok(const Pass& p, std::string& err) {
    if (!p.staged || p.g.T != 12) {
        err = "jit: the adjoint kernel takes stage-scheduled passes of tile width 12";
        return false;
    }
    return true;
}

void jit_rtc_block(const Pass& p, std::vector<float2>& out) {
    out.clear();
    if (p.rtc)
        for (const auto& mi : rtc_list(p)) out.push_back(p.ops[mi.first].cf[mi.second]);
    if (out.empty()) out.push_back(make_float2(0.f, 0.f));  // (the block has at least one entry)
}

namespace {

// class of a coefficient as the run-time-coefficient generator sees it: the
// literals 0, 1, -1, i, -i; a parameter-block entry read as real or as complex
int32_t coef_class(float2 c) {
    const CplxF k{c.x, c.y};
    if (trivial_coef(k)) return 1 + (int32_t)(k.re + 1.f) * 3 + (int32_t)(k.im + 1.f);
    return k.im == 0.f ? 20 : 21;
}
}  // namespace

// Everything the generators read from a run-time-coefficient pass: its tile
// geometry, and per op the kind, qubits, codes and flags and the class of each
// coefficient (never its value).  Two passes with equal signatures get the same
// kernel source (for the same kernel variant).
std::vector<int32_t> jit_pass_signature(const Pass& p) {
    std::vector<int32_t> s{p.g.N, p.g.T, p.g.L, p.g.H, p.rtc ? 1 : 0, p.staged ? 1 : 0, p.epilogue ? 1 : 0};
    for (int m = 0; m < p.g.H; ++m) s.push_back(p.g.hb[m]);
    for (const DevOp& op : p.ops) {
        s.insert(s.end(), {op.kind, op.nq, op.flags, (int32_t)op.aux2});
        s.insert(s.end(), op.lb, op.lb + 4);
        s.insert(s.end(), op.gb, op.gb + 4);
        s.insert(s.end(), op.slot, op.slot + 4);
        s.insert(s.end(), op.perm, op.perm + 8);
        for (int k = 0; k < 16; ++k) {
            if (p.rtc) s.push_back(coef_class(op.cf[k]));
            else {  // (literal coefficients: the values themselves)
                int32_t b[2];
                std::memcpy(b, &op.cf[k], sizeof b);
                s.insert(s.end(), b, b + 2);
            }
        }
    }
    return s;
}

const JitKernel* jit_sig_find(const std::vector<int32_t>& sig) {
    std::lock_guard<std::mutex> lk(g_mu);
    const auto it = g_by_sig.find(sig);
    return it == g_by_sig.end() ? nullptr : it->second;
}

std::string jit_adjoint_source(const Pass& p, std::string& err) {
    if (!adjoint_ok(p, err)) return std::string();
    return generate_adjoint(p, err);
}

const JitKernel* jit_adjoint_load(const Pass& p, const std::string& src, const std::vector<int32_t>& sig,
                                  std::string& err) {
    if (const JitKernel* k = jit_sig_find(sig)) return k;
    if (!adjoint_ok(p, err)) return nullptr;
    if (src.empty()) {
        err = "jit: no adjoint kernel source";
        return nullptr;
    }
    static const char* const names[1] = {"smoq_adj_e0"};
    const JitKernel* k = load_source(src, 1 << (p.g.T - 4), (size_t)16 << p.g.T, 1, names, err);
    if (k) {
        const_cast<JitKernel*>(k)->rtc = p.rtc;
        std::lock_guard<std::mutex> lk(g_mu);
        g_by_sig.emplace(sig, k);
    }
    return k;
}

bool jit_check_adjoint(const Pass& p, std::string& err, std::string* info, std::string* source) {
    if (!adjoint_ok(p, err)) return false;
    const std::string src = generate_adjoint(p, err);
    if (src.empty()) return false;
    if (source) {
        *source = src;
        return true;
    }
    std::vector<char> cubin;
    return compile_cubin(src, cubin, err, info);
}

bool jit_available() { return nvrtc().ok; }

// NVRTC on host threads for every request whose kernel is neither loaded nor
// compiled yet; the cubins wait in g_cubins until jit_pass_kernel loads them on
// the calling thread (the worker threads make no CUDA calls)
void jit_precompile(const std::vector<JitRequest>& reqs) {
    if (!nvrtc().ok) return;
    std::vector<std::string> srcs;
    for (const JitRequest& r : reqs) {
        if (!r.p || !r.p->staged || (r.p->g.T != 12 && r.p->g.T != 13)) continue;
        std::string err;
        std::string src = generate(*r.p, r.p->epilogue, r.nbuf, r.groups, r.minb_add, err);
        if (!src.empty()) srcs.push_back(std::move(src));
    }
    std::vector<const std::string*> ptr;
    for (const std::string& x : srcs) ptr.push_back(&x);
    jit_precompile_sources(ptr);
}

void jit_precompile_sources(const std::vector<const std::string*>& srcs) {
    if (!nvrtc().ok) return;
    std::vector<std::string> todo;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        std::set<std::string> seen;
        for (const std::string* src : srcs) {
            if (!src || src->empty() || g_cache.count(*src) || g_cubins.count(*src) || !seen.insert(*src).second)
                continue;
            todo.push_back(*src);
        }
    }
    if (todo.empty()) return;
    std::vector<std::vector<char>> out(todo.size());
    std::atomic<size_t> next(0);
    auto work = [&]() {
        for (size_t i; (i = next++) < todo.size();) {
            std::string err;
            if (!compile_cubin(todo[i], out[i], err)) out[i].clear();  // jit_pass_kernel reports the error
        }
    };
    const size_t nt = std::max<size_t>(1, std::min<size_t>(todo.size(), std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
    std::lock_guard<std::mutex> lk(g_mu);
    for (size_t i = 0; i < todo.size(); ++i)
        if (!out[i].empty()) g_cubins.emplace(std::move(todo[i]), std::move(out[i]));
}

uint64_t jit_pass_key(const Pass& p, int nbuf) {
    std::string err;
    const std::string src = generate(p, p.epilogue, nbuf, 2, 0, err);
    return src.empty() ? 0 : fnv1a(src);
}

cudaError_t launch_jit(smoq_ctx* ctx, const TileArgs& a, const JitKernel* k, bool epi, const float2* coefs) {
    const void* fn = k->fn[epi ? 1 : 0];
    if (!fn || (k->rtc && !coefs)) return cudaErrorInvalidValue;
    int64_t grid = (int64_t)ctx->num_sms * k->per_sm[epi ? 1 : 0];
    if (grid > a.ntiles) grid = a.ntiles;
    TileArgs args = a;
    void* params[] = {&args, const_cast<float2*>(coefs)};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)k->threads), params, k->smem, ctx->stream);
}

}  // namespace smoq

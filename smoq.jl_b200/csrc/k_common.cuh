// k_common.cuh -- device helpers: complex arithmetic, bit insertion, PTX
// wrappers for the Blackwell bulk-copy engine (cp.async.bulk + mbarrier) and
// bounded waits.  No wait in this library spins without an iteration limit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "smoq_internal.h"
#include "circuit_common.cuh"

namespace smoq {

enum : int32_t { DEVERR_TIMEOUT = 1, DEVERR_BADINPUT = 2, DEVERR_BOUNDS = 3 };

// Diagnostic builds (-DSMOQ_DEVICE_CHECKS): kernels test the extent of every
// bulk copy and partial-sum index they are about to issue, record a violation
// as DEVERR_BOUNDS | site << 8 in the error word and skip the access.
#ifdef SMOQ_DEVICE_CHECKS
#define SMOQ_INBOUNDS(cond, err, site) \
    ((cond) ? true : ((err) ? (atomicExch((err), DEVERR_BOUNDS | ((site) << 8)), false) : false))
#else
#define SMOQ_INBOUNDS(cond, err, site) true
#endif

template <typename R> struct CT;
template <> struct CT<float> { using T = float2; };
template <> struct CT<double> { using T = double2; };

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 czero(float2) { return make_float2(0.f, 0.f); }
__device__ __forceinline__ double2 czero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double cabs2d(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }
__device__ __forceinline__ double cabs2d(double2 a) { return a.x * a.x + a.y * a.y; }

template <typename R> __device__ __forceinline__ typename CT<R>::T coef(const DevOp& op, int i);
template <> __device__ __forceinline__ float2 coef<float>(const DevOp& op, int i) { return op.cf[i]; }
template <> __device__ __forceinline__ double2 coef<double>(const DevOp& op, int i) { return op.cd[i]; }

// insert a zero bit at position p
template <typename I> __device__ __forceinline__ I ins0(I x, int p) {
    I lo = x & ((I(1) << p) - 1);
    return ((x >> p) << (p + 1)) | lo;
}

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait on an mbarrier phase: gives up after kWaitLimitNs of wall time
// (a legitimate tile copy completes in microseconds) or 2^22 polls, whichever
// comes first, records DEVERR_TIMEOUT and returns false.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* err,
                                                  uint64_t limit_ns = kWaitLimitNs) {
    const uint64_t t0 = globaltimer_ns();
    for (int it = 0; it < (1 << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63 && globaltimer_ns() - t0 > limit_ns) break;
    }
    if (err) atomicExch(err, DEVERR_TIMEOUT);
    return false;
}
// bulk global -> shared copy, completion counted on the mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bulk shared -> global copy (bulk async-group completion)
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ------------------------------------------------------------ random numbers
// philox10 / u01_53 (Philox4x32-10 and its 53-bit uniform) live in
// circuit_common.cuh with the other per-trajectory rules.

// ------------------------------------------------------------ op application
// Apply one fused op to the amplitude array `psi` indexed by I.  `bits` are
// the op's qubit positions in that index space.  `nthr`/`tid` stride the
// groups.  Used on a shared-memory tile (I = uint32_t, local bits) and on a
// whole state in HBM (I = uint64_t, global bits).  `mp` maps a logical index
// to its storage position (identity, or a bank swizzle of a shared-memory
// layout); it must be XOR-linear, mp(x ^ y) = mp(x) ^ mp(y), so that a group's
// other members sit at fixed XOR offsets from its first.
struct IdMap {
    template <typename I>
    __device__ __forceinline__ I operator()(I i) const { return i; }
};
template <typename R, typename I, typename Map = IdMap>
__device__ __forceinline__ void sweep_op(const DevOp& op, typename CT<R>::T* psi, int nbits,
                                         const int* bits, I tid, I nthr, Map mp = Map()) {
    using C = typename CT<R>::T;
    const int kind = op.kind;
    if (kind == OPK_DENSE1) {
        const int a = bits[0];
        const C m0 = coef<R>(op, 0), m1 = coef<R>(op, 1), m2 = coef<R>(op, 2), m3 = coef<R>(op, 3);
        const I n = I(1) << (nbits - 1);
        const I oa = mp(I(1) << a);
        for (I g = tid; g < n; g += nthr) {
            const I i0 = mp(ins0(g, a)), i1 = i0 ^ oa;
            C x = psi[i0], y = psi[i1];
            psi[i0] = cfma(m0, x, cmul(m1, y));
            psi[i1] = cfma(m2, x, cmul(m3, y));
        }
    } else if (kind == OPK_DENSE2 || kind == OPK_PARITY2) {
        const int a = bits[0], b = bits[1];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const I sa = mp(I(1) << a), sb = mp(I(1) << b);  // storage offsets of the op's bits
        const I n = I(1) << (nbits - 2);
        if (kind == OPK_DENSE2) {
            C m[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) m[k] = coef<R>(op, k);
            for (I g = tid; g < n; g += nthr) {
                const I i0 = mp(ins0(ins0(g, lo), hi));
                const I ix[4] = {i0, i0 ^ sa, i0 ^ sb, i0 ^ sa ^ sb};
                C v[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) v[k] = psi[ix[k]];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    C acc = cmul(m[4 * r], v[0]);
                    acc = cfma(m[4 * r + 1], v[1], acc);
                    acc = cfma(m[4 * r + 2], v[2], acc);
                    acc = cfma(m[4 * r + 3], v[3], acc);
                    psi[ix[r]] = acc;
                }
            }
        } else {
            // even block (00,11): e0 e1 / e2 e3 ; odd block (01,10): o0 o1 / o2 o3
            const C e0 = coef<R>(op, 0), e1 = coef<R>(op, 1), e2 = coef<R>(op, 2), e3 = coef<R>(op, 3);
            const C o0 = coef<R>(op, 4), o1 = coef<R>(op, 5), o2 = coef<R>(op, 6), o3 = coef<R>(op, 7);
            for (I g = tid; g < n; g += nthr) {
                const I i0 = mp(ins0(ins0(g, lo), hi));
                const I i1 = i0 ^ sa, i2 = i0 ^ sb, i3 = i0 ^ sa ^ sb;
                C v0 = psi[i0], v1 = psi[i1], v2 = psi[i2], v3 = psi[i3];
                psi[i0] = cfma(e0, v0, cmul(e1, v3));
                psi[i3] = cfma(e2, v0, cmul(e3, v3));
                psi[i1] = cfma(o0, v1, cmul(o1, v2));
                psi[i2] = cfma(o2, v1, cmul(o3, v2));
            }
        }
    } else if (kind == OPK_MONO) {
        const int nq = op.nq;
        int sorted[3] = {bits[0], nq > 1 ? bits[1] : 0, nq > 2 ? bits[2] : 0};
        // insertion sort of the nq positions
        for (int i = 1; i < nq; ++i)
            for (int j = i; j > 0 && sorted[j] < sorted[j - 1]; --j) {
                int t = sorted[j]; sorted[j] = sorted[j - 1]; sorted[j - 1] = t;
            }
        const int dim = 1 << nq;
        const I n = I(1) << (nbits - nq);
        for (I g = tid; g < n; g += nthr) {
            I i0 = g;
            for (int i = 0; i < nq; ++i) i0 = ins0(i0, sorted[i]);
            I ix[8];
            C v[8];
            for (int m = 0; m < dim; ++m) {
                I x = i0;
                for (int t = 0; t < nq; ++t) x |= (I)((m >> t) & 1) << bits[t];
                ix[m] = x;
                v[m] = psi[mp(x)];
            }
            for (int r = 0; r < dim; ++r) psi[mp(ix[r])] = cmul(coef<R>(op, r), v[op.perm[r]]);
        }
    }
}

// Bank spreading.  A shared-memory phase of 16 (complex64) or 8 (complex128)
// lanes covers one 128-byte row; a sweep over an op on bits inside that row
// has every phase hit each bank twice (one such bit) or four times (two).  The
// lanes whose group index has the bits just above the row's free bits set read
// their group with the op's low bits flipped: flip pattern s in the op's
// matrix index space (bit 0 = qubit 0, bit 1 = qubit 1), group member k at
// logical member k ^ s, matrix M'[k][j] = M[k ^ s][j ^ s].  s is fixed per
// thread (groups stride by blockDim, a multiple of 16).
template <typename R>
__device__ __forceinline__ int lane_flip(uint32_t tid, int a, int b) {
    constexpr int B = sizeof(R) == 4 ? 4 : 3;  // amplitude bits of one 128-byte row
    const bool la = a < B, lb = b >= 0 && b < B;
    if (la && lb) {
        const int f = (int)(tid >> (B - 2)) & 3;  // bit 0 flips the lower of the two positions
        return a < b ? f : ((f & 1) << 1) | (f >> 1);
    }
    if (la) return (int)(tid >> (B - 1)) & 1;
    if (lb) return ((int)(tid >> (B - 1)) & 1) << 1;
    return 0;
}
__device__ __forceinline__ uint32_t flip_bits(int s, int a, int b) {
    return ((s & 1) ? 1u << a : 0u) | ((s & 2) ? 1u << b : 0u);
}

// a x + b y for real a, b and complex x, y
template <typename R, typename C>
__device__ __forceinline__ C rmix(R a, C x, R b, C y) {
    C z;
    z.x = fma(a, x.x, b * y.x);
    z.y = fma(a, x.y, b * y.y);
    return z;
}

// The same op on a linear shared-memory tile with bank spreading (lane_flip);
// dense ops with real coefficients (OPF_REAL) multiply by real scalars.
template <typename R>
__device__ __forceinline__ void sweep_op_spread(const DevOp& op, typename CT<R>::T* psi, int T, uint32_t tid,
                                                uint32_t nthr) {
    using C = typename CT<R>::T;
    constexpr int B = sizeof(R) == 4 ? 4 : 3;  // amplitude bits of one 128-byte bank row
    const bool low = (op.kind == OPK_DENSE1 || op.kind == OPK_DENSE2 || op.kind == OPK_PARITY2) &&
                     (op.lb[0] < B || (op.kind != OPK_DENSE1 && op.lb[1] < B));
    if (!low) {  // no member bit inside a bank row: nothing to spread, coefficients stay uniform
        sweep_op<R, uint32_t>(op, psi, T, op.lb, tid, nthr);
        return;
    }
    if (op.kind == OPK_DENSE1) {
        const int a = op.lb[0];
        const int f = lane_flip<R>(tid, a, -1);
        const C c0 = coef<R>(op, 0), c1 = coef<R>(op, 1), c2 = coef<R>(op, 2), c3 = coef<R>(op, 3);
        const C m0 = f ? c3 : c0, m1 = f ? c2 : c1, m2 = f ? c1 : c2, m3 = f ? c0 : c3;
        const bool real = op.flags & OPF_REAL;
        for (uint32_t g = tid; g < (1u << (T - 1)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(g, a) ^ ((uint32_t)f << a), i1 = i0 ^ (1u << a);
            const C x = psi[i0], y = psi[i1];
            if (real) {
                psi[i0] = rmix(m0.x, x, m1.x, y);
                psi[i1] = rmix(m2.x, x, m3.x, y);
            } else {
                psi[i0] = cfma(m0, x, cmul(m1, y));
                psi[i1] = cfma(m2, x, cmul(m3, y));
            }
        }
    } else if (op.kind == OPK_DENSE2) {
        const int a = op.lb[0], b = op.lb[1];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int f = lane_flip<R>(tid, a, b);
        const uint32_t fb = flip_bits(f, a, b);
        C m[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) m[k] = coef<R>(op, (((k >> 2) ^ f) << 2) | ((k & 3) ^ f));
        for (uint32_t g = tid; g < (1u << (T - 2)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(ins0<uint32_t>(g, lo), hi) ^ fb;
            const uint32_t ix[4] = {i0, i0 ^ (1u << a), i0 ^ (1u << b), i0 ^ (1u << a) ^ (1u << b)};
            C v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = psi[ix[k]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C acc = cmul(m[4 * r], v[0]);
                acc = cfma(m[4 * r + 1], v[1], acc);
                acc = cfma(m[4 * r + 2], v[2], acc);
                acc = cfma(m[4 * r + 3], v[3], acc);
                psi[ix[r]] = acc;
            }
        }
    } else if (op.kind == OPK_PARITY2) {
        const int a = op.lb[0], b = op.lb[1];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        // flipped members: s = 1, 2 exchange the even and odd blocks, s = 2, 3 reverse each block
        const int f = lane_flip<R>(tid, a, b);
        const uint32_t fb = flip_bits(f, a, b);
        const int eb = (f == 1 || f == 2) ? 4 : 0, ob = 4 - eb;
        const bool rv = f >= 2;
        const C e0 = coef<R>(op, eb + (rv ? 3 : 0)), e1 = coef<R>(op, eb + (rv ? 2 : 1));
        const C e2 = coef<R>(op, eb + (rv ? 1 : 2)), e3 = coef<R>(op, eb + (rv ? 0 : 3));
        const C o0 = coef<R>(op, ob + (rv ? 3 : 0)), o1 = coef<R>(op, ob + (rv ? 2 : 1));
        const C o2 = coef<R>(op, ob + (rv ? 1 : 2)), o3 = coef<R>(op, ob + (rv ? 0 : 3));
        for (uint32_t g = tid; g < (1u << (T - 2)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(ins0<uint32_t>(g, lo), hi) ^ fb;
            const uint32_t i1 = i0 ^ (1u << a), i2 = i0 ^ (1u << b), i3 = i1 ^ (1u << b);
            const C v0 = psi[i0], v1 = psi[i1], v2 = psi[i2], v3 = psi[i3];
            psi[i0] = cfma(e0, v0, cmul(e1, v3));
            psi[i3] = cfma(e2, v0, cmul(e3, v3));
            psi[i1] = cfma(o0, v1, cmul(o1, v2));
            psi[i2] = cfma(o2, v1, cmul(o3, v2));
        }
    } else {
        sweep_op<R, uint32_t>(op, psi, T, op.lb, tid, nthr);
    }
}

// ------------------------------------------------------- tile bulk loads
// first global index of tile t and the state it belongs to
__device__ __forceinline__ uint64_t tile_base(const TileArgs& a, int64_t t, int64_t& b) {
    b = t / a.tiles_per_state;
    const int64_t r0 = t - b * a.tiles_per_state;
    uint64_t base = (uint64_t)r0 << a.g.L;
    for (int m = 0; m < a.g.H; ++m) base = ins0<uint64_t>(base, a.g.hb[m]);
    return base;
}

// issue the bulk copies that bring tile t into `buf` (completion on `bar`)
template <typename C>
__device__ __forceinline__ void issue_tile_load(const TileArgs& a, int64_t t, C* buf, uint64_t* bar) {
    int64_t b;
    const uint64_t base = tile_base(a, t, b);
    const C* gs = reinterpret_cast<const C*>(a.psi) + b * a.state_len;
    const uint32_t nseg = 1u << a.g.H;
    const uint32_t seg_bytes = (uint32_t)sizeof(C) << a.g.L;
    if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, ((uint32_t)sizeof(C)) << a.g.T);
    for (uint32_t s = threadIdx.x; s < nseg; s += blockDim.x) {
        uint64_t off = base;
        for (int m = 0; m < a.g.H; ++m) off |= (uint64_t)((s >> m) & 1) << a.g.hb[m];
        bulk_g2s(buf + ((size_t)s << a.g.L), gs + off, seg_bytes, bar);
    }
}

}  // namespace smoq

// k_stage.cu -- the stage-sweep fused pass (sm_100a).
//
// Same contract as tile_pass_kernel (one HBM read + one HBM write of every
// tile, the pass's whole op program applied in between, bulk copies in and
// out), but the program runs as STAGES instead of one shared-memory sweep
// per op.  A stage names 4 tile bits S0 < S1 < S2 < S3; a GROUP is the 16
// amplitudes whose index differs only in those bits.  Each thread loads the
// G groups it owns into registers, applies every member op of the stage
// there (ops on S bits, diagonals on any bit), and writes them back.  A
// chain of bond gates (q, q+1), (q+1, q+2), (q+2, q+3) is one stage: 2
// shared-memory sweeps instead of 6.  The G groups of a thread share one
// decode of every op (its coefficients, positions and kind), which is what
// keeps the instruction count near the arithmetic itself.
//
// Bank conflicts.  Amplitude index bits below LB (4 for complex64, 3 for
// complex128) select the shared-memory bank group a half-warp (quarter-warp)
// reaches.  When a stage holds such bits, every thread of the group would
// hit the same banks.  So thread g reads element r of its group at stage
// bits r ^ rot(g), rot(g) taken from the lane bits the group deposit sends
// to bits >= LB: the 16 (8) threads of a phase then cover all bank groups.
// An op applied to the rotated registers uses M'[i][j] = M[i ^ s][j ^ s],
// s = the rotation bits at the op's stage positions: the coefficient index
// is XORed, the register arithmetic stays the same for every thread.
//
// Diagonals whose qubits all lie outside the tile are one complex number per
// tile: they are multiplied into a per-stage scalar applied once at the end.
//
// Launch: complex64 G = 2 groups per thread (T = 12: 128 threads, T = 13:
// 256), complex128 G = 1 (T = 12 only: 256 threads); one tile
// buffer per CTA and several CTAs per SM, so one CTA's bulk copies and
// barriers overlap another's arithmetic; persistent grid over tiles.
#include <cuda_runtime.h>
#include <stdint.h>
#include "k_common.cuh"

namespace smoq {

// ---------------------------------------------------------------- op bodies
// v holds G groups of 16 (group j at v[16 j + r]); every body runs the same
// (already rotated) coefficients over all G groups.

// 1-qubit op on stage position P; c[] = rotated 2x2 (row-major)
template <typename C, int G, int P>
__device__ __forceinline__ void st1(C* v, const C* c) {
#pragma unroll
    for (int e = 0; e < 16 * G; ++e) {
        if (e & (1 << P)) continue;
        const int f = e | (1 << P);
        const C x = v[e], y = v[f];
        v[e] = cfma(c[0], x, cmul(c[1], y));
        v[f] = cfma(c[2], x, cmul(c[3], y));
    }
}

// 2-qubit dense op on stage positions P0 < P1 (op qubit 0 on P0)
template <typename C, int G, int P0, int P1>
__device__ __forceinline__ void st2_dense(C* v, const C* m) {
#pragma unroll
    for (int e = 0; e < 16 * G; ++e) {
        if (e & ((1 << P0) | (1 << P1))) continue;
        const int ix[4] = {e, e | (1 << P0), e | (1 << P1), e | (1 << P0) | (1 << P1)};
        C x[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] = v[ix[k]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            C acc = cmul(m[4 * r], x[0]);
            acc = cfma(m[4 * r + 1], x[1], acc);
            acc = cfma(m[4 * r + 2], x[2], acc);
            acc = cfma(m[4 * r + 3], x[3], acc);
            v[ix[r]] = acc;
        }
    }
}

// 2-qubit parity-preserving op: block A acts on matrix indices (0, 3),
// block B on (1, 2); each block is a 2x2 (row-major a[0..3], b[0..3]).
// DIAGA: block A is diagonal (a[1] = a[2] = 0), known for the whole CTA.
template <typename C, int G, int P0, int P1, bool DIAGA>
__device__ __forceinline__ void st2_parity(C* v, const C* a, const C* b) {
#pragma unroll
    for (int e = 0; e < 16 * G; ++e) {
        if (e & ((1 << P0) | (1 << P1))) continue;
        const int i1 = e | (1 << P0), i2 = e | (1 << P1), i3 = e | (1 << P0) | (1 << P1);
        const C x0 = v[e], x3 = v[i3], x1 = v[i1], x2 = v[i2];
        if (DIAGA) {
            v[e] = cmul(a[0], x0);
            v[i3] = cmul(a[3], x3);
        } else {
            v[e] = cfma(a[0], x0, cmul(a[1], x3));
            v[i3] = cfma(a[2], x0, cmul(a[3], x3));
        }
        v[i1] = cfma(b[0], x1, cmul(b[1], x2));
        v[i2] = cfma(b[2], x1, cmul(b[3], x2));
    }
}

template <typename R, int G>
__device__ __forceinline__ void stage_op1(typename CT<R>::T* v, const DevOp& op, int rot) {
    using C = typename CT<R>::T;
    const int P = op.slot[0];
    const int x = ((rot >> P) & 1) * 3;  // (i ^ s) * 2 + (j ^ s) = (2i + j) ^ 3s
    C c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = coef<R>(op, k ^ x);
    switch (P) {
        case 0: st1<C, G, 0>(v, c); break;
        case 1: st1<C, G, 1>(v, c); break;
        case 2: st1<C, G, 2>(v, c); break;
        default: st1<C, G, 3>(v, c); break;
    }
}

template <typename R, int G>
__device__ __forceinline__ void stage_dense2(typename CT<R>::T* v, const DevOp& op, int rot) {
    using C = typename CT<R>::T;
    const int P0 = op.slot[0], P1 = op.slot[1];
    const int s = ((rot >> P0) & 1) | (((rot >> P1) & 1) << 1);
    const int x = s * 5;  // (i ^ s) * 4 + (j ^ s) = (4i + j) ^ 5s
    C m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) m[k] = coef<R>(op, k ^ x);
    switch (P0 * 4 + P1) {
        case 1: st2_dense<C, G, 0, 1>(v, m); break;
        case 2: st2_dense<C, G, 0, 2>(v, m); break;
        case 3: st2_dense<C, G, 0, 3>(v, m); break;
        case 6: st2_dense<C, G, 1, 2>(v, m); break;
        case 7: st2_dense<C, G, 1, 3>(v, m); break;
        default: st2_dense<C, G, 2, 3>(v, m); break;
    }
}

template <typename C, int G, int P0, int P1>
__device__ __forceinline__ void st2_parity_mode(C* v, const C* a, const C* b, bool diaga) {
    if (diaga) st2_parity<C, G, P0, P1, true>(v, a, b);
    else st2_parity<C, G, P0, P1, false>(v, a, b);
}

template <typename R, int G>
__device__ __forceinline__ void stage_parity2(typename CT<R>::T* v, const DevOp& op, int rot, int rotmask) {
    using C = typename CT<R>::T;
    const int P0 = op.slot[0], P1 = op.slot[1];
    const int s = ((rot >> P0) & 1) | (((rot >> P1) & 1) << 1);
    // parity blocks of M'[i][j] = M[i ^ s][j ^ s]: an odd s swaps the even
    // (00, 11) and odd (01, 10) blocks, s >= 2 mirrors both
    const int par = (s ^ (s >> 1)) & 1;
    const int x = (s >> 1) * 3;
    const int ba = par ? 4 : 0, bb = par ? 0 : 4;
    C a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a[k] = coef<R>(op, ba + (k ^ x));
        b[k] = coef<R>(op, bb + (k ^ x));
    }
    // the even block is diagonal and no thread rotates these positions
    const bool diaga = (op.flags & 1) && ((rotmask >> P0) & 1) == 0 && ((rotmask >> P1) & 1) == 0;
    switch (P0 * 4 + P1) {
        case 1: st2_parity_mode<C, G, 0, 1>(v, a, b, diaga); break;
        case 2: st2_parity_mode<C, G, 0, 2>(v, a, b, diaga); break;
        case 3: st2_parity_mode<C, G, 0, 3>(v, a, b, diaga); break;
        case 6: st2_parity_mode<C, G, 1, 2>(v, a, b, diaga); break;
        case 7: st2_parity_mode<C, G, 1, 3>(v, a, b, diaga); break;
        default: st2_parity_mode<C, G, 2, 3>(v, a, b, diaga); break;
    }
}

// global index of tile-local index j
__device__ __forceinline__ uint64_t global_of_local(const TileGeom& g, uint64_t base, uint32_t j) {
    uint64_t gi = base | (j & ((1u << g.L) - 1));
    const uint32_t h = j >> g.L;
    for (int m = 0; m < g.H; ++m) gi |= (uint64_t)((h >> m) & 1) << g.hb[m];
    return gi;
}

__device__ __forceinline__ float2 cone(float2) { return make_float2(1.f, 0.f); }
__device__ __forceinline__ double2 cone(double2) { return make_double2(1.0, 0.0); }

// ----------------------------------------------------------------- a stage
// Thread tid owns groups tid + j * NT (j < G) of the stage.
template <typename R, int G, int NT>
__device__ __forceinline__ void run_stage(const TileArgs& a, const DevOp& h, int nmem, const DevOp* mem,
                                          typename CT<R>::T* tile, uint32_t tid, uint64_t base, int64_t b) {
    using C = typename CT<R>::T;
    C v[16 * G];
    const int S0 = h.perm[0], S1 = h.perm[1], S2 = h.perm[2], S3 = h.perm[3];
    auto deposit = [&](uint32_t g) {
        return ins0<uint32_t>(ins0<uint32_t>(ins0<uint32_t>(ins0<uint32_t>(g, S0), S1), S2), S3);
    };
    int rot = 0, rotmask = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int lb = h.perm[4 + q];
        if (lb >= 0) {
            rot |= (int)((tid >> lb) & 1) << q;
            rotmask |= 1 << q;
        }
    }
    uint32_t o0 = 1u << S0, o1 = 1u << S1, o2 = 1u << S2, o3 = 1u << S3;
    uint32_t ga = deposit(tid) ^ ((rot & 1) ? o0 : 0u) ^ ((rot & 2) ? o1 : 0u) ^ ((rot & 4) ? o2 : 0u) ^
                        ((rot & 8) ? o3 : 0u);
    uint32_t gstep = G > 1 ? deposit((uint32_t)NT) : 0u;  // address offset of group j = 1
    // tile-local index held by register i (group i / 16, stage bits (i % 16) ^ rot)
#define ST_AD(i)                                                                                             \
    (ga ^ (((i) >> 4) ? gstep : 0u) ^ (((i) & 1) ? o0 : 0u) ^ (((i) & 2) ? o1 : 0u) ^ (((i) & 4) ? o2 : 0u) ^ \
     (((i) & 8) ? o3 : 0u))
#pragma unroll
    for (int i = 0; i < 16 * G; ++i) v[i] = tile[ST_AD(i)];

    C scal = cone(C());
    bool have_scal = false;  // uniform over the CTA
    for (int m = 0; m < nmem; ++m) {
        const DevOp& op = mem[m];
        const int kind = op.kind;
        if (kind == OPK_PARITY2) {
            stage_parity2<R, G>(v, op, rot, rotmask);
        } else if (kind == OPK_DIAG) {
            int sh[4];
            int cm = 0;
            bool ontile = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool in = q < op.nq;
                sh[q] = (in && op.lb[q] >= 0) ? op.lb[q] : -1;
                ontile |= sh[q] >= 0;
                if (in && op.lb[q] < 0) cm |= (int)((base >> op.gb[q]) & 1) << q;
            }
            if (!ontile) {
                scal = cmul(coef<R>(op, cm), scal);
                have_scal = true;
                continue;
            }
#pragma unroll
            for (int i = 0; i < 16 * G; ++i) {
                int mi = cm;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (sh[q] >= 0) mi |= (int)((ST_AD(i) >> sh[q]) & 1) << q;
                v[i] = cmul(coef<R>(op, mi), v[i]);
            }
        } else if (kind == OPK_STATESCALE) {
            scal = cscale(scal, (R)((const double*)op.aux)[b]);
            have_scal = true;
        } else if (kind == OPK_REALTAB) {
            const double* tab = (const double*)op.aux;
            const int ntab = (int)op.aux2;
#pragma unroll
            for (int i = 0; i < 16 * G; ++i) {
                const uint64_t gi = global_of_local(a.g, base, ST_AD(i));
                double f = 1.0;
                for (int q = 0; q < ntab; ++q) f *= tab[q * 256 + ((gi >> (8 * q)) & 255)];
                v[i] = cscale(v[i], (R)f);
            }
        } else if (op.nq == 1) {
            stage_op1<R, G>(v, op, rot);
        } else {
            stage_dense2<R, G>(v, op, rot);
        }
    }
    if (have_scal) {
#pragma unroll
        for (int i = 0; i < 16 * G; ++i) v[i] = cmul(scal, v[i]);
    }
    // make the address terms opaque here: the store recomputes the 16 G
    // addresses instead of keeping the load's copies live across the ops
    asm volatile("" : "+r"(ga), "+r"(o0), "+r"(o1), "+r"(o2), "+r"(o3), "+r"(gstep));
#pragma unroll
    for (int i = 0; i < 16 * G; ++i) tile[ST_AD(i)] = v[i];
#undef ST_AD
}

// ----------------------------------------------------------------- kernel
template <typename R, bool EPI, int NT, int G, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const TileArgs a) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* tile = reinterpret_cast<C*>(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ double red[NT / 32][16];
    const int tid = threadIdx.x;
    const int T = a.g.T, L = a.g.L, H = a.g.H;
    const uint32_t amps = 1u << T;  // = 16 * G * NT (checked at launch)
    const uint32_t nseg = 1u << H;
    const uint32_t seg_bytes = (uint32_t)sizeof(C) << L;

    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;

    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        int64_t b;
        const uint64_t base = tile_base(a, t, b);
        C* gs = reinterpret_cast<C*>(a.psi) + b * a.state_len;
        issue_tile_load<C>(a, t, tile, &bar);
        const bool ok = mbar_wait_bounded(&bar, phase, a.err);
        if (!__syncthreads_and(ok)) {
            mbar_wait_bounded(&bar, phase, nullptr);  // let copies in flight land
            return;
        }
        phase ^= 1;

        // ---- the stages
        for (int o = 0; o < a.nops;) {
            const DevOp& h = a.ops[o];
            if (h.nq == 0) {
                // a wide op (3-qubit permutation): one plain shared-memory sweep
                const DevOp& op = a.ops[o + 1];
                sweep_op<R, uint32_t>(op, tile, T, op.lb, (uint32_t)tid, (uint32_t)NT);
                __syncthreads();
                o += 2;
                continue;
            }
            const int nmem = (int)h.aux2;
            run_stage<R, G, NT>(a, h, nmem, a.ops + o + 1, tile, (uint32_t)tid, base, b);
            __syncthreads();
            o += 1 + nmem;
        }

        // ---- optional epilogue: |psi|^2 and per tile-bit populations
        if (EPI) {
            constexpr int nb = NT == 128 ? 7 : NT == 256 ? 8 : 9;  // thread-index bits of j
            double acc[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) acc[q] = 0.0;
            for (uint32_t j = tid; j < amps; j += NT) {
                const double p = cabs2d(tile[j]);
                acc[0] += p;
#pragma unroll
                for (int l = nb; l < 15; ++l)
                    if (l < T && ((j >> l) & 1)) acc[1 + l] += p;
            }
#pragma unroll
            for (int l = 0; l < nb; ++l) acc[1 + l] = ((tid >> l) & 1) ? acc[0] : 0.0;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                double x = acc[q];
                for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
                if ((tid & 31) == 0) red[tid >> 5][q] = x;
            }
            __syncthreads();
            if (tid < 16) {
                double s = 0;
                for (int w = 0; w < NT / 32; ++w) s += red[w][tid];
                red[0][tid] = s;  // each tid < 16 owns column tid: no race
            }
            __syncthreads();
            if (tid == 0) {
                double* out = a.ep.partials + (size_t)t * (1 + a.ep.npop);
                out[0] = red[0][0];
                for (int q = 0; q < a.ep.npop; ++q) {
                    const int qq = a.ep.popq[q];
                    int l = -1;
                    if (qq < L) l = qq;
                    for (int m = 0; m < H; ++m)
                        if (a.g.hb[m] == qq) l = L + m;
                    out[1 + q] = (l >= 0) ? red[0][1 + l] : (((base >> qq) & 1) ? red[0][0] : 0.0);
                }
            }
            __syncthreads();
        }

        // ---- store: generic-proxy writes -> async-proxy reads need the fence
        fence_proxy_async_smem();
        __syncthreads();
        for (uint32_t s = tid; s < nseg; s += NT) {
            uint64_t off = base;
            for (int m = 0; m < H; ++m) off |= (uint64_t)((s >> m) & 1) << a.g.hb[m];
            bulk_s2g(gs + off, tile + ((size_t)s << L), seg_bytes);
        }
        bulk_commit();
        bulk_wait_read0();
        __syncthreads();
    }
    bulk_wait0();
}

// ------------------------------------------------------------------ launch
// Configurations [dtype][T - 12]: threads, groups per thread, CTAs per SM the
// register budget is sized for (128 registers a thread, 255 for complex128 T=12).
template <typename R, bool EPI, int NT, int G, int MINB>
static cudaError_t st_init_one(smoq_ctx* ctx, int dt, int T) {
    auto kern = stage_kernel<R, EPI, NT, G, MINB>;
    const size_t smem = sizeof(typename CT<R>::T) << T;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
    if (e != cudaSuccess) return e;
    ctx->st_occ[dt][EPI ? 1 : 0][T - 12] = per_sm < 1 ? 1 : per_sm;
    return cudaSuccess;
}

template <bool EPI>
static cudaError_t st_init_epi(smoq_ctx* ctx) {
    cudaError_t e;
    if ((e = st_init_one<float, EPI, 128, 2, 4>(ctx, 0, 12)) != cudaSuccess) return e;
    if ((e = st_init_one<float, EPI, 256, 2, 2>(ctx, 0, 13)) != cudaSuccess) return e;
    return st_init_one<double, EPI, 256, 1, 1>(ctx, 1, 12);
}

cudaError_t stage_kernels_init(smoq_ctx* ctx) {
    cudaError_t e = st_init_epi<false>(ctx);
    if (e != cudaSuccess) return e;
    return st_init_epi<true>(ctx);
}

template <typename R, bool EPI, int NT, int G, int MINB>
static cudaError_t st_launch(smoq_ctx* ctx, const TileArgs& a, int dt) {
    const int T = a.g.T;
    if ((1u << T) != 16u * G * NT) return cudaErrorInvalidValue;
    int per_sm = ctx->st_occ[dt][EPI ? 1 : 0][T - 12];
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)ctx->num_sms * per_sm;
    if (grid > a.ntiles) grid = a.ntiles;
    stage_kernel<R, EPI, NT, G, MINB><<<(unsigned)grid, NT, sizeof(typename CT<R>::T) << T, ctx->stream>>>(a);
    return cudaGetLastError();
}

template <bool EPI>
static cudaError_t st_launch_epi(smoq_ctx* ctx, const TileArgs& a, int dtype) {
    const int T = a.g.T;
    if (dtype == SMOQ_C64) {
        if (T == 12) return st_launch<float, EPI, 128, 2, 4>(ctx, a, 0);
        if (T == 13) return st_launch<float, EPI, 256, 2, 2>(ctx, a, 0);
    } else {
        if (T == 12) return st_launch<double, EPI, 256, 1, 1>(ctx, a, 1);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage(smoq_ctx* ctx, const TileArgs& a, int dtype, bool epi) {
    return epi ? st_launch_epi<true>(ctx, a, dtype) : st_launch_epi<false>(ctx, a, dtype);
}

}  // namespace smoq

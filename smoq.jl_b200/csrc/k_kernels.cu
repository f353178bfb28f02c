// k_kernels.cu -- the CUDA kernels of libsmoq_cuda.so (sm_100a).
//
//  * tile_pass_kernel: the fused gate pass.  A CTA owns one tile at a time:
//    2^T amplitudes whose index varies over the low L bits and H chosen high
//    bits.  The tile's 2^H contiguous segments (2^L amplitudes each) are
//    brought into shared memory by the bulk-copy engine (cp.async.bulk,
//    completion on an mbarrier), every op of the pass's program is applied
//    in shared memory, and the segments go back with bulk stores.  One HBM
//    read + one HBM write of the tile per pass, however many gates the
//    program holds.  Persistent: the grid is a multiple of the SM count and
//    CTAs stride over tiles.
//  * direct_op_kernel: one op on a whole state straight from HBM (the plain,
//    one-launch-per-gate path behind the single-gate C entry points).
//  * diag_reduce / pauli_reduce + finalize: FP64 expectation reductions,
//    per-block partials then a deterministic second pass.
#include <cuda_runtime.h>
#include <stdint.h>
#include "k_common.cuh"

namespace smoq {

constexpr int TILE_THREADS = 256;
constexpr int RED_THREADS = 256;

// bit value of an op qubit inside a tile: tile bit -> from the local index,
// otherwise constant over the tile (from the tile's base index)
struct DiagBits {
    int nq;
    int shift[3];     // local bit, or -1
    int constv[3];    // value when not a tile bit
};

template <typename R>
__device__ __forceinline__ void tile_diag(const DevOp& op, typename CT<R>::T* tile, uint32_t amps,
                                          uint64_t base) {
    const int nq = op.nq;
    int sh[4] = {-1, -1, -1, -1};
    int cm = 0;  // constant part of the matrix index
    for (int t = 0; t < nq; ++t) {
        if (op.lb[t] >= 0) sh[t] = op.lb[t];
        else cm |= (int)((base >> op.gb[t]) & 1) << t;
    }
    for (uint32_t j = threadIdx.x; j < amps; j += blockDim.x) {
        int m = cm;
#pragma unroll
        for (int t = 0; t < 4; ++t)
            if (sh[t] >= 0) m |= (int)((j >> sh[t]) & 1) << t;
        tile[j] = cmul(coef<R>(op, m), tile[j]);  // op lives in global memory: a cached load
    }
}

template <typename R>
__device__ __forceinline__ void tile_realtab(const DevOp& op, typename CT<R>::T* tile, const TileGeom& g,
                                             uint64_t base) {
    const double* tab = (const double*)op.aux;
    const int ntab = (int)op.aux2;
    const uint32_t amps = 1u << g.T;
    const uint32_t lowmask = (1u << g.L) - 1;
    for (uint32_t j = threadIdx.x; j < amps; j += blockDim.x) {
        uint64_t gi = base | (j & lowmask);
        uint32_t h = j >> g.L;
        for (int m = 0; m < g.H; ++m) gi |= (uint64_t)((h >> m) & 1) << g.hb[m];
        double f = 1.0;
        for (int k = 0; k < ntab; ++k) f *= tab[k * 256 + ((gi >> (8 * k)) & 255)];
        tile[j] = cscale(tile[j], (R)f);
    }
}

template <typename R, bool EPI>
__global__ void __launch_bounds__(TILE_THREADS) tile_pass_kernel(const TileArgs a) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* tile = reinterpret_cast<C*>(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ double red[TILE_THREADS / 32][16];
    const int tid = threadIdx.x;
    const int T = a.g.T, L = a.g.L, H = a.g.H;
    const uint32_t amps = 1u << T;
    const uint32_t nseg = 1u << H;
    const uint32_t seg_bytes = (uint32_t)sizeof(C) << L;

    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;

    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int64_t b = t / a.tiles_per_state;
        const int64_t r = t - b * a.tiles_per_state;
        uint64_t base = (uint64_t)r << L;
        for (int m = 0; m < H; ++m) base = ins0<uint64_t>(base, a.g.hb[m]);
        C* gs = reinterpret_cast<C*>(a.psi) + b * a.state_len;

        // ---- load: one bulk copy per contiguous segment
        if (tid == 0) mbar_arrive_expect_tx(&bar, amps * (uint32_t)sizeof(C));
        for (uint32_t s = tid; s < nseg; s += blockDim.x) {
            uint64_t off = base;
            for (int m = 0; m < H; ++m) off |= (uint64_t)((s >> m) & 1) << a.g.hb[m];
            if (SMOQ_INBOUNDS(b * a.tiles_per_state < a.ntiles && off + (1ull << L) <= (uint64_t)a.state_len, a.err, 1))
                bulk_g2s(tile + ((size_t)s << L), gs + off, seg_bytes, &bar);
        }
        const bool ok = mbar_wait_bounded(&bar, phase, a.err);
        if (!__syncthreads_and(ok)) {
            mbar_wait_bounded(&bar, phase, nullptr);  // let copies in flight land
            return;
        }
        phase ^= 1;

        // ---- the pass program, in shared memory
        for (int o = 0; o < a.nops; ++o) {
            const DevOp& op = a.ops[o];
            const int kind = op.kind;
            if (kind == OPK_DIAG) {
                tile_diag<R>(op, tile, amps, base);
            } else if (kind == OPK_STATESCALE) {
                const R s = (R)((const double*)op.aux)[b];
                for (uint32_t j = tid; j < amps; j += blockDim.x) tile[j] = cscale(tile[j], s);
            } else if (kind == OPK_REALTAB) {
                tile_realtab<R>(op, tile, a.g, base);
            } else {
                sweep_op_spread<R>(op, tile, T, (uint32_t)tid, (uint32_t)blockDim.x);
            }
            __syncthreads();
        }

        // ---- optional epilogue: |psi|^2 and per-bit populations of this tile
        if (EPI) {
            double v[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = 0.0;
            for (uint32_t j = tid; j < amps; j += blockDim.x) {
                const double p = cabs2d(tile[j]);
                v[0] += p;
#pragma unroll
                for (int l = 8; l < 15; ++l)
                    if (l < T && ((j >> l) & 1)) v[1 + l] += p;
            }
#pragma unroll
            for (int l = 0; l < 8; ++l)
                if (l < T) v[1 + l] = ((tid >> l) & 1) ? v[0] : 0.0;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                double x = v[k];
                for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
                if ((tid & 31) == 0) red[tid >> 5][k] = x;
            }
            __syncthreads();
            if (tid < 16) {
                double s = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][tid];
                red[0][tid] = s;  // each tid < 16 owns column tid: no race
            }
            __syncthreads();
            if (tid == 0) {
                double* out = a.ep.partials + (size_t)t * (1 + a.ep.npop);
                out[0] = red[0][0];
                for (int k = 0; k < a.ep.npop; ++k) {
                    const int q = a.ep.popq[k];
                    int l = -1;
                    if (q < L) l = q;
                    for (int m = 0; m < H; ++m)
                        if (a.g.hb[m] == q) l = L + m;
                    out[1 + k] = (l >= 0) ? red[0][1 + l] : (((base >> q) & 1) ? red[0][0] : 0.0);
                }
            }
            __syncthreads();
        }

        // ---- store: generic-proxy writes -> async-proxy reads need the fence
        fence_proxy_async_smem();
        __syncthreads();
        for (uint32_t s = tid; s < nseg; s += blockDim.x) {
            uint64_t off = base;
            for (int m = 0; m < H; ++m) off |= (uint64_t)((s >> m) & 1) << a.g.hb[m];
            if (SMOQ_INBOUNDS(b * a.tiles_per_state < a.ntiles && off + (1ull << L) <= (uint64_t)a.state_len, a.err, 2))
                bulk_s2g(gs + off, tile + ((size_t)s << L), seg_bytes);
        }
        bulk_commit();
        bulk_wait_read0();
        __syncthreads();
    }
    bulk_wait0();
}

// ------------------------------------------------------------ direct kernels
template <typename R>
__global__ void __launch_bounds__(256) direct_op_kernel(typename CT<R>::T* psi, int N, int64_t B,
                                                         const DevOp op) {
    using C = typename CT<R>::T;
    const int64_t len = (int64_t)1 << N;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
    const int kind = op.kind;
    if (kind == OPK_DIAG || kind == OPK_STATESCALE) {
        C ph[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) ph[m] = coef<R>(op, m);
        const uint64_t total = (uint64_t)B * len;
        for (uint64_t i = tid; i < total; i += nthr) {
            C p;
            if (kind == OPK_DIAG) {
                int m = 0;
                for (int t = 0; t < op.nq; ++t) m |= (int)((i >> op.gb[t]) & 1) << t;
                p = ph[0];
#pragma unroll
                for (int k = 1; k < 16; ++k)
                    if (m == k) p = ph[k];
            } else {
                p = czero(ph[0]);
                p.x = (R)((const double*)op.aux)[i >> N];
            }
            psi[i] = cmul(p, psi[i]);
        }
        return;
    }
    // pair / quartet / group ops: the state index space of each batch member
    for (int64_t b = 0; b < B; ++b)
        sweep_op<R, uint64_t>(op, psi + b * len, N, op.gb, tid, nthr);
}

// --------------------------------------------------------------- failure path
// A wait that nothing completes: the barrier's one arrival comes with an
// expectation of 16 bytes that no copy delivers, so the bounded wait of the
// tile kernels (mbar_wait_bounded) runs out after limit_ns, records
// DEVERR_TIMEOUT in the error word and returns.  No copy is issued, so nothing
// is in flight when the block exits.
__global__ void wait_timeout_probe_kernel(int32_t* err, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar, 16);
        mbar_wait_bounded(&bar, 0, err, limit_ns);
    }
}

cudaError_t launch_wait_timeout_probe(smoq_ctx* ctx, uint64_t limit_ns) {
    wait_timeout_probe_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_err, limit_ns);
    ctx->launches++;
    return cudaGetLastError();
}

// --------------------------------------------------------------- reductions
// out_partials[(b * nblk + blk) * nobs + o] = sum over this block's amplitudes
// of |psi|^2 * (-1)^{popc(i & zmask_o)}.  Accumulation in FP64.
constexpr int MAX_DIAG_OBS = 32;
struct ZMasks {
    uint64_t m[MAX_DIAG_OBS];
};

template <typename R>
__global__ void __launch_bounds__(RED_THREADS) diag_reduce_kernel(const typename CT<R>::T* psi, int N,
                                                                   ZMasks zm, int nobs,
                                                                   double* partials) {
    const int64_t len = (int64_t)1 << N;
    const int64_t b = blockIdx.y;
    const int nblk = gridDim.x;
    const typename CT<R>::T* s = psi + b * len;
    double acc[MAX_DIAG_OBS];
#pragma unroll
    for (int o = 0; o < MAX_DIAG_OBS; ++o) acc[o] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
         i += (int64_t)nblk * blockDim.x) {
        const double p = cabs2d(s[i]);
#pragma unroll
        for (int o = 0; o < MAX_DIAG_OBS; ++o)
            if (o < nobs) acc[o] += (__popcll((uint64_t)i & zm.m[o]) & 1) ? -p : p;
    }
    __shared__ double red[RED_THREADS / 32][MAX_DIAG_OBS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < MAX_DIAG_OBS; ++o) {
        if (o < nobs) {
            double x = acc[o];
            for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
            if (lane == 0) red[w][o] = x;
        }
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double x = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x += red[k][threadIdx.x];
        partials[((size_t)b * nblk + blockIdx.x) * nobs + threadIdx.x] = x;
    }
}

// The same sums through a 16-point Walsh-Hadamard transform per chunk of 16
// consecutive amplitudes (N >= 4).  Within a chunk starting at i0 the index
// bits above bit 3 are fixed, so
//   sum_j p_{i0+j} (-1)^{popc((i0 + j) & m)} = (-1)^{popc(i0 & m)} W[m & 15],
// W = the transform of the chunk's 16 probabilities.  Per amplitude that is
// about 8 FP64 operations whatever the number of observables (the direct
// loop above costs one popcount, select and add per observable).
template <typename C>
__device__ __forceinline__ void load16_abs2(const C* c, double* w);
template <>
__device__ __forceinline__ void load16_abs2<float2>(const float2* c, double* w) {
    const float4* c4 = reinterpret_cast<const float4*>(c);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float4 v = c4[k];
        w[2 * k] = (double)v.x * v.x + (double)v.y * v.y;
        w[2 * k + 1] = (double)v.z * v.z + (double)v.w * v.w;
    }
}
template <>
__device__ __forceinline__ void load16_abs2<double2>(const double2* c, double* w) {
#pragma unroll
    for (int k = 0; k < 16; ++k) w[k] = cabs2d(c[k]);
}

template <typename R>
__global__ void __launch_bounds__(RED_THREADS) diag_reduce_wht_kernel(const typename CT<R>::T* psi, int N,
                                                                       ZMasks zm, int nobs, double* partials) {
    const int64_t len = (int64_t)1 << N;
    const int64_t b = blockIdx.y;
    const int nblk = gridDim.x;
    const typename CT<R>::T* s = psi + b * len;
    __shared__ double wsm[16][RED_THREADS];  // column threadIdx.x belongs to this thread
    double acc[MAX_DIAG_OBS];
#pragma unroll
    for (int o = 0; o < MAX_DIAG_OBS; ++o) acc[o] = 0.0;
    const int64_t nchunks = len >> 4;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nchunks;
         q += (int64_t)nblk * blockDim.x) {
        double w[16];
        load16_abs2(s + (q << 4), w);
#pragma unroll
        for (int h = 1; h < 16; h <<= 1)
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (!(j & h)) {
                    const double x = w[j], y = w[j + h];
                    w[j] = x + y;
                    w[j + h] = x - y;
                }
#pragma unroll
        for (int m = 0; m < 16; ++m) wsm[m][threadIdx.x] = w[m];
        const uint64_t i0 = (uint64_t)q << 4;
#pragma unroll
        for (int o = 0; o < MAX_DIAG_OBS; ++o)
            if (o < nobs) {
                const double x = wsm[zm.m[o] & 15][threadIdx.x];
                acc[o] += (__popcll(i0 & zm.m[o]) & 1) ? -x : x;
            }
    }
    __shared__ double red[RED_THREADS / 32][MAX_DIAG_OBS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < MAX_DIAG_OBS; ++o) {
        if (o < nobs) {
            double x = acc[o];
            for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
            if (lane == 0) red[w][o] = x;
        }
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double x = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x += red[k][threadIdx.x];
        partials[((size_t)b * nblk + blockIdx.x) * nobs + threadIdx.x] = x;
    }
}

// <P> for a Pauli string with X/Y part xmask != 0:
//   <P> = sum_{i: bit x0 of i = 0} 2 Re( conj(psi_{i^x}) c_i psi_i ),
//   c_i = i^{ny} (-1)^{popc(i & zmask)}  (P|i> = c_i |i ^ xmask>, Y = iXZ)
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) pauli_reduce_kernel(const typename CT<R>::T* psi, int N,
                                                                    uint64_t xmask, uint64_t zmask,
                                                                    int ny, double* partials) {
    const int64_t len = (int64_t)1 << N;
    const int64_t half = len >> 1;
    const int x0 = __ffsll((long long)xmask) - 1;
    const int64_t b = blockIdx.y;
    const int nblk = gridDim.x;
    const typename CT<R>::T* s = psi + b * len;
    // i^{ny}: 0 -> 1, 1 -> i, 2 -> -1, 3 -> -i
    const int yk = ny & 3;
    double acc = 0.0;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < half;
         g += (int64_t)nblk * blockDim.x) {
        const uint64_t i = ins0<uint64_t>((uint64_t)g, x0);
        const uint64_t j = i ^ xmask;
        const auto a = s[i], c = s[j];
        // z = conj(c) * a
        const double zr = (double)c.x * a.x + (double)c.y * a.y;
        const double zi = (double)c.x * a.y - (double)c.y * a.x;
        double re;
        switch (yk) {
            case 0: re = zr; break;
            case 1: re = -zi; break;
            case 2: re = -zr; break;
            default: re = zi; break;
        }
        if (__popcll(i & zmask) & 1) re = -re;
        acc += 2.0 * re;
    }
    __shared__ double red[RED_THREADS / 32];
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x += red[k];
        partials[(size_t)b * nblk + blockIdx.x] = x;
    }
}

// out[b * nobs + o] = sum_k partials[(b * nblk + k) * nobs + o], fixed order
__global__ void finalize_kernel(const double* partials, int64_t B, int nblk, int nobs, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * nobs) return;
    const int64_t b = i / nobs, o = i - b * nobs;
    double s = 0;
    for (int k = 0; k < nblk; ++k) s += partials[((size_t)b * nblk + k) * nobs + o];
    out[i] = s;
}

// ---------------------------------------------------------------- utilities
template <typename R>
__global__ void set_basis_kernel(typename CT<R>::T* psi, int N, int64_t B, uint64_t index) {
    const int64_t len = (int64_t)1 << N;
    const uint64_t total = (uint64_t)B * len;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        typename CT<R>::T v = czero(psi[0]);
        if ((i & (uint64_t)(len - 1)) == index) v.x = (R)1;
        psi[i] = v;
    }
}

template <typename R>
__global__ void scale_kernel(typename CT<R>::T* psi, int N, int64_t B, const double* per_state,
                             double scalar) {
    const int64_t len = (int64_t)1 << N;
    const uint64_t total = (uint64_t)B * len;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double f = per_state ? per_state[i >> N] * scalar : scalar;
        psi[i] = cscale(psi[i], (R)f);
    }
}

template <typename RD, typename RS>
__global__ void convert_kernel(typename CT<RD>::T* dst, const typename CT<RS>::T* src, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        typename CT<RD>::T v;
        v.x = (RD)src[i].x;
        v.y = (RD)src[i].y;
        dst[i] = v;
    }
}

// ===================================================================== launch
static int grid_for(const smoq_state* st, uint64_t work, int threads) {
    const int sms = st->ctx->num_sms;
    uint64_t want = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)sms * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

cudaError_t launch_direct_op(smoq_state* st, const DevOp& op) {
    smoq_ctx* ctx = st->ctx;
    const uint64_t work = ((uint64_t)1 << st->N) * st->batch;
    const int grid = grid_for(st, work / 2, 256);
    if (st->dtype == SMOQ_C64)
        direct_op_kernel<float><<<grid, 256, 0, ctx->stream>>>((float2*)st->ptr, st->N, st->batch, op);
    else
        direct_op_kernel<double><<<grid, 256, 0, ctx->stream>>>((double2*)st->ptr, st->N, st->batch, op);
    ctx->launches++;
    return cudaGetLastError();
}

size_t tile_max_smem(int amp_bytes, int T) { return (size_t)amp_bytes << T; }

// Opt the tile kernels in to large dynamic shared memory and record their
// occupancy for every tile width, once per context (never during capture).
template <typename R, bool EPI>
static cudaError_t init_tile_t(smoq_ctx* ctx, int dt) {
    auto kern = tile_pass_kernel<R, EPI>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tile_max_smem((int)sizeof(typename CT<R>::T), dt == 0 ? 14 : 13));
    if (e != cudaSuccess) return e;
    for (int T = 1; T <= (dt == 0 ? 14 : 13); ++T) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TILE_THREADS,
                                                          tile_max_smem((int)sizeof(typename CT<R>::T), T));
        if (e != cudaSuccess) return e;
        ctx->tile_occ[dt][EPI ? 1 : 0][T] = per_sm < 1 ? 1 : per_sm;
    }
    return cudaSuccess;
}

cudaError_t tile_kernels_init(smoq_ctx* ctx) {
    cudaError_t e;
    if ((e = init_tile_t<float, false>(ctx, 0)) != cudaSuccess) return e;
    if ((e = init_tile_t<float, true>(ctx, 0)) != cudaSuccess) return e;
    if ((e = init_tile_t<double, false>(ctx, 1)) != cudaSuccess) return e;
    return init_tile_t<double, true>(ctx, 1);
}

template <typename R, bool EPI>
static cudaError_t launch_tile_t(smoq_ctx* ctx, const TileArgs& a, size_t smem, int dt) {
    int per_sm = ctx->tile_occ[dt][EPI ? 1 : 0][a.g.T];
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)ctx->num_sms * per_sm;
    if (grid > a.ntiles) grid = a.ntiles;
    tile_pass_kernel<R, EPI><<<(unsigned)grid, TILE_THREADS, smem, ctx->stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_tile_pass(smoq_ctx* ctx, smoq_state* st, const Pass& p, const DevOp* d_ops,
                             const Epilogue* ep) {
    TileArgs a;
    a.psi = st->ptr;
    a.state_len = (int64_t)1 << st->N;
    a.tiles_per_state = (int64_t)1 << (st->N - p.g.T);
    a.ntiles = a.tiles_per_state * st->batch;
    a.ops = d_ops;
    a.nops = (int32_t)p.ops.size();
    a.err = ctx->d_err;
    a.g = p.g;
    if (ep) a.ep = *ep;
    else { a.ep.partials = nullptr; a.ep.npop = 0; }
    const size_t smem = tile_max_smem((int)st->amp_bytes(), p.g.T);
    cudaError_t e;
    const bool epi = ep && ep->partials;
    if (p.jit) {
        e = launch_jit(ctx, a, p.jit, epi, p.rtc ? p.coefs.data() : nullptr);
        ctx->launches++;
        return e;
    }
    if (p.staged) {
        e = launch_stage(ctx, a, st->dtype, epi);
        ctx->launches++;
        return e;
    }
    if (st->dtype == SMOQ_C64)
        e = epi ? launch_tile_t<float, true>(ctx, a, smem, 0) : launch_tile_t<float, false>(ctx, a, smem, 0);
    else
        e = epi ? launch_tile_t<double, true>(ctx, a, smem, 1) : launch_tile_t<double, false>(ctx, a, smem, 1);
    ctx->launches++;
    return e;
}

static int red_blocks(const smoq_state* st) {
    const int64_t len = (int64_t)1 << st->N;
    int64_t want = (len + RED_THREADS * 8 - 1) / (RED_THREADS * 8);
    int64_t cap = (int64_t)st->ctx->num_sms * 4;
    if (st->batch > 1) {
        cap = (cap + st->batch - 1) / st->batch;
        if (cap < 1) cap = 1;
    }
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

size_t diag_reduce_scratch_doubles(smoq_state* st, int nobs) {
    return (size_t)red_blocks(st) * st->batch * (nobs > 0 ? nobs : 1);
}

cudaError_t launch_diag_reduce(smoq_ctx* ctx, smoq_state* st, const uint64_t* zmasks, int nobs,
                               double* d_out) {
    const int nblk = red_blocks(st);
    ZMasks zm;
    for (int o = 0; o < MAX_DIAG_OBS; ++o) zm.m[o] = o < nobs ? zmasks[o] : 0;
    dim3 grid(nblk, st->batch);
    if (st->N >= 4) {
        if (st->dtype == SMOQ_C64)
            diag_reduce_wht_kernel<float><<<grid, RED_THREADS, 0, ctx->stream>>>((const float2*)st->ptr, st->N,
                                                                                  zm, nobs, ctx->d_scratch);
        else
            diag_reduce_wht_kernel<double><<<grid, RED_THREADS, 0, ctx->stream>>>((const double2*)st->ptr,
                                                                                   st->N, zm, nobs, ctx->d_scratch);
    } else if (st->dtype == SMOQ_C64) {
        diag_reduce_kernel<float><<<grid, RED_THREADS, 0, ctx->stream>>>((const float2*)st->ptr, st->N, zm,
                                                                          nobs, ctx->d_scratch);
    } else {
        diag_reduce_kernel<double><<<grid, RED_THREADS, 0, ctx->stream>>>((const double2*)st->ptr, st->N,
                                                                           zm, nobs, ctx->d_scratch);
    }
    const int64_t outs = (int64_t)st->batch * nobs;
    finalize_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_scratch, st->batch,
                                                                             nblk, nobs, d_out);
    ctx->launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_pauli_reduce(smoq_ctx* ctx, smoq_state* st, uint64_t xmask, uint64_t zmask, int ny,
                                double* d_out) {
    const int nblk = red_blocks(st);
    dim3 grid(nblk, st->batch);
    if (st->dtype == SMOQ_C64)
        pauli_reduce_kernel<float><<<grid, RED_THREADS, 0, ctx->stream>>>((const float2*)st->ptr, st->N,
                                                                           xmask, zmask, ny, ctx->d_scratch);
    else
        pauli_reduce_kernel<double><<<grid, RED_THREADS, 0, ctx->stream>>>(
            (const double2*)st->ptr, st->N, xmask, zmask, ny, ctx->d_scratch);
    finalize_kernel<<<(unsigned)((st->batch + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_scratch, st->batch,
                                                                                   nblk, 1, d_out);
    ctx->launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_set_basis(smoq_state* st, uint64_t index) {
    const uint64_t work = ((uint64_t)1 << st->N) * st->batch;
    const int grid = grid_for(st, work, 256);
    if (st->dtype == SMOQ_C64)
        set_basis_kernel<float><<<grid, 256, 0, st->ctx->stream>>>((float2*)st->ptr, st->N, st->batch, index);
    else
        set_basis_kernel<double><<<grid, 256, 0, st->ctx->stream>>>((double2*)st->ptr, st->N, st->batch,
                                                                     index);
    st->ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_scale(smoq_state* st, const double* d_scale, double scalar) {
    const uint64_t work = ((uint64_t)1 << st->N) * st->batch;
    const int grid = grid_for(st, work, 256);
    if (st->dtype == SMOQ_C64)
        scale_kernel<float><<<grid, 256, 0, st->ctx->stream>>>((float2*)st->ptr, st->N, st->batch, d_scale,
                                                                scalar);
    else
        scale_kernel<double><<<grid, 256, 0, st->ctx->stream>>>((double2*)st->ptr, st->N, st->batch,
                                                                 d_scale, scalar);
    st->ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_convert(smoq_state* dst, smoq_state* src) {
    const uint64_t n = ((uint64_t)1 << src->N) * src->batch;
    const int grid = grid_for(src, n, 256);
    cudaStream_t s = src->ctx->stream;
    if (dst->dtype == SMOQ_C64 && src->dtype == SMOQ_C128)
        convert_kernel<float, double><<<grid, 256, 0, s>>>((float2*)dst->ptr, (const double2*)src->ptr, n);
    else if (dst->dtype == SMOQ_C128 && src->dtype == SMOQ_C64)
        convert_kernel<double, float><<<grid, 256, 0, s>>>((double2*)dst->ptr, (const float2*)src->ptr, n);
    else
        return cudaMemcpyAsync(dst->ptr, src->ptr, src->bytes(), cudaMemcpyDeviceToDevice, s);
    src->ctx->launches++;
    return cudaGetLastError();
}

}  // namespace smoq

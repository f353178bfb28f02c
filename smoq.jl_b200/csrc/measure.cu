// measure.cu -- Born-rule sampling and projective Z measurements.
//
// Replaces sample_from_probabilities / projective_measurement_all! /
// _measure_z_single! (utils/cpu/cpuQuantumStateMeasurements.jl:203,484,224)
// and the benchmark's cumsum + searchsortedfirst shot loop
// (SmoQ.jl_benchmarks/benchmark_random_circuit_sampling/run_benchmark_smoq_Float64.jl:424-435).
//
// Uniforms: Philox4x32-10 (the same generator as the MCWF driver), key =
// seed, counter = (shot_lo, shot_hi, stream_lo, stream_hi) with stream =
// stream0 + state index; u = 53-bit uniform from the first two words.  An
// index is the first i whose cumulative |psi|^2 reaches u (the inverse CDF of
// the reference), the last index when rounding leaves u above the total.
//
// Sampling is two-level so that a shot reads O(log 2^N + 256) values:
//   1. chunk_sum_kernel: FP64 |psi|^2 sums of 256-amplitude chunks;
//   2. chunk_scan_kernel: per state, inclusive prefix sums of the chunk sums
//      (one CTA per state, blocked: each thread a contiguous range);
//   3. sample_kernel: one warp per shot -- binary search over the chunk
//      prefixes, then a warp scan inside the chunk.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

namespace smoq {

constexpr int SAMPLE_CHUNK = 256;  // amplitudes per first-level chunk (8 per lane)

__device__ __forceinline__ double shot_uniform(uint64_t seed, uint64_t shot, uint64_t stream) {
    uint32_t c[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
    philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return u01_53(c[0], c[1]);
}

// sums[c] = sum of |psi|^2 over chunk c (chunks of all states, state-major)
template <typename R>
__global__ void __launch_bounds__(256) chunk_sum_kernel(const typename CT<R>::T* psi, int64_t nchunks,
                                                        double* sums) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nchunks; c += warps) {
        const typename CT<R>::T* p = psi + c * SAMPLE_CHUNK + lane * 8;
        double s = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += cabs2d(p[k]);
        for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
        if (lane == 0) sums[c] = s;
    }
}

// in place: sums of state b (per_state chunks) -> inclusive prefix sums
__global__ void __launch_bounds__(1024) chunk_scan_kernel(double* sums, int64_t per_state) {
    __shared__ double part[1024];
    double* s = sums + (int64_t)blockIdx.x * per_state;
    const int64_t per_thread = (per_state + blockDim.x - 1) / blockDim.x;
    int64_t lo = (int64_t)threadIdx.x * per_thread, hi = lo + per_thread;
    if (lo > per_state) lo = per_state;
    if (hi > per_state) hi = per_state;
    double t = 0;
    for (int64_t i = lo; i < hi; ++i) t += s[i];
    part[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive prefix of the thread totals, in order
        double run = 0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
            const double x = part[k];
            part[k] = run;
            run += x;
        }
    }
    __syncthreads();
    double run = part[threadIdx.x];
    for (int64_t i = lo; i < hi; ++i) {
        run += s[i];
        s[i] = run;
    }
}

// one warp per (state, shot): out[b * nshots + shot] = sampled index
template <typename R>
__global__ void __launch_bounds__(256) sample_kernel(const typename CT<R>::T* psi, int N, int64_t B, int64_t nshots,
                                                     const double* prefix, uint64_t seed, uint64_t stream0,
                                                     int64_t* out) {
    const int lane = threadIdx.x & 31;
    const int64_t per_state = ((int64_t)1 << N) / SAMPLE_CHUNK;
    const int64_t total = B * nshots;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total; w += warps) {
        const int64_t b = w / nshots, shot = w - b * nshots;
        const double u = shot_uniform(seed, (uint64_t)shot, stream0 + (uint64_t)b);
        const double* pf = prefix + b * per_state;
        // first chunk whose inclusive prefix reaches u (else the last chunk)
        int64_t lo = 0, hi = per_state - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (pf[mid] >= u) hi = mid;
            else lo = mid + 1;
        }
        const int64_t c = lo;
        const double base = c > 0 ? pf[c - 1] : 0.0;
        const typename CT<R>::T* p = psi + b * ((int64_t)1 << N) + c * SAMPLE_CHUNK + lane * 8;
        double v[8], ls = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[k] = cabs2d(p[k]);
            ls += v[k];
        }
        double incl = ls;  // inclusive warp scan of the lane sums
        for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        const unsigned hit = __ballot_sync(0xffffffffu, base + incl >= u);
        int64_t idx = c * SAMPLE_CHUNK + SAMPLE_CHUNK - 1;  // rounding fallback: chunk end
        if (hit) {
            const int L = __ffs(hit) - 1;
            if (lane == L) {
                double run = base + incl - ls;
                int j = 7;
                for (int k = 0; k < 8; ++k) {
                    run += v[k];
                    if (run >= u) {
                        j = k;
                        break;
                    }
                }
                idx = c * SAMPLE_CHUNK + L * 8 + j;
            }
            idx = __shfl_sync(0xffffffffu, idx, L);
        }
        if (lane == 0) out[w] = idx;
    }
}

// collapse state b onto basis index idx[b]
template <typename R>
__global__ void collapse_all_kernel(typename CT<R>::T* psi, int N, int64_t B, const int64_t* idx) {
    const int64_t len = (int64_t)1 << N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B * len; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> N;
        typename CT<R>::T z = czero(psi[0]);
        if ((i & (len - 1)) == idx[b]) z.x = (R)1;
        psi[i] = z;
    }
}

// collapse qubit q of state b onto outcome[b], scaling the kept half by scale[b]
template <typename R>
__global__ void collapse_qubit_kernel(typename CT<R>::T* psi, int N, int64_t B, int q, const int32_t* outcome,
                                      const double* scale) {
    const int64_t len = (int64_t)1 << N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B * len; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> N;
        const int bit = (int)((i >> q) & 1);
        psi[i] = bit == outcome[b] ? cscale(psi[i], (R)scale[b]) : czero(psi[i]);
    }
}

// outcome[b] = (u < P0[b]) ? 0 : 1, scale[b] = 1/sqrt(P(outcome)); z[2b] = norm^2,
// z[2b + 1] = <Z_q> (unnormalised), so P(1) = (z[2b] - z[2b + 1]) / 2
__global__ void decide_qubit_kernel(int64_t B, const double* z, uint64_t seed, uint64_t stream0, int32_t* outcome,
                                    double* scale) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const double u = shot_uniform(seed, 0, stream0 + (uint64_t)b);
    const double P1 = 0.5 * (z[2 * b] - z[2 * b + 1]), P0 = z[2 * b] - P1;
    const int o = u < P0 ? 0 : 1;
    outcome[b] = o;
    const double keep = o ? P1 : P0;
    scale[b] = keep > 0 ? 1.0 / sqrt(keep) : 0.0;
}

static int grid_for_items(const smoq_ctx* ctx, int64_t items, int per_block) {
    int64_t g = (items + per_block - 1) / per_block;
    const int64_t cap = (int64_t)ctx->num_sms * 8;
    return (int)std::max<int64_t>(1, std::min(g, cap));
}

}  // namespace smoq

using namespace smoq;

smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);
smoq_status smoq_internal_zreduce(smoq_ctx* ctx, smoq_state* st, const uint64_t* zmasks, int nobs, double* out);

#define MCK(call)                                                         \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return smoq_internal_cuda(ctx, e_, #call); \
    } while (0)

namespace {
// device buffer freed on the ctx stream when the scope ends
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s;
    explicit DevBuf(cudaStream_t st) : s(st) {}
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

smoq_status sample_into(smoq_state* st, int64_t nshots, uint64_t seed, uint64_t stream0, int64_t* d_out) {
    smoq_ctx* ctx = st->ctx;
    const int64_t per_state = ((int64_t)1 << st->N) / SAMPLE_CHUNK;
    const int64_t nchunks = per_state * st->batch;
    DevBuf pre(ctx->stream);
    MCK(cudaMallocAsync(&pre.p, (size_t)nchunks * sizeof(double), ctx->stream));
    double* prefix = (double*)pre.p;
    const int g1 = grid_for_items(ctx, nchunks, 8);
    if (st->dtype == SMOQ_C64)
        chunk_sum_kernel<float><<<g1, 256, 0, ctx->stream>>>((const float2*)st->ptr, nchunks, prefix);
    else
        chunk_sum_kernel<double><<<g1, 256, 0, ctx->stream>>>((const double2*)st->ptr, nchunks, prefix);
    chunk_scan_kernel<<<(unsigned)st->batch, 1024, 0, ctx->stream>>>(prefix, per_state);
    const int g3 = grid_for_items(ctx, st->batch * nshots, 8);
    if (st->dtype == SMOQ_C64)
        sample_kernel<float><<<g3, 256, 0, ctx->stream>>>((const float2*)st->ptr, st->N, st->batch, nshots, prefix,
                                                          seed, stream0, d_out);
    else
        sample_kernel<double><<<g3, 256, 0, ctx->stream>>>((const double2*)st->ptr, st->N, st->batch, nshots,
                                                           prefix, seed, stream0, d_out);
    ctx->launches += 3;
    MCK(cudaGetLastError());
    return SMOQ_OK;
}

smoq_status check_measure_state(smoq_state* st) {
    if (!st || !st->ctx) return SMOQ_ERR_BADINPUT;
    if (st->N < 8)
        return smoq_internal_fail(st->ctx, SMOQ_ERR_BADINPUT, "sampling needs N >= 8 (256-amplitude chunks)");
    return SMOQ_OK;
}
}  // namespace

extern "C" {

smoq_status smoq_sample(smoq_state* st, long long nshots, unsigned long long seed, unsigned long long stream,
                        long long* out) {
    if (smoq_status s = check_measure_state(st)) return s;
    smoq_ctx* ctx = st->ctx;
    if (nshots < 0 || (nshots > 0 && !out)) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad shot count");
    if (nshots == 0) return SMOQ_OK;
    DevBuf d(ctx->stream);
    const size_t bytes = (size_t)st->batch * (size_t)nshots * sizeof(int64_t);
    MCK(cudaMallocAsync(&d.p, bytes, ctx->stream));
    if (smoq_status s = sample_into(st, nshots, seed, stream, (int64_t*)d.p)) return s;
    MCK(cudaMemcpyAsync(out, d.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    MCK(cudaStreamSynchronize(ctx->stream));
    return SMOQ_OK;
}

smoq_status smoq_measure_all(smoq_state* st, unsigned long long seed, unsigned long long stream, long long* outcome) {
    if (smoq_status s = check_measure_state(st)) return s;
    smoq_ctx* ctx = st->ctx;
    if (!outcome) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "null outcome");
    DevBuf d(ctx->stream);
    MCK(cudaMallocAsync(&d.p, (size_t)st->batch * sizeof(int64_t), ctx->stream));
    if (smoq_status s = sample_into(st, 1, seed, stream, (int64_t*)d.p)) return s;
    const int g = grid_for_items(ctx, ((int64_t)1 << st->N) * st->batch, 256);
    if (st->dtype == SMOQ_C64)
        collapse_all_kernel<float><<<g, 256, 0, ctx->stream>>>((float2*)st->ptr, st->N, st->batch, (const int64_t*)d.p);
    else
        collapse_all_kernel<double><<<g, 256, 0, ctx->stream>>>((double2*)st->ptr, st->N, st->batch,
                                                                (const int64_t*)d.p);
    ctx->launches++;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(outcome, d.p, (size_t)st->batch * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    MCK(cudaStreamSynchronize(ctx->stream));
    return SMOQ_OK;
}

smoq_status smoq_measure_qubit(smoq_state* st, int q, unsigned long long seed, unsigned long long stream,
                               int* outcome) {
    if (!st || !st->ctx) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = st->ctx;
    if (q < 0 || q >= st->N) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "measure_qubit: qubit out of range");
    if (!outcome) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "null outcome");
    const int64_t B = st->batch;
    DevBuf d(ctx->stream);
    const size_t need = (size_t)B * (3 * sizeof(double) + sizeof(int32_t));
    MCK(cudaMallocAsync(&d.p, need, ctx->stream));
    double* d_z = (double*)d.p;      // [B][2]: norm^2 and <Z_q>, FP64 Z-string sums
    double* d_scale = d_z + 2 * B;
    int32_t* d_out = (int32_t*)(d_scale + B);
    const uint64_t masks[2] = {0ull, 1ull << q};
    if (smoq_status s = smoq_internal_zreduce(ctx, st, masks, 2, d_z)) return s;
    decide_qubit_kernel<<<(unsigned)((B + 127) / 128), 128, 0, ctx->stream>>>(B, d_z, seed, stream, d_out, d_scale);
    const int g = grid_for_items(ctx, ((int64_t)1 << st->N) * B, 256);
    if (st->dtype == SMOQ_C64)
        collapse_qubit_kernel<float><<<g, 256, 0, ctx->stream>>>((float2*)st->ptr, st->N, B, q, d_out, d_scale);
    else
        collapse_qubit_kernel<double><<<g, 256, 0, ctx->stream>>>((double2*)st->ptr, st->N, B, q, d_out, d_scale);
    ctx->launches += 2;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(outcome, d_out, (size_t)B * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    MCK(cudaStreamSynchronize(ctx->stream));
    return SMOQ_OK;
}

}  // extern "C"

// dm.cu -- density-matrix evolution on the state-vector engine.
//
// A density matrix rho of N qubits is stored as Julia stores Matrix{ComplexF64}:
// column-major, rho[i, j] at i + j 2^N.  Read as a state vector of 2N qubits,
// bits 0..N-1 are the row index and bits N..2N-1 the column index, and every
// linear map on rho is a gate program on that vector:
//   * U rho U^dag (evolve_trotter_rho_cpu!, cpuQuantumChannelUnitaryEvolutionTrotter.jl:266-285):
//     U on the row qubits q, conj(U) on the column qubits q + N;
//   * one Euler step of a jump's dissipator, rho += gamma dt (L rho L^dag -
//     {L^dag L, rho} / 2) (_apply_dissipator_dm!, cpuQuantumChannelLindbladianEvolution.jl:377-460):
//     a 4x4 (not unitary) map on the pair (row bit q, column bit q), local
//     index m = row bit + 2 column bit.
// So a DM step is an ordinary Trotter plan on 2N qubits -- fused, tiled and
// (for complex64) compiled like any other -- and N up to 16 runs on one GPU
// (2^32 amplitudes).  Observables <Z...> read the diagonal: dm_zreduce_kernel.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <complex>
#include <cstring>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

namespace smoq {

constexpr int DM_MAX_OBS = 32;
struct DmMasks {
    uint64_t m[DM_MAX_OBS];
};

// partials[b][blk][o] = sum over this block's diagonal entries of Re rho_ii (-1)^popc(i & m_o)
template <typename R>
__global__ void __launch_bounds__(256) dm_zreduce_kernel(const typename CT<R>::T* rho, int N, DmMasks zm, int nobs,
                                                         double* partials) {
    const int64_t dim = (int64_t)1 << N;
    const int64_t b = blockIdx.y;
    const typename CT<R>::T* s = rho + b * dim * dim;
    double acc[DM_MAX_OBS];
#pragma unroll
    for (int o = 0; o < DM_MAX_OBS; ++o) acc[o] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += (int64_t)gridDim.x * blockDim.x) {
        const double p = (double)s[i + i * dim].x;
#pragma unroll
        for (int o = 0; o < DM_MAX_OBS; ++o)
            if (o < nobs) acc[o] += (__popcll((uint64_t)i & zm.m[o]) & 1) ? -p : p;
    }
    __shared__ double red[8][DM_MAX_OBS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < DM_MAX_OBS; ++o) {
        if (o >= nobs) continue;
        double x = acc[o];
        for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
        if (lane == 0) red[w][o] = x;
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double x = 0;
        for (int k = 0; k < 8; ++k) x += red[k][threadIdx.x];
        partials[((size_t)b * gridDim.x + blockIdx.x) * nobs + threadIdx.x] = x;
    }
}

}  // namespace smoq

using namespace smoq;

smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);

namespace {
using cdd = std::complex<double>;

// 4x4 superoperator of one jump's Euler dissipator step, local index m = r + 2c
// (r = row bit, c = column bit of the jump's qubit), written column-major
// interleaved as a smoq_trotter_gate on (q, q + N)
void dissipator_gate(const smoq_jump_op& j, int N, double dt, smoq_trotter_gate& g) {
    cdd L[2][2] = {{0, 0}, {0, 0}};
    switch (j.type) {
        case 0: L[0][1] = 1; break;              // sigma- = |0><1|
        case 1: L[1][0] = 1; break;              // sigma+ = |1><0|
        case 2: L[0][0] = 1; L[1][1] = -1; break;  // sigma_z
        default: L[0][1] = 1; L[1][0] = 1; break;  // sigma_x
    }
    cdd LL[2][2];  // L^dag L
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            LL[a][b] = 0;
            for (int k = 0; k < 2; ++k) LL[a][b] += std::conj(L[k][a]) * L[k][b];
        }
    const double f = j.gamma * dt;
    std::memset(&g, 0, sizeof(g));
    g.nq = 2;
    g.q[0] = j.qubit;
    g.q[1] = j.qubit + N;
    for (int mo = 0; mo < 4; ++mo)
        for (int mi = 0; mi < 4; ++mi) {
            const int ro = mo & 1, co = mo >> 1, ri = mi & 1, ci = mi >> 1;
            cdd s = (mo == mi) ? 1.0 : 0.0;
            s += f * (L[ro][ri] * std::conj(L[co][ci])                // L rho L^dag
                      - 0.5 * (co == ci ? LL[ro][ri] : 0.0)          // L^dag L rho / 2
                      - 0.5 * (ro == ri ? LL[ci][co] : 0.0));        // rho L^dag L / 2
            g.U[2 * (mi * 4 + mo)] = s.real();                       // column-major
            g.U[2 * (mi * 4 + mo) + 1] = s.imag();
        }
}
}  // namespace

extern "C" {

smoq_status smoq_dm_plan_create(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_trotter_gate* gates, int ngates,
                                const smoq_jump_op* jumps, int njumps, double dt, smoq_plan** out) {
    if (!ctx || !out) return SMOQ_ERR_BADINPUT;
    if (N < 1 || N > 16) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "density matrices: N must be 1..16");
    if (ngates < 0 || (ngates > 0 && !gates) || njumps < 0 || (njumps > 0 && !jumps))
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad gate or jump list");
    std::vector<smoq_trotter_gate> all;
    all.reserve(2 * ngates + njumps);
    for (int t = 0; t < ngates; ++t) {
        const smoq_trotter_gate& u = gates[t];
        if (u.nq < 1 || u.nq > 2) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "gates act on 1 or 2 qubits");
        for (int k = 0; k < u.nq; ++k)
            if (u.q[k] < 0 || u.q[k] >= N) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "gate qubit out of range");
        all.push_back(u);          // U on the row index
        smoq_trotter_gate c = u;   // conj(U) on the column index
        for (int k = 0; k < u.nq; ++k) c.q[k] = u.q[k] + N;
        for (int k = 1; k < 32; k += 2) c.U[k] = -c.U[k];
        all.push_back(c);
    }
    for (int t = 0; t < njumps; ++t) {
        if (jumps[t].qubit < 0 || jumps[t].qubit >= N || jumps[t].type < 0 || jumps[t].type > 3 || jumps[t].gamma < 0)
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad jump operator");
        smoq_trotter_gate g;
        dissipator_gate(jumps[t], N, dt, g);
        all.push_back(g);
    }
    return smoq_trotter_plan_create(ctx, 2 * N, dtype, all.data(), (int)all.size(), 1, out);
}

smoq_status smoq_dm_expect_zstrings(smoq_state* rho, int N, const uint64_t* zmasks, int nobs, double* out) {
    if (!rho || !rho->ctx) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = rho->ctx;
    if (rho->N != 2 * N) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "density matrix state must have 2N qubits");
    if (nobs < 1 || nobs > DM_MAX_OBS || !zmasks || !out)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "1..32 Z-string masks and an output are needed");
    DmMasks zm;
    for (int o = 0; o < DM_MAX_OBS; ++o) zm.m[o] = o < nobs ? zmasks[o] : 0;
    const int64_t dim = (int64_t)1 << N;
    const int nblk = (int)std::min<int64_t>((dim + 255) / 256, (int64_t)ctx->num_sms * 2);
    const int64_t B = rho->batch;
    double* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, (size_t)(B * nblk * nobs) * sizeof(double), ctx->stream);
    if (e != cudaSuccess) return smoq_internal_cuda(ctx, e, "dm_expect_zstrings");
    dim3 grid(nblk, (unsigned)B);
    if (rho->dtype == SMOQ_C64)
        dm_zreduce_kernel<float><<<grid, 256, 0, ctx->stream>>>((const float2*)rho->ptr, N, zm, nobs, buf);
    else
        dm_zreduce_kernel<double><<<grid, 256, 0, ctx->stream>>>((const double2*)rho->ptr, N, zm, nobs, buf);
    ctx->launches++;
    e = cudaGetLastError();
    std::vector<double> part((size_t)(B * nblk * nobs));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(part.data(), buf, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(buf, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return smoq_internal_cuda(ctx, e, "dm_expect_zstrings");
    for (int64_t b = 0; b < B; ++b)
        for (int o = 0; o < nobs; ++o) {
            double s = 0;
            for (int k = 0; k < nblk; ++k) s += part[((size_t)b * nblk + k) * nobs + o];
            out[b * nobs + o] = s;
        }
    return SMOQ_OK;
}

}  // extern "C"

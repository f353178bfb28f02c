// qrc.cu -- quantum reservoir computing: the bitwise MCWF trajectory loop.
//
// Replaces _run_traj_loop_bitwise! and the bitwise run_mcwf_simulation
// (utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:451-530, :531-590)
// with encode_input_ry_psi! and qrc_reset_psi! (utils/cpu/cpuQRCstep.jl:96,
// :332).  Per input k of the series, every trajectory
//   A. encodes the window of inputs as |psi_in> = prod_q Ry(pi u_q)|0> on the
//      L input qubits,
//   B. measures one rail (rail 1: the input rail = low L bits; rail 2: the
//      reservoir = high L bits) with the inverse-CDF draw r, keeps the
//      normalised conditional state of the other rail and writes
//      |psi_in> (x) |phi> (psi_in on the low bits),
//   C. runs n_substeps Trotter steps,
//   D. measures the ladder's observable set (X, Y, Z per qubit; XX, YY, ZZ per
//      rail bond, then per rung) and adds it to the trajectory sums.
//
// B200 layout: the whole state of a trajectory lives in SHARED MEMORY for the
// whole series (2^N amplitudes: 128 KB at N = 14 complex64, 64 KB at N = 12
// complex128), one CTA per trajectory, persistent over trajectories; HBM
// sees only the initial state and the feature sums.  The Trotter steps are
// the planner's fused op program for a tile that spans the whole state.
//
// Randomness: r = 53-bit uniform of Philox4x32-10, key = seed, counter =
// (step, trajectory id) -- the draw of smoq_sample for shot = step, stream =
// trajectory id -- so the oracle can replay every trajectory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

namespace smoq {

// one observable group: q2 < 0 -> (X, Y, Z) of q1 at out..out+2; else (XX, YY, ZZ)
struct QrcObs {
    int32_t q1, q2, out, pad;
};

struct QrcArgs {
    const void* psi0;      // 2^N amplitudes (the state's precision)
    const double* enc;     // [T][L][2]: cos, sin of the half angles of the input window
    const DevOp* ops;      // one input's evolution, planned on a whole-state tile
    const QrcObs* obs;
    double* X;             // [T][n_ops] sums over trajectories
    double* X_traj;        // [n_traj][T][n_ops] or nullptr
    int64_t n_traj;
    uint64_t seed, traj_offset;
    int32_t nops, nobs, n_ops;
    int32_t N, L, T, protocol;
};

constexpr int kQrcThreads = 256;

// the 53-bit uniform of counter (shot, stream) under key seed (Philox4x32-10)
__device__ __forceinline__ double qrc_uniform(uint64_t seed, uint64_t shot, uint64_t stream) {
    uint32_t c[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const uint64_t a = c[0] >> 5, b = c[1] >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

// one evolution op on the whole state in shared memory (qubit t at bit lb[t])
template <typename R>
__device__ __forceinline__ void qrc_apply(const DevOp& op, typename CT<R>::T* psi, int N, typename CT<R>::T* dco) {
    using C = typename CT<R>::T;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    if (op.kind == OPK_DIAG) {
        if (tid < 16) dco[tid] = coef<R>(op, (int)tid);
        __syncthreads();
        int sh[4] = {0, 0, 0, 0}, in = 0;
        for (int t = 0; t < op.nq; ++t) sh[t] = op.lb[t], in |= 1 << t;
        for (uint32_t j = tid; j < (1u << N); j += nthr) {
            int m = 0;
#pragma unroll
            for (int t = 0; t < 4; ++t) m |= (int)((j >> sh[t]) & (uint32_t)(in >> t) & 1u) << t;
            psi[j] = cmul(dco[m], psi[j]);
        }
    } else {
        sweep_op<R, uint32_t>(op, psi, N, op.lb, tid, nthr);
    }
}

template <typename R>
__global__ void __launch_bounds__(kQrcThreads) qrc_traj_kernel(const QrcArgs A) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t dim = 1u << A.N, d = 1u << A.L;
    C* psi = reinterpret_cast<C*>(sm);
    C* phi = psi + dim;
    double* pin = reinterpret_cast<double*>(phi + d);  // encoded input amplitudes (real)
    double* prob = pin + d;                            // outcome probabilities
    double* part = prob + d;                           // one partial per thread
    double* red = part + kQrcThreads;                  // [warps][n_ops]
    __shared__ C dco[16];
    __shared__ int s_out;
    __shared__ double s_inv;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    const C* p0 = reinterpret_cast<const C*>(A.psi0);
    for (int64_t t = blockIdx.x; t < A.n_traj; t += gridDim.x) {
        for (uint32_t a = tid; a < dim; a += blockDim.x) psi[a] = p0[a];
        const uint64_t traj = A.traj_offset + (uint64_t)t;
        for (int k = 0; k < A.T; ++k) {
            // A. the encoded input, prod_q (bit q ? sin : cos)
            const double* e = A.enc + (size_t)k * A.L * 2;
            for (uint32_t i = tid; i < d; i += blockDim.x) {
                double v = 1.0;
                for (int q = 0; q < A.L; ++q) v *= ((i >> q) & 1) ? e[2 * q + 1] : e[2 * q];
                pin[i] = v;
            }
            __syncthreads();
            // B. probabilities of the measured rail: x = the measured index, y = the kept one
            {
                const uint32_t x = (uint32_t)tid & (d - 1), np = (uint32_t)blockDim.x / d;
                double s = 0;
                for (uint32_t y = (uint32_t)tid / d; y < d; y += np) {
                    const C v = psi[A.protocol == 1 ? x + d * y : y + d * x];
                    s += (double)v.x * v.x + (double)v.y * v.y;
                }
                part[tid] = s;
            }
            __syncthreads();
            for (uint32_t x = tid; x < d; x += blockDim.x) {
                double s = 0;
                for (uint32_t p = 0; p < (uint32_t)blockDim.x / d; ++p) s += part[x + d * p];
                prob[x] = s;
            }
            __syncthreads();
            if (tid == 0) {
                double total = 0;
                for (uint32_t x = 0; x < d; ++x) total += prob[x];
                const double r = qrc_uniform(A.seed, (uint64_t)k, traj);
                int outcome = 0;  // (no crossing: the first outcome, as the reference)
                double cum = 0;
                for (uint32_t x = 0; x < d; ++x) {
                    cum += prob[x] / total;
                    if (r <= cum) {
                        outcome = (int)x;
                        break;
                    }
                }
                const double nrm = sqrt(prob[outcome]);
                s_out = outcome;
                s_inv = nrm > 1e-12 ? 1.0 / nrm : 0.0;  // 0: the reset falls back to |0>
            }
            __syncthreads();
            const uint32_t o = (uint32_t)s_out;
            const double inv = s_inv;
            for (uint32_t y = tid; y < d; y += blockDim.x) {
                C v;
                if (inv > 0) {
                    const C w = psi[A.protocol == 1 ? o + d * y : y + d * o];
                    v.x = (R)((double)w.x * inv);
                    v.y = (R)((double)w.y * inv);
                } else {
                    v.x = (R)(y == 0 ? 1 : 0);
                    v.y = (R)0;
                }
                phi[y] = v;
            }
            __syncthreads();
            for (uint32_t a = tid; a < dim; a += blockDim.x) {
                const C v = phi[a >> A.L];
                const R w = (R)pin[a & (d - 1)];
                C z;
                z.x = w * v.x;
                z.y = w * v.y;
                psi[a] = z;
            }
            __syncthreads();
            // C. n_substeps Trotter steps
            for (int q = 0; q < A.nops; ++q) {
                qrc_apply<R>(A.ops[q], psi, A.N, dco);
                __syncthreads();
            }
            // D. observables: each warp sums its share of every group into its row
            for (int g = 0; g < A.nobs; ++g) {
                const QrcObs ob = A.obs[g];
                R s0 = 0, s1 = 0, s2 = 0;
                if (ob.q2 < 0) {
                    const int b = ob.q1;
                    for (uint32_t h = tid; h < dim / 2; h += blockDim.x) {
                        const uint32_t i0 = ins0<uint32_t>(h, b), i1 = i0 | (1u << b);
                        const C u = psi[i0], v = psi[i1];
                        s0 += u.x * v.x + u.y * v.y;                    // Re conj(u) v
                        s1 += u.x * v.y - u.y * v.x;                    // Im conj(u) v
                        s2 += (u.x * u.x + u.y * u.y) - (v.x * v.x + v.y * v.y);
                    }
                    s0 *= 2;
                    s1 *= 2;
                } else {
                    const int a = ob.q1, b = ob.q2, lo = a < b ? a : b, hi = a < b ? b : a;
                    for (uint32_t h = tid; h < dim / 4; h += blockDim.x) {
                        const uint32_t i00 = ins0<uint32_t>(ins0<uint32_t>(h, lo), hi);
                        const uint32_t i10 = i00 | (1u << a), i01 = i00 | (1u << b), i11 = i10 | (1u << b);
                        const C v00 = psi[i00], v10 = psi[i10], v01 = psi[i01], v11 = psi[i11];
                        const R c0 = v00.x * v11.x + v00.y * v11.y;     // Re conj(v00) v11
                        const R c1 = v10.x * v01.x + v10.y * v01.y;     // Re conj(v10) v01
                        s0 += c0 + c1;
                        s1 += c1 - c0;
                        s2 += (v00.x * v00.x + v00.y * v00.y) + (v11.x * v11.x + v11.y * v11.y) -
                              (v10.x * v10.x + v10.y * v10.y) - (v01.x * v01.x + v01.y * v01.y);
                    }
                    s0 *= 2;
                    s1 *= 2;
                }
                double w0 = s0, w1 = s1, w2 = s2;
#pragma unroll
                for (int dd = 16; dd > 0; dd >>= 1) {
                    w0 += __shfl_xor_sync(0xffffffffu, w0, dd);
                    w1 += __shfl_xor_sync(0xffffffffu, w1, dd);
                    w2 += __shfl_xor_sync(0xffffffffu, w2, dd);
                }
                if (lane == 0) {
                    double* row = red + (size_t)warp * A.n_ops + ob.out;
                    row[0] = w0;
                    row[1] = w1;
                    row[2] = w2;
                }
            }
            __syncthreads();
            for (int f = tid; f < A.n_ops; f += blockDim.x) {
                double s = 0;
                for (int w = 0; w < nwarps; ++w) s += red[(size_t)w * A.n_ops + f];
                atomicAdd(&A.X[(size_t)k * A.n_ops + f], s);
                if (A.X_traj) A.X_traj[((size_t)t * A.T + k) * A.n_ops + f] = s;
            }
            __syncthreads();
        }
    }
}

// shared memory of one trajectory CTA
size_t qrc_smem_bytes(int N, int L, int n_ops, size_t amp_bytes) {
    const size_t d = (size_t)1 << L;
    return (amp_bytes << N) + d * amp_bytes + 2 * d * sizeof(double) + kQrcThreads * sizeof(double) +
           (size_t)(kQrcThreads / 32) * n_ops * sizeof(double);
}

constexpr size_t kQrcMaxSmem = 200 * 1024;

cudaError_t qrc_kernels_init(smoq_ctx* ctx) {
    (void)ctx;
    cudaError_t e = cudaFuncSetAttribute(qrc_traj_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kQrcMaxSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(qrc_traj_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kQrcMaxSmem);
}

}  // namespace smoq

using namespace smoq;

smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);
smoq_status smoq_internal_plan_step(smoq_plan* P, smoq_ctx** ctx, int* N, int* dtype, const std::vector<GateIR>** step);
int smoq_internal_low_bits(smoq_ctx* ctx, int dtype);

#define QCK(call)                                                         \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return smoq_internal_cuda(ctx, e_, #call); \
    } while (0)

extern "C" smoq_status smoq_qrc_run(smoq_plan* plan, const smoq_qrc_params* p, const double* psi0,
                                    const double* padded_u, int T, int64_t n_traj, double* X, double* X_traj) {
    smoq_ctx* ctx = nullptr;
    int N = 0, dtype = 0;
    const std::vector<GateIR>* step = nullptr;
    if (!plan || smoq_internal_plan_step(plan, &ctx, &N, &dtype, &step) != SMOQ_OK) return SMOQ_ERR_BADINPUT;
    if (!p || !X || !padded_u) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "qrc_run: null argument");
    const int L = p->L;
    // the reset reshapes the state as 2^L x 2^L (qrc_reset_psi! is called with L_in = L_res = L)
    if (L < 1 || 2 * L != N) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "qrc_run: the plan must act on N = 2L qubits");
    if (L > 7 || (dtype == SMOQ_C128 && L > 6))
        return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED,
                                  "qrc_run: a trajectory's state must fit in shared memory (L <= 7 complex64, 6 complex128)");
    if (T < 1 || n_traj < 1 || p->n_substeps < 0)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "qrc_run: T, n_traj must be >= 1, n_substeps >= 0");
    if (p->encoding != 0 && p->encoding != 1) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "qrc_run: unknown encoding");
    if (p->reset != 1 && p->reset != 2)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT,
                                  "Unknown protocol: use :traceout_rail_1 or :traceout_rail_2");
    const int n_ops = 3 * N + 3 * (L - 1) * 2 + 3 * L;

    // C. one input's evolution: n_substeps Trotter steps, fused on a tile spanning the state
    std::vector<GateIR> ev;
    for (int s = 0; s < p->n_substeps; ++s) ev.insert(ev.end(), step->begin(), step->end());
    std::vector<DevOp> ops;
    if (!ev.empty()) {
        std::vector<Pass> passes;
        try {
            passes = plan_passes(ev, N, N, std::min(N, smoq_internal_low_bits(ctx, dtype)), -1, 0);
        } catch (const std::exception& ex) {
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, ex.what());
        }
        for (const Pass& ps : passes)
            for (const DevOp& op : ps.ops) {
                const bool kind_ok = op.kind == OPK_DENSE1 || op.kind == OPK_DENSE2 || op.kind == OPK_PARITY2 ||
                                     op.kind == OPK_MONO || op.kind == OPK_DIAG;
                bool bits_ok = op.nq >= 0 && op.nq <= 4;
                for (int t = 0; bits_ok && t < op.nq; ++t) bits_ok = op.lb[t] == op.gb[t] && op.lb[t] >= 0 && op.lb[t] < N;
                if (!kind_ok || !bits_ok)
                    return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, "qrc_run: evolution op outside the whole-state tile");
                ops.push_back(op);
            }
    }
    // D. observable groups in the reference's order
    std::vector<QrcObs> obs;
    int out = 0;
    for (int q = 0; q < N; ++q, out += 3) obs.push_back({q, -1, out, 0});
    for (int r = 0; r < 2; ++r)
        for (int s = 0; s + 1 < L; ++s, out += 3) obs.push_back({r * L + s, r * L + s + 1, out, 0});
    for (int s = 0; s < L; ++s, out += 3) obs.push_back({s, L + s, out, 0});
    // A. the input windows (encode_input_ry_psi!: Ry(pi u) on qubit q -> cos, sin of pi u / 2)
    std::vector<double> enc((size_t)T * L * 2);
    for (int k = 0; k < T; ++k)
        for (int q = 0; q < L; ++q) {
            // padded_u[k + q] (:batch) or padded_u[k + L] (:broadcast), 1-based k and q
            const double u = padded_u[p->encoding == 1 ? (int64_t)k + L : (int64_t)k + q + 1];
            enc[((size_t)k * L + q) * 2] = std::cos(M_PI * u / 2);
            enc[((size_t)k * L + q) * 2 + 1] = std::sin(M_PI * u / 2);
        }
    // the initial state, in the state's precision
    const size_t dim = (size_t)1 << N, amp = dtype == SMOQ_C64 ? 8 : 16;
    std::vector<unsigned char> init(dim * amp, 0);
    for (size_t a = 0; a < dim; ++a) {
        const double re = psi0 ? psi0[2 * a] : (a == 0 ? 1.0 : 0.0), im = psi0 ? psi0[2 * a + 1] : 0.0;
        if (dtype == SMOQ_C64) {
            const float f[2] = {(float)re, (float)im};
            std::memcpy(&init[a * amp], f, sizeof(f));
        } else {
            const double f[2] = {re, im};
            std::memcpy(&init[a * amp], f, sizeof(f));
        }
    }
    const size_t smem = qrc_smem_bytes(N, L, n_ops, amp);
    if (smem > kQrcMaxSmem) return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, "qrc_run: state too large for shared memory");

    // one device allocation: initial state | windows | ops | groups | sums | per-trajectory features
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_init = al(init.size()), b_enc = al(enc.size() * 8), b_ops = al(std::max<size_t>(1, ops.size()) * sizeof(DevOp)),
                 b_obs = al(obs.size() * sizeof(QrcObs)), b_X = al((size_t)T * n_ops * 8),
                 b_Xt = X_traj ? al((size_t)n_traj * T * n_ops * 8) : 0;
    char* buf = nullptr;
    QCK(cudaMallocAsync((void**)&buf, b_init + b_enc + b_ops + b_obs + b_X + b_Xt, ctx->stream));
    std::unique_ptr<char, std::function<void(char*)>> hold(buf, [ctx](char* q) { cudaFreeAsync(q, ctx->stream); });
    char* c = buf;
    QrcArgs A;
    A.psi0 = c;
    QCK(cudaMemcpyAsync(c, init.data(), init.size(), cudaMemcpyHostToDevice, ctx->stream));
    c += b_init;
    A.enc = (const double*)c;
    QCK(cudaMemcpyAsync(c, enc.data(), enc.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    c += b_enc;
    A.ops = (const DevOp*)c;
    if (!ops.empty()) QCK(cudaMemcpyAsync(c, ops.data(), ops.size() * sizeof(DevOp), cudaMemcpyHostToDevice, ctx->stream));
    c += b_ops;
    A.obs = (const QrcObs*)c;
    QCK(cudaMemcpyAsync(c, obs.data(), obs.size() * sizeof(QrcObs), cudaMemcpyHostToDevice, ctx->stream));
    c += b_obs;
    A.X = (double*)c;
    QCK(cudaMemsetAsync(c, 0, (size_t)T * n_ops * 8, ctx->stream));
    c += b_X;
    A.X_traj = X_traj ? (double*)c : nullptr;
    A.n_traj = n_traj;
    A.seed = p->seed;
    A.traj_offset = p->traj_offset;
    A.nops = (int32_t)ops.size();
    A.nobs = (int32_t)obs.size();
    A.n_ops = n_ops;
    A.N = N;
    A.L = L;
    A.T = T;
    A.protocol = p->reset;
    const void* fn = dtype == SMOQ_C64 ? (const void*)qrc_traj_kernel<float> : (const void*)qrc_traj_kernel<double>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kQrcThreads, smem) != cudaSuccess || per_sm < 1) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    const int grid = (int)std::min<int64_t>(n_traj, (int64_t)ctx->num_sms * per_sm);
    if (dtype == SMOQ_C64) qrc_traj_kernel<float><<<grid, kQrcThreads, smem, ctx->stream>>>(A);
    else qrc_traj_kernel<double><<<grid, kQrcThreads, smem, ctx->stream>>>(A);
    ctx->launches++;
    QCK(cudaGetLastError());
    std::vector<double> sums((size_t)T * n_ops);
    QCK(cudaMemcpyAsync(sums.data(), A.X, sums.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (X_traj) QCK(cudaMemcpyAsync(X_traj, A.X_traj, (size_t)n_traj * T * n_ops * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QCK(cudaStreamSynchronize(ctx->stream));
    // X_sum ./ n_traj
    for (size_t x = 0; x < sums.size(); ++x) X[x] = sums[x] / (double)n_traj;
    return SMOQ_OK;
}

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
// With the context's engine option at 3 the states stream through HBM
// instead: per input, the plan's compiled passes (a CUDA graph), then one
// kernel for the features of that input and the reset for the next.
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

// one group sweep over the amplitude quadruples of qubits (a, b): (XX, YY, ZZ) at
// out, and, where out_a / out_b >= 0, (X, Y, Z) of a / b there
struct QrcObs {
    int32_t a, b, out, out_a, out_b, pad;
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

// 128 threads per trajectory CTA (measured at L = 6: 143 ms against 157-171 ms with 256
// threads and 205 ms with 512; 64 threads were no faster); the reset splits the
// threads over the 2^L outcomes, so 2^L <= kQrcThreads (L <= 7)
#ifndef SMOQ_QRC_THREADS
#define SMOQ_QRC_THREADS 128
#endif
constexpr int kQrcThreads = SMOQ_QRC_THREADS;
static_assert(kQrcThreads >= 128 && kQrcThreads % 32 == 0, "the reset needs 2^L <= threads for L <= 7");
// CTAs per SM the register budget is sized for (64 and 128 registers a thread; shared
// memory allows 6 at L = 6 complex64)
#ifndef SMOQ_QRC_MINB_C64
#define SMOQ_QRC_MINB_C64 8
#endif
#ifndef SMOQ_QRC_MINB_C128
#define SMOQ_QRC_MINB_C128 4
#endif

// Bank swizzle of a trajectory's state in shared memory: amplitude j is stored
// at j ^ M(j), M XORing the bits inside one 128-byte bank row (16 complex64 or 8
// complex128 amplitudes) with masks keyed by the two bits above the row.  The
// masks make the 16 (8) lanes of a half-warp (quarter-warp) phase hit distinct
// banks in every pair sweep on a qubit inside the row and in the 2-qubit sweeps
// of adjacent qubits there (without it, 42% of the shared-memory wavefronts of
// the ladder workload were bank conflicts).  An involution on [0, 2^N).
template <typename R>
struct QrcSwizzle {
    __device__ __forceinline__ uint32_t operator()(uint32_t j) const {
        return sizeof(R) == 4 ? j ^ (((j >> 4) & 1u) * 15u) ^ (((j >> 5) & 1u) * 10u)
                              : j ^ (((j >> 3) & 1u) * 7u) ^ (((j >> 4) & 1u) * 5u);
    }
};

// warp sum of x added into this warp's feature row
__device__ __forceinline__ void qrc_flush(double x, double* row, int f, int lane) {
#pragma unroll
    for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
    if (lane == 0) row[f] = x;
}

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

// one evolution op on the whole (swizzled) state in shared memory (qubit t at bit lb[t])
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
            const uint32_t js = QrcSwizzle<R>()(j);
            psi[js] = cmul(dco[m], psi[js]);
        }
    } else {
        sweep_op<R, uint32_t>(op, psi, N, op.lb, tid, nthr, QrcSwizzle<R>());
    }
}

// shared-memory scratch of a trajectory CTA, after the 2^N-amplitude state
template <typename R>
struct QrcScratch {
    typename CT<R>::T* phi;  // the kept rail's normalised state (2^L)
    double* pin;             // encoded input amplitudes (real, 2^L)
    double* prob;            // outcome probabilities (2^L)
    double* part;            // one partial per thread
    double* red;             // [warps][n_ops] feature rows
};
template <typename R>
__device__ __forceinline__ QrcScratch<R> qrc_scratch(unsigned char* sm, uint32_t dim, uint32_t d) {
    using C = typename CT<R>::T;
    QrcScratch<R> S;
    S.phi = reinterpret_cast<C*>(sm) + dim;
    S.pin = reinterpret_cast<double*>(S.phi + d);
    S.prob = S.pin + d;
    S.part = S.prob + d;
    S.red = S.part + kQrcThreads;
    return S;
}

// A + B for input k: encode the window, measure the rail of psi (shared memory)
// with the draw of (k, traj), write |psi_in> (x) |phi> to out (shared memory
// through the swizzle, or global through the identity; out may alias psi: every
// read of psi ends before the first write)
template <typename R, typename OutMap>
__device__ __forceinline__ void qrc_reset(const QrcArgs& A, int k, uint64_t traj, const typename CT<R>::T* psi,
                                          typename CT<R>::T* out, OutMap om, const QrcScratch<R>& S) {
    const QrcSwizzle<R> sw;
    using C = typename CT<R>::T;
    __shared__ int s_out;
    __shared__ double s_inv;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t dim = 1u << A.N, d = 1u << A.L;
    // the encoded input, prod_q (bit q ? sin : cos)
    const double* e = A.enc + (size_t)k * A.L * 2;
    for (uint32_t i = tid; i < d; i += nthr) {
        double v = 1.0;
        for (int q = 0; q < A.L; ++q) v *= ((i >> q) & 1) ? e[2 * q + 1] : e[2 * q];
        S.pin[i] = v;
    }
    // probabilities of the measured rail: x = the measured index, y = the kept one
    {
        const uint32_t x = tid & (d - 1), np = nthr / d;
        double s = 0;
        for (uint32_t y = tid / d; y < d; y += np) {
            const C v = psi[sw(A.protocol == 1 ? x + d * y : y + d * x)];
            s += (double)v.x * v.x + (double)v.y * v.y;
        }
        S.part[tid] = s;
    }
    __syncthreads();
    for (uint32_t x = tid; x < d; x += nthr) {
        double s = 0;
        for (uint32_t p = 0; p < nthr / d; ++p) s += S.part[x + d * p];
        S.prob[x] = s;
    }
    __syncthreads();
    if (tid == 0) {
        double total = 0;
        for (uint32_t x = 0; x < d; ++x) total += S.prob[x];
        const double r = qrc_uniform(A.seed, (uint64_t)k, traj);
        int outcome = 0;  // (no crossing: the first outcome, as the reference)
        double cum = 0;
        for (uint32_t x = 0; x < d; ++x) {
            cum += S.prob[x] / total;
            if (r <= cum) {
                outcome = (int)x;
                break;
            }
        }
        const double nrm = sqrt(S.prob[outcome]);
        s_out = outcome;
        s_inv = nrm > 1e-12 ? 1.0 / nrm : 0.0;  // 0: the reset falls back to |0>
    }
    __syncthreads();
    const uint32_t o = (uint32_t)s_out;
    const double inv = s_inv;
    for (uint32_t y = tid; y < d; y += nthr) {
        C v;
        if (inv > 0) {
            const C w = psi[sw(A.protocol == 1 ? o + d * y : y + d * o)];
            v.x = (R)((double)w.x * inv);
            v.y = (R)((double)w.y * inv);
        } else {
            v.x = (R)(y == 0 ? 1 : 0);
            v.y = (R)0;
        }
        S.phi[y] = v;
    }
    __syncthreads();
    for (uint32_t a = tid; a < dim; a += nthr) {
        const C v = S.phi[a >> A.L];
        const R w = (R)S.pin[a & (d - 1)];
        C z;
        z.x = w * v.x;
        z.y = w * v.y;
        out[om(a)] = z;
    }
}

// D: the features of input k of trajectory t (chunk-relative index tc for X_traj
// is t itself) from psi in shared memory: one sweep per bond or rung, per-warp
// rows, then one atomic add per feature into the trajectory sums
template <typename R>
__device__ __forceinline__ void qrc_features(const QrcArgs& A, int k, int64_t t, const typename CT<R>::T* psi,
                                             const QrcScratch<R>& S) {
    using C = typename CT<R>::T;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
    const uint32_t dim = 1u << A.N;
    for (int g = 0; g < A.nobs; ++g) {
        const QrcObs ob = A.obs[g];
        const int a = ob.a, b = ob.b, lo = a < b ? a : b, hi = a < b ? b : a;
        const QrcSwizzle<R> sw;
        const uint32_t oa = sw(1u << a), ob_ = sw(1u << b);
        R xx = 0, yy = 0, zz = 0, xa = 0, ya = 0, za = 0, xb = 0, yb = 0, zb = 0;
        for (uint32_t h = tid; h < dim / 4; h += nthr) {
            const uint32_t i00 = sw(ins0<uint32_t>(ins0<uint32_t>(h, lo), hi));  // (XOR-linear swizzle)
            const uint32_t i10 = i00 ^ oa, i01 = i00 ^ ob_, i11 = i10 ^ ob_;
            const C v00 = psi[i00], v10 = psi[i10], v01 = psi[i01], v11 = psi[i11];
            const R n00 = v00.x * v00.x + v00.y * v00.y, n10 = v10.x * v10.x + v10.y * v10.y;
            const R n01 = v01.x * v01.x + v01.y * v01.y, n11 = v11.x * v11.x + v11.y * v11.y;
            const R c0 = v00.x * v11.x + v00.y * v11.y;  // Re conj(v00) v11
            const R c1 = v10.x * v01.x + v10.y * v01.y;  // Re conj(v10) v01
            xx += c0 + c1;
            yy += c1 - c0;
            zz += (n00 + n11) - (n10 + n01);
            // conj(v00) v10 + conj(v01) v11: the pairs of qubit a
            xa += (v00.x * v10.x + v00.y * v10.y) + (v01.x * v11.x + v01.y * v11.y);
            ya += (v00.x * v10.y - v00.y * v10.x) + (v01.x * v11.y - v01.y * v11.x);
            za += (n00 + n01) - (n10 + n11);
            // conj(v00) v01 + conj(v10) v11: the pairs of qubit b
            xb += (v00.x * v01.x + v00.y * v01.y) + (v10.x * v11.x + v10.y * v11.y);
            yb += (v00.x * v01.y - v00.y * v01.x) + (v10.x * v11.y - v10.y * v11.x);
            zb += (n00 + n10) - (n01 + n11);
        }
        double* row = S.red + (size_t)warp * A.n_ops;
        qrc_flush(2.0 * (double)xx, row, ob.out, lane);
        qrc_flush(2.0 * (double)yy, row, ob.out + 1, lane);
        qrc_flush((double)zz, row, ob.out + 2, lane);
        if (ob.out_a >= 0) {
            qrc_flush(2.0 * (double)xa, row, ob.out_a, lane);
            qrc_flush(2.0 * (double)ya, row, ob.out_a + 1, lane);
            qrc_flush((double)za, row, ob.out_a + 2, lane);
        }
        if (ob.out_b >= 0) {
            qrc_flush(2.0 * (double)xb, row, ob.out_b, lane);
            qrc_flush(2.0 * (double)yb, row, ob.out_b + 1, lane);
            qrc_flush((double)zb, row, ob.out_b + 2, lane);
        }
    }
    __syncthreads();
    for (int f = tid; f < A.n_ops; f += nthr) {
        double s = 0;
        for (int w = 0; w < nwarps; ++w) s += S.red[(size_t)w * A.n_ops + f];
        atomicAdd(&A.X[(size_t)k * A.n_ops + f], s);
        if (A.X_traj) A.X_traj[((size_t)t * A.T + k) * A.n_ops + f] = s;
    }
}

// The resident kernel: each trajectory's state stays in shared memory for the
// whole series; the evolution runs as shared-memory sweeps of the fused ops.
template <typename R>
__global__ void __launch_bounds__(kQrcThreads, sizeof(R) == 4 ? SMOQ_QRC_MINB_C64 : SMOQ_QRC_MINB_C128)
    qrc_traj_kernel(const QrcArgs A) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t dim = 1u << A.N, d = 1u << A.L;
    C* psi = reinterpret_cast<C*>(sm);
    const QrcScratch<R> S = qrc_scratch<R>(sm, dim, d);
    __shared__ C dco[16];
    const int tid = threadIdx.x;
    const C* p0 = reinterpret_cast<const C*>(A.psi0);
    for (int64_t t = blockIdx.x; t < A.n_traj; t += gridDim.x) {
        for (uint32_t a = tid; a < dim; a += blockDim.x) psi[QrcSwizzle<R>()(a)] = p0[a];
        __syncthreads();
        const uint64_t traj = A.traj_offset + (uint64_t)t;
        for (int k = 0; k < A.T; ++k) {
            qrc_reset<R>(A, k, traj, psi, psi, QrcSwizzle<R>(), S);
            __syncthreads();
            for (int q = 0; q < A.nops; ++q) {  // n_substeps Trotter steps
                qrc_apply<R>(A.ops[q], psi, A.N, dco);
                __syncthreads();
            }
            qrc_features<R>(A, k, t, psi, S);
            __syncthreads();
        }
    }
}

// The streaming kernel, between the compiled evolution passes: for trajectories
// t0 .. t0 + nchunk - 1 (state c at dst + c 2^N), the features of input k_obs
// (k_obs >= 0) and the reset for input k_obs + 1 (< T).  src: the states to read
// (src_stride 0: every trajectory starts from the same state).
template <typename R>
__global__ void __launch_bounds__(kQrcThreads, sizeof(R) == 4 ? SMOQ_QRC_MINB_C64 : SMOQ_QRC_MINB_C128)
    qrc_obs_reset_kernel(const QrcArgs A, const void* src, int64_t src_stride, void* dst, int k_obs, int64_t t0,
                         int64_t nchunk) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t dim = 1u << A.N, d = 1u << A.L;
    C* psi = reinterpret_cast<C*>(sm);
    const QrcScratch<R> S = qrc_scratch<R>(sm, dim, d);
    const int tid = threadIdx.x;
    for (int64_t c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const C* in = reinterpret_cast<const C*>(src) + c * src_stride;
        for (uint32_t a = tid; a < dim; a += blockDim.x) psi[QrcSwizzle<R>()(a)] = in[a];
        __syncthreads();
        if (k_obs >= 0) {
            qrc_features<R>(A, k_obs, t0 + c, psi, S);
            __syncthreads();
        }
        if (k_obs + 1 < A.T) {
            qrc_reset<R>(A, k_obs + 1, A.traj_offset + (uint64_t)(t0 + c), psi,
                         reinterpret_cast<C*>(dst) + c * (int64_t)dim, IdMap(), S);
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
    const void* fns[4] = {(const void*)qrc_traj_kernel<float>, (const void*)qrc_traj_kernel<double>,
                          (const void*)qrc_obs_reset_kernel<float>, (const void*)qrc_obs_reset_kernel<double>};
    for (const void* f : fns)
        if (cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQrcMaxSmem))
            return e;
    return cudaSuccess;
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

    // the evolution: shared-memory sweeps inside the resident kernel, or, when the
    // context's engine option is 3, the plan's compiled passes between streaming
    // kernels (the states in HBM).  Both are FP32/FP64-issue-bound at about the same
    // rate on the ladder workloads (dense 4x4 ops after field fusion), so the
    // resident kernel, with no HBM traffic, is the default.
    const bool streaming = ctx->engine == 3 && p->n_substeps > 0;
    // C. one input's evolution: n_substeps Trotter steps, fused on a tile spanning the state
    std::vector<GateIR> ev;
    for (int s = 0; !streaming && s < p->n_substeps; ++s) ev.insert(ev.end(), step->begin(), step->end());
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
    // D. one group sweep per rail bond (also carrying X, Y, Z of its lower qubit) and per
    // rung (the last rung carries the rails' last qubits); outputs in the reference's
    // order: (X, Y, Z) of qubit q at 3q, then the bonds of rail 0, rail 1, then the rungs
    std::vector<QrcObs> obs;
    int out = 3 * N;
    for (int r = 0; r < 2; ++r)
        for (int s = 0; s + 1 < L; ++s, out += 3) obs.push_back({r * L + s, r * L + s + 1, out, 3 * (r * L + s), -1, 0});
    for (int s = 0; s < L; ++s, out += 3)
        obs.push_back({s, L + s, out, s == L - 1 ? 3 * s : -1, s == L - 1 ? 3 * (L + s) : -1, 0});
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
    auto per_sm = [&](const void* fn) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kQrcThreads, smem) != cudaSuccess || n < 1) {
            (void)cudaGetLastError();
            n = 1;
        }
        return (int64_t)n;
    };
    std::unique_ptr<void, std::function<void(void*)>> hold_states(nullptr, [ctx](void* q) {
        if (q) cudaFreeAsync(q, ctx->stream);
    });
    if (!streaming) {
        const void* fn = dtype == SMOQ_C64 ? (const void*)qrc_traj_kernel<float> : (const void*)qrc_traj_kernel<double>;
        const int grid = (int)std::min<int64_t>(n_traj, (int64_t)ctx->num_sms * per_sm(fn));
        if (dtype == SMOQ_C64) qrc_traj_kernel<float><<<grid, kQrcThreads, smem, ctx->stream>>>(A);
        else qrc_traj_kernel<double><<<grid, kQrcThreads, smem, ctx->stream>>>(A);
        ctx->launches++;
        QCK(cudaGetLastError());
    } else {
        // trajectories in chunks of at most 4 GiB of states; per input: the plan's
        // compiled passes (n_substeps steps, one CUDA graph), then one kernel for the
        // features of this input and the reset for the next
        const size_t sbytes = dim * amp;
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_traj, (int64_t)(((size_t)4 << 30) / sbytes)));
        void* states = nullptr;
        QCK(cudaMallocAsync(&states, (size_t)chunk * sbytes, ctx->stream));
        hold_states.reset(states);
        smoq_state st;
        st.ctx = ctx;
        st.N = N;
        st.dtype = dtype;
        st.owned = false;
        st.ptr = states;
        const void* fn = dtype == SMOQ_C64 ? (const void*)qrc_obs_reset_kernel<float>
                                           : (const void*)qrc_obs_reset_kernel<double>;
        const int64_t slots = (int64_t)ctx->num_sms * per_sm(fn);
        auto obs_reset = [&](const void* src, int64_t stride, int k_obs, int64_t t0, int64_t nb) {
            const int grid = (int)std::min<int64_t>(nb, slots);
            if (dtype == SMOQ_C64)
                qrc_obs_reset_kernel<float><<<grid, kQrcThreads, smem, ctx->stream>>>(A, src, stride, states, k_obs, t0, nb);
            else
                qrc_obs_reset_kernel<double><<<grid, kQrcThreads, smem, ctx->stream>>>(A, src, stride, states, k_obs, t0, nb);
            ctx->launches++;
            return cudaGetLastError();
        };
        for (int64_t t0 = 0; t0 < n_traj; t0 += chunk) {
            const int64_t nb = std::min<int64_t>(chunk, n_traj - t0);
            st.batch = (int)nb;
            QCK(obs_reset(A.psi0, 0, -1, t0, nb));
            for (int k = 0; k < T; ++k) {
                if (smoq_status s = smoq_trotter_step(plan, &st, p->n_substeps)) return s;
                QCK(obs_reset(states, (int64_t)dim, k, t0, nb));
            }
        }
    }
    std::vector<double> sums((size_t)T * n_ops);
    QCK(cudaMemcpyAsync(sums.data(), A.X, sums.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (X_traj) QCK(cudaMemcpyAsync(X_traj, A.X_traj, (size_t)n_traj * T * n_ops * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QCK(cudaStreamSynchronize(ctx->stream));
    // X_sum ./ n_traj
    for (size_t x = 0; x < sums.size(); ++x) X[x] = sums[x] / (double)n_traj;
    return SMOQ_OK;
}

// circuit.cu -- circuits with noise channels, projective measurements, resets
// and classical conditions on a batch of trajectories: the pure-state
// (MCWF) branch of apply_circuit! (utils/cpu/cpuVariationalQuantumCircuitExecutor.jl:95-146)
// with apply_noise_mcwf! (:187), apply_measure_psi! (:210) and
// apply_reset_psi! (:220).
//
// Every state of the smoq_state is one trajectory.  The op list is cut at
// its stochastic and conditional ops; the gates between two cuts run as one
// fused sequence (smoq_apply_sequence: planned tile passes) on the whole
// batch.  At a cut, each trajectory draws its own uniform u from
// Philox4x32-10 (key = seed, counter = (op index, 0x80000000, trajectory)),
// so the result does not depend on the batch size or on the order of
// trajectories:
//  * pauli_noise_kernel -- depolarizing, bit flip, phase flip, dephasing:
//    the draw picks I, X, Y or Z per trajectory (the decision needs no
//    reduction); blocks of trajectories that drew I return at once, so a
//    weak channel costs a pass over the few trajectories that drew a Pauli;
//  * qubit_stats_kernel + branch_kernel -- amplitude damping, measurement,
//    reset: an FP64 reduction of |psi|^2 over the qubit's two halves per
//    trajectory, then one pass in which every block sums its trajectory's
//    partials in a fixed order, draws u, picks the branch and applies the
//    branch's real 2x2 map (collapse / jump / damping / force, with the
//    renormalisation folded in) to the qubit's pairs;
//  * cond_gate_kernel -- a gate with if_outcome: applied only to the
//    trajectories whose recorded outcome is 1.
// Outcomes live on the device ([batch][n_meas] int32) until the call ends.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);
smoq_status smoq_internal_ops_to_ir(int N, const smoq_op* ops, int n, const double* theta,
                                    std::vector<smoq::GateIR>& out);

namespace smoq {
namespace {

constexpr int kCircThreads = 256;

// the trajectory's condition: if_outcome slot `cond` (0-based, -1 = always)
__device__ __forceinline__ bool cond_met(const int32_t* outcomes, int n_meas, int64_t b, int cond) {
    return cond < 0 || outcomes[b * n_meas + cond] == 1;
}

struct PauliNoise {
    int32_t type;        // SMOQ_N_*
    int32_t q;
    int32_t cond;        // outcome slot or -1
    uint32_t op_index;
    double p;
};

template <typename R>
__global__ void __launch_bounds__(kCircThreads) pauli_noise_kernel(typename CT<R>::T* psi, int N, PauliNoise nz,
                                                                   uint64_t seed, uint64_t traj0,
                                                                   const int32_t* outcomes, int n_meas) {
    using C = typename CT<R>::T;
    const int64_t b = blockIdx.y;
    if (!cond_met(outcomes, n_meas, b, nz.cond)) return;
    const int code = pauli_code(nz.type, nz.p, circuit_draw(seed, nz.op_index, traj0 + (uint64_t)b));
    if (code == 0) return;
    C* s = psi + (b << N);
    const uint64_t npairs = (uint64_t)1 << (N - 1), bit = (uint64_t)1 << nz.q;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ins0<uint64_t>(g, nz.q), i1 = i0 | bit;
        C a0 = s[i0], a1 = s[i1];
        if (code == 1) {  // X: swap
            s[i0] = a1;
            s[i1] = a0;
        } else if (code == 2) {  // Y: (a0, a1) -> (-i a1, i a0), :297-306
            C n0, n1;
            n0.x = a1.y;
            n0.y = -a1.x;
            n1.x = -a0.y;
            n1.y = a0.x;
            s[i0] = n0;
            s[i1] = n1;
        } else {  // Z
            a1.x = -a1.x;
            a1.y = -a1.y;
            s[i1] = a1;
        }
    }
}

// partials[(b * nblk + blk) * 2 + h] = sum of |psi_i|^2 over the block's amplitudes of
// trajectory b whose bit q is h (FP64)
template <typename R>
__global__ void __launch_bounds__(kCircThreads) qubit_stats_kernel(const typename CT<R>::T* psi, int N, int q,
                                                                   double* partials) {
    const int64_t b = blockIdx.y;
    const typename CT<R>::T* s = psi + (b << N);
    const uint64_t len = (uint64_t)1 << N;
    double h[2] = {0, 0};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x)
        h[(i >> q) & 1] += cabs2d(s[i]);
    __shared__ double red[kCircThreads / 32][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        double x = h[k];
        for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
        if (lane == 0) red[w][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double x = 0;
        for (int k = 0; k < kCircThreads / 32; ++k) x += red[k][threadIdx.x];
        partials[((size_t)b * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = x;
    }
}

struct Branch {
    int32_t kind;        // BranchKind
    int32_t q;
    int32_t cond;        // outcome slot or -1
    int32_t out_slot;    // measurement: the outcome slot it records
    int32_t target;      // reset: 0 zero, 1 one, 2 plus, 3 minus
    uint32_t op_index;
    int32_t nblk;        // stats partials per trajectory
    double gamma;        // amplitude damping
};

template <typename R>
__global__ void __launch_bounds__(kCircThreads) branch_kernel(typename CT<R>::T* psi, int N, Branch br,
                                                              const double* partials, uint64_t seed,
                                                              uint64_t traj0, int32_t* outcomes, int n_meas) {
    using C = typename CT<R>::T;
    const int64_t b = blockIdx.y;
    if (!cond_met(outcomes, n_meas, b, br.cond)) return;
    __shared__ double sK[4];
    if (threadIdx.x == 0) {
        // the trajectory's halves, summed in block order (every block gets the same)
        double s0 = 0, s1 = 0;
        const double* p = partials + (size_t)b * br.nblk * 2;
        for (int k = 0; k < br.nblk; ++k) s0 += p[2 * k], s1 += p[2 * k + 1];
        double K[4];
        int m;
        branch_map(br.kind, br.target, br.gamma, s0, s1, circuit_draw(seed, br.op_index, traj0 + (uint64_t)b), K, &m);
        for (int k = 0; k < 4; ++k) sK[k] = K[k];
        if (blockIdx.x == 0 && m >= 0) outcomes[b * n_meas + br.out_slot] = m;
    }
    __syncthreads();
    const R k00 = (R)sK[0], k01 = (R)sK[1], k10 = (R)sK[2], k11 = (R)sK[3];
    C* s = psi + (b << N);
    const uint64_t npairs = (uint64_t)1 << (N - 1), bit = (uint64_t)1 << br.q;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ins0<uint64_t>(g, br.q), i1 = i0 | bit;
        const C a0 = s[i0], a1 = s[i1];
        C n0, n1;
        n0.x = k00 * a0.x + k01 * a1.x;
        n0.y = k00 * a0.y + k01 * a1.y;
        n1.x = k10 * a0.x + k11 * a1.x;
        n1.y = k10 * a0.y + k11 * a1.y;
        s[i0] = n0;
        s[i1] = n1;
    }
}

// one gate, only on the trajectories whose outcome slot `cond` holds 1
template <typename R>
__global__ void __launch_bounds__(kCircThreads) cond_gate_kernel(typename CT<R>::T* psi, int N, const DevOp op,
                                                                 const int32_t* outcomes, int n_meas, int cond) {
    using C = typename CT<R>::T;
    const int64_t b = blockIdx.y;
    if (!cond_met(outcomes, n_meas, b, cond)) return;
    C* s = psi + (b << N);
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nthr = (uint64_t)gridDim.x * blockDim.x;
    if (op.kind == OPK_DIAG) {
        const uint64_t len = (uint64_t)1 << N;
        for (uint64_t i = tid; i < len; i += nthr) {
            int m = 0;
            for (int t = 0; t < op.nq; ++t) m |= (int)((i >> op.gb[t]) & 1) << t;
            s[i] = cmul(coef<R>(op, m), s[i]);
        }
        return;
    }
    sweep_op<R, uint64_t>(op, s, N, op.gb, tid, nthr);
}

// one step of the cut op list
struct Step {
    enum Kind { GATES, NOISE, BRANCH, COND_GATE } kind;
    std::vector<smoq_op> gates;  // GATES: fused as one sequence
    PauliNoise nz{};
    Branch br{};
    int op_index = -1;           // COND_GATE: the op
    int cond = -1;
};

bool is_gate(int t) { return t >= SMOQ_G_RX && t <= SMOQ_G_U2; }
bool is_pauli_noise(int t) {
    return t == SMOQ_N_DEPOLARIZING || t == SMOQ_N_DEPHASING || t == SMOQ_N_BIT_FLIP || t == SMOQ_N_PHASE_FLIP ||
           t == SMOQ_N_PHASE_DAMPING;
}
bool is_measure(int t) { return t == SMOQ_M_MEASURE_Z || t == SMOQ_M_MEASURE_X || t == SMOQ_M_MEASURE_Y; }

smoq_op plain_gate(int type, int q) {
    smoq_op o{};
    o.type = type;
    o.q[0] = q;
    o.param = -1;
    return o;
}

// grid over (blocks per trajectory, trajectories): about 4 waves of the SMs in all
dim3 circuit_grid(const smoq_ctx* ctx, int N, int batch, uint64_t units) {
    const uint64_t want = std::max<uint64_t>(1, (uint64_t)ctx->num_sms * 4 / (uint64_t)batch);
    const uint64_t need = std::max<uint64_t>(1, (units + kCircThreads * 4 - 1) / (kCircThreads * 4));
    (void)N;
    return dim3((unsigned)std::min<uint64_t>({want, need, 65535}), (unsigned)batch);
}

}  // namespace
}  // namespace smoq

using namespace smoq;

extern "C" smoq_status smoq_apply_sequence(smoq_state* st, const smoq_op* ops, int n, const double* theta);

extern "C" smoq_status smoq_apply_circuit_mcwf(smoq_state* st, const smoq_op* ops, int n, const double* theta,
                                               uint64_t seed, uint64_t traj_offset, int32_t* outcomes) {
    if (!st || !st->ctx || (!ops && n > 0) || n < 0) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = st->ctx;
    const int N = st->N;
    if (st->batch > 65535) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "circuit: at most 65535 trajectories");
    // ---- cut the op list (apply_circuit!, Executor.jl:101-114)
    std::vector<Step> steps;
    int n_meas = 0;
    auto gates_step = [&]() -> std::vector<smoq_op>& {
        if (steps.empty() || steps.back().kind != Step::GATES) {
            steps.emplace_back();
            steps.back().kind = Step::GATES;
        }
        return steps.back().gates;
    };
    for (int i = 0; i < n; ++i) {
        const smoq_op& o = ops[i];
        const std::string where = "circuit op " + std::to_string(i) + ": ";
        if (o.if_outcome < 0) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "if_outcome < 0").c_str());
        // a condition on a measurement that has not happened yet never holds (:103-105)
        if (o.if_outcome > n_meas) continue;
        const int cond = o.if_outcome - 1;  // -1: always
        const int q = o.q[0];
        if (!is_gate(o.type) && (q < 0 || q >= N))
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "qubit out of range").c_str());
        if (is_gate(o.type)) {
            if (cond < 0) {
                gates_step().push_back(o);
            } else {
                steps.emplace_back();
                steps.back().kind = Step::COND_GATE;
                steps.back().op_index = i;
                steps.back().cond = cond;
            }
        } else if (is_pauli_noise(o.type)) {
            if (!(o.angle >= 0.0 && o.angle <= 1.0))
                return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "noise probability must be in [0,1]").c_str());
            steps.emplace_back();
            Step& s = steps.back();
            s.kind = Step::NOISE;
            s.nz.type = o.type;
            s.nz.q = q;
            s.nz.cond = cond;
            s.nz.op_index = (uint32_t)i;
            s.nz.p = o.angle;
        } else if (o.type == SMOQ_N_AMPLITUDE_DAMPING || is_measure(o.type) || o.type == SMOQ_R_RESET) {
            if (o.type == SMOQ_N_AMPLITUDE_DAMPING && !(o.angle >= 0.0 && o.angle <= 1.0))
                return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "gamma must be in [0,1]").c_str());
            if (is_measure(o.type) && cond >= 0)
                return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED,
                                          (where + "a conditional measurement is not supported").c_str());
            if (o.type == SMOQ_R_RESET && (o.q[1] < 0 || o.q[1] > 3))
                return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "reset target must be 0..3").c_str());
            // basis changes of projective_measurement! (cpuQuantumStateMeasurements.jl:326-341)
            if (o.type == SMOQ_M_MEASURE_X) gates_step().push_back(plain_gate(SMOQ_G_H, q));
            if (o.type == SMOQ_M_MEASURE_Y) {
                gates_step().push_back(plain_gate(SMOQ_G_SDG, q));
                gates_step().push_back(plain_gate(SMOQ_G_H, q));
            }
            steps.emplace_back();
            Step& s = steps.back();
            s.kind = Step::BRANCH;
            s.br.kind = o.type == SMOQ_N_AMPLITUDE_DAMPING ? BR_AMPDAMP : (is_measure(o.type) ? BR_MEASURE : BR_RESET);
            s.br.q = q;
            s.br.cond = cond;
            s.br.out_slot = is_measure(o.type) ? n_meas++ : -1;
            s.br.target = o.type == SMOQ_R_RESET ? o.q[1] : 0;
            s.br.op_index = (uint32_t)i;
            s.br.gamma = o.angle;
            if (o.type == SMOQ_M_MEASURE_X) gates_step().push_back(plain_gate(SMOQ_G_H, q));
            if (o.type == SMOQ_M_MEASURE_Y) {
                gates_step().push_back(plain_gate(SMOQ_G_H, q));
                gates_step().push_back(plain_gate(SMOQ_G_S, q));
            }
        } else if (o.type == SMOQ_N_THERMAL_RELAXATION || o.type == SMOQ_T_TRACE_OUT ||
                   o.type == SMOQ_L_LINDBLAD_STEP) {
            // no effect on a pure state in the reference (Executor.jl:187-201, :231-249)
        } else {
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, (where + "unknown op type").c_str());
        }
    }
    // ---- device buffers: outcomes [batch][n_meas], stats partials
    const int64_t B = st->batch;
    const dim3 g_pairs = circuit_grid(ctx, N, (int)B, (uint64_t)1 << (N > 0 ? N - 1 : 0));
    const dim3 g_amps = circuit_grid(ctx, N, (int)B, (uint64_t)1 << N);
    const int nblk = (int)g_amps.x;
    int32_t* d_out = nullptr;
    double* d_part = nullptr;
    const size_t out_bytes = (size_t)std::max<int64_t>(1, B * n_meas) * sizeof(int32_t);
    cudaError_t e = cudaMallocAsync((void**)&d_out, out_bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_part, (size_t)B * nblk * 2 * sizeof(double), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, out_bytes, ctx->stream);
    struct Free {
        smoq_ctx* c;
        void* p[2];
        ~Free() {
            for (void* x : p)
                if (x) cudaFreeAsync(x, c->stream);
        }
    } hold{ctx, {d_out, d_part}};
    if (e != cudaSuccess) return smoq_internal_cuda(ctx, e, "circuit buffers");
    const bool c64 = st->dtype == SMOQ_C64;
    for (const Step& s : steps) {
        if (s.kind == Step::GATES) {
            if (s.gates.empty()) continue;
            if (smoq_status r = smoq_apply_sequence(st, s.gates.data(), (int)s.gates.size(), theta)) return r;
            continue;
        }
        if (s.kind == Step::NOISE) {
            if (c64)
                pauli_noise_kernel<float><<<g_pairs, kCircThreads, 0, ctx->stream>>>(
                    (float2*)st->ptr, N, s.nz, seed, traj_offset, d_out, std::max(1, n_meas));
            else
                pauli_noise_kernel<double><<<g_pairs, kCircThreads, 0, ctx->stream>>>(
                    (double2*)st->ptr, N, s.nz, seed, traj_offset, d_out, std::max(1, n_meas));
            ctx->launches++;
        } else if (s.kind == Step::BRANCH) {
            Branch br = s.br;
            br.nblk = nblk;
            if (c64) {
                qubit_stats_kernel<float><<<g_amps, kCircThreads, 0, ctx->stream>>>((const float2*)st->ptr, N, br.q,
                                                                                     d_part);
                branch_kernel<float><<<g_pairs, kCircThreads, 0, ctx->stream>>>(
                    (float2*)st->ptr, N, br, d_part, seed, traj_offset, d_out, std::max(1, n_meas));
            } else {
                qubit_stats_kernel<double><<<g_amps, kCircThreads, 0, ctx->stream>>>((const double2*)st->ptr, N,
                                                                                      br.q, d_part);
                branch_kernel<double><<<g_pairs, kCircThreads, 0, ctx->stream>>>(
                    (double2*)st->ptr, N, br, d_part, seed, traj_offset, d_out, std::max(1, n_meas));
            }
            ctx->launches += 2;
        } else {  // COND_GATE
            std::vector<GateIR> ir;
            smoq_op one = ops[s.op_index];
            one.if_outcome = 0;
            if (smoq_status r = smoq_internal_ops_to_ir(N, &one, 1, theta, ir))
                return smoq_internal_fail(ctx, r, "circuit: bad conditional gate");
            DevOp op;
            try {
                build_devop(ir[0], nullptr, op);
            } catch (const std::exception& ex) {
                return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, ex.what());
            }
            if (c64)
                cond_gate_kernel<float><<<g_amps, kCircThreads, 0, ctx->stream>>>((float2*)st->ptr, N, op, d_out,
                                                                                   std::max(1, n_meas), s.cond);
            else
                cond_gate_kernel<double><<<g_amps, kCircThreads, 0, ctx->stream>>>((double2*)st->ptr, N, op, d_out,
                                                                                    std::max(1, n_meas), s.cond);
            ctx->launches++;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return smoq_internal_cuda(ctx, e, "circuit kernel");
    }
    if (outcomes && n_meas > 0)
        e = cudaMemcpyAsync(outcomes, d_out, (size_t)B * n_meas * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return smoq_internal_cuda(ctx, e, "circuit");
    return SMOQ_OK;
}

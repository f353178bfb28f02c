// mcwf.cu -- batched Monte Carlo wave-function evolution (quantum jumps).
//
// One state of the batch per trajectory.  A step of the first-order
// quantum-jump rule (the same rule the oracle's so_mcwf_step states, with the
// reference lines it follows):
//   1. the coherent Trotter step, with the previous step's renormalisation
//      factor folded into the first pass (OPK_STATESCALE);
//   2. the no-jump decay psi_i *= f(i), f a product over qubits of per-bit
//      factors (sigma- on an excited bit, sigma+ on a ground bit, and the
//      uniform L^dag L = I part of sigma_z / sigma_x), applied in the last pass
//      from byte tables (OPK_REALTAB); that pass's epilogue writes per-tile
//      FP64 partial sums of |psi|^2 and of the populations the jump weights
//      need;
//   3. mcwf_decide_kernel, one thread per trajectory: norm^2 and populations
//      from the partials, two uniforms from Philox4x32-10 with counter
//      (step, trajectory) and key = seed, the jump decision and channel,
//      and the next renormalisation factor;
//   4. mcwf_jump_kernel applies the chosen jump operator to the trajectories
//      that jumped (blocks of the others exit at once);
//   5. every record_every steps, one FP64 pass of Z / ZZ reductions,
//      normalised per trajectory, and the trajectory means.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

namespace smoq {

struct DJump {
    int32_t type;    // 0 sigma-, 1 sigma+, 2 sigma_z, 3 sigma_x
    int32_t qubit;
    int32_t popidx;  // index into the epilogue's populations (sigma+/-), else -1
    int32_t pad;
    double gamma;
};

constexpr int kJumpRows = 256;  // block rows of the jump kernel (jumpers per step: typically dozens)

__global__ void mcwf_decide_kernel(int B, int64_t tiles_per_state, int npop, const double* partials,
                                   const DJump* ops, int nops, double dt, uint64_t seed, uint64_t traj_offset,
                                   uint64_t step, int32_t* jump, double* scale, int32_t* counts,
                                   int32_t* jumpers, int32_t* njump) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    // FP64 sums over this trajectory's tiles, in tile order
    double nrm = 0;
    const double* p = partials + (size_t)b * tiles_per_state * (1 + npop);
    for (int64_t t = 0; t < tiles_per_state; ++t) nrm += p[t * (1 + npop)];
    const uint64_t tr = traj_offset + (uint64_t)b;
    uint32_t c[4] = {(uint32_t)step, (uint32_t)(step >> 32), (uint32_t)tr, (uint32_t)(tr >> 32)};
    philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double uj = u01_53(c[0], c[1]), uc = u01_53(c[2], c[3]);
    const double dp = 1.0 - nrm;
    int chosen = -1;
    double new_norm = nrm;
    if (uj < dp && dp > 0) {
        auto ev_of = [&](int o) {
            if (ops[o].type == 0 || ops[o].type == 1) {
                double s = 0;
                for (int64_t t = 0; t < tiles_per_state; ++t) s += p[t * (1 + npop) + 1 + ops[o].popidx];
                return ops[o].type == 0 ? s : nrm - s;
            }
            return nrm;
        };
        double wsum = 0;
        for (int o = 0; o < nops; ++o) wsum += ops[o].gamma * dt * ev_of(o) / nrm;
        if (wsum > 0) {
            const double target = uc * wsum;
            double cum = 0, chosen_ev = nrm;
            chosen = nops - 1;
            for (int o = 0; o < nops; ++o) {
                const double ev = ev_of(o);
                cum += ops[o].gamma * dt * ev / nrm;
                chosen_ev = ev;
                if (target < cum) {
                    chosen = o;
                    break;
                }
            }
            new_norm = (ops[chosen].type == 0 || ops[chosen].type == 1) ? chosen_ev : nrm;
            counts[b] += 1;
            jumpers[atomicAdd(njump, 1)] = b;  // (the list order does not matter)
        }
    }
    jump[b] = chosen;
    scale[b] = 1.0 / sqrt(new_norm);
}

// the chosen jump applied to the trajectories on the step's jumper list: block row y
// takes list entries y, y + gridDim.y, ... (a few dozen jumpers per step among
// thousands of trajectories: the grid stays small)
template <typename R>
__global__ void mcwf_jump_kernel(typename CT<R>::T* psi, int N, const int32_t* jump, const DJump* ops,
                                 const int32_t* jumpers, const int32_t* njump, int B) {
    using C = typename CT<R>::T;
    const int nj = *njump;
    for (int e = blockIdx.y; e < nj; e += gridDim.y) {
    const int b = jumpers[e];
    if (b < 0 || b >= B) continue;
    const int o = jump[b];
    if (o < 0) continue;
    const int64_t len = (int64_t)1 << N;
    C* s = psi + (int64_t)b * len;
    const int q = ops[o].qubit, ty = ops[o].type;
    const uint64_t m = 1ull << q;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (len >> 1);
         g += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ins0<uint64_t>((uint64_t)g, q), i1 = i0 | m;
        const C a = s[i0], c = s[i1];
        if (ty == 0) {          // sigma- = |0><1|
            s[i0] = c;
            s[i1] = czero(a);
        } else if (ty == 1) {   // sigma+ = |1><0|
            s[i1] = a;
            s[i0] = czero(a);
        } else if (ty == 2) {   // sigma_z
            s[i1] = cscale(c, (R)-1);
        } else {                // sigma_x
            s[i0] = c;
            s[i1] = a;
        }
    }
    }
}

// tmp[b * (1 + k) + j]: Z-string sums with j = 0 the squared norm; writes the
// normalised values into rec[b * stride + off + j - 1]
__global__ void mcwf_record_kernel(int B, int k, const double* tmp, double* rec, int stride, int off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * k) return;
    const int b = i / k, j = i - b * k;
    rec[(size_t)b * stride + off + j] = tmp[(size_t)b * (1 + k) + 1 + j] / tmp[(size_t)b * (1 + k)];
}

// mean over trajectories, FP64, fixed order
__global__ void mcwf_mean_kernel(int B, int nobs, const double* rec, double* mean) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nobs) return;
    double s = 0;
    for (int b = 0; b < B; ++b) s += rec[(size_t)b * nobs + j];
    mean[j] = s / B;
}

}  // namespace smoq

using namespace smoq;

// pieces of capi.cu this file uses
smoq_status smoq_internal_plan_step(smoq_plan* plan, std::vector<GateIR>& out, int& N, int& dtype, int& order);
smoq_status smoq_internal_prepare(smoq_ctx* ctx, smoq_state* st, const std::vector<GateIR>& gates,
                                  int epilogue_special, bool reusable, void** prog_handle,
                                  bool variational = false);
smoq_status smoq_internal_rerun(smoq_ctx* ctx, smoq_state* st, void* prog_handle, const Epilogue* ep);
void smoq_internal_free_prog(void* prog_handle);
smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);
smoq_status smoq_internal_zreduce(smoq_ctx* ctx, smoq_state* st, const uint64_t* zmasks, int nobs, double* d_out);
int64_t smoq_internal_tiles_per_state(void* prog_handle);

#define MCK(call)                                                         \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return smoq_internal_cuda(ctx, e_, #call); \
    } while (0)

namespace {
struct DevBufs {
    std::vector<void*> ptrs;
    cudaStream_t s = nullptr;
    ~DevBufs() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
    template <typename T>
    cudaError_t alloc(T** p, size_t n) {
        cudaError_t e = cudaMallocAsync((void**)p, std::max<size_t>(n, 1) * sizeof(T), s);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};
}  // namespace

extern "C" smoq_status smoq_mcwf_run(smoq_plan* plan, smoq_state* st, const smoq_jump_op* ops, int nops, double dt,
                                     uint64_t seed, uint64_t traj_offset, int steps, int record_every, double* z_mean,
                                     double* zz_mean, double* z_traj, double* zz_traj, int* jumps) {
    if (!plan || !st || !st->ctx) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = st->ctx;
    std::vector<GateIR> step;
    int N = 0, dtype = 0, order = 0;
    if (smoq_status s = smoq_internal_plan_step(plan, step, N, dtype, order)) return s;
    if (N != st->N || dtype != st->dtype) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "plan/state shape mismatch");
    if (order != 1) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "MCWF needs a first-order (order 1) Trotter plan");
    if (nops < 0 || (nops > 0 && !ops) || steps < 0 || record_every < 1 || !z_mean || !zz_mean || N < 2)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad MCWF arguments");
    if (!(dt > 0) || !std::isfinite(dt)) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "dt must be positive");
    if (st->batch > 65535) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "at most 65535 trajectories per call");
    // jump ops, decay factors and the populations the weights need
    std::vector<DJump> dj(std::max(1, nops));
    std::vector<int> popq;
    double gz = 0;
    std::vector<double> a(N, 1.0), bq(N, 1.0);  // factor of an excited / a ground bit
    for (int o = 0; o < nops; ++o) {
        const smoq_jump_op& j = ops[o];
        if (j.type < 0 || j.type > 3 || j.qubit < 0 || j.qubit >= N || !(j.gamma >= 0) || j.gamma * dt >= 1.0)
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad jump operator (type, qubit, or gamma*dt >= 1)");
        dj[o].type = j.type;
        dj[o].qubit = j.qubit;
        dj[o].gamma = j.gamma;
        dj[o].popidx = -1;
        if (j.type == 0 || j.type == 1) {
            int idx = -1;
            for (size_t k = 0; k < popq.size(); ++k)
                if (popq[k] == j.qubit) idx = (int)k;
            if (idx < 0) {
                idx = (int)popq.size();
                popq.push_back(j.qubit);
            }
            dj[o].popidx = idx;
            if (j.type == 0) a[j.qubit] *= std::sqrt(1.0 - j.gamma * dt);
            else bq[j.qubit] *= std::sqrt(1.0 - j.gamma * dt);
        } else {
            gz += j.gamma;
        }
    }
    if (gz * dt >= 1.0) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "sum of dephasing rates * dt >= 1");
    if (popq.size() > 40) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "at most 40 distinct sigma+- qubits");
    const int ntab = (N + 7) / 8;
    std::vector<double> tabs((size_t)ntab * 256, 1.0);
    for (int k = 0; k < ntab; ++k)
        for (int v = 0; v < 256; ++v) {
            double f = 1.0;
            for (int i = 0; i < 8; ++i) {
                const int q = 8 * k + i;
                if (q >= N) break;
                f *= ((v >> i) & 1) ? a[q] : bq[q];
            }
            tabs[(size_t)k * 256 + v] = f;
        }
    const double fu = std::sqrt(1.0 - dt * gz);
    for (int v = 0; v < 256; ++v) tabs[v] *= fu;

    const int B = st->batch;
    const int nrec = steps / record_every + 1;
    DevBufs buf;
    buf.s = ctx->stream;
    double *d_tabs, *d_scale, *d_rec, *d_mean, *d_tmp, *d_part;
    int32_t *d_jump, *d_counts;
    DJump* d_ops;
    const int nobs = 2 * N - 1;  // Z_i, then Z_i Z_{i+1}
    MCK(buf.alloc(&d_tabs, tabs.size()));
    MCK(buf.alloc(&d_scale, B));
    MCK(buf.alloc(&d_jump, B));
    MCK(buf.alloc(&d_counts, B));
    int32_t *d_jumpers, *d_njump;
    MCK(buf.alloc(&d_jumpers, B));
    MCK(buf.alloc(&d_njump, 1));
    MCK(buf.alloc(&d_ops, dj.size()));
    MCK(buf.alloc(&d_rec, (size_t)nrec * B * nobs));
    MCK(buf.alloc(&d_mean, (size_t)nrec * nobs));
    MCK(buf.alloc(&d_tmp, (size_t)B * 32));
    MCK(cudaMemcpyAsync(d_tabs, tabs.data(), tabs.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    MCK(cudaMemcpyAsync(d_ops, dj.data(), dj.size() * sizeof(DJump), cudaMemcpyHostToDevice, ctx->stream));
    MCK(cudaMemsetAsync(d_counts, 0, B * sizeof(int32_t), ctx->stream));
    std::vector<double> ones(B, 1.0);
    MCK(cudaMemcpyAsync(d_scale, ones.data(), B * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));

    // the step program: renormalise, coherent step, decay (+ epilogue)
    std::vector<GateIR> prog;
    GateIR sc;
    sc.special = OPK_STATESCALE;
    sc.aux = d_scale;
    sc.diag = true;
    prog.push_back(sc);
    prog.insert(prog.end(), step.begin(), step.end());
    // The no-jump decay is a product of one-qubit real diagonals (diag(bq, a) per
    // qubit, times fu).  The compiled complex64 kernels fold such diagonals into their
    // stage phases, so there they enter as diagonal gates and the table op stays only
    // as a marker that keeps the norm and population epilogue in the step's last
    // pass; the other engines apply the byte tables in one sweep.
    const bool fold_decay = st->dtype == SMOQ_C64 && (ctx->engine == 3 || (ctx->engine < 0 && jit_available()));
    if (fold_decay) {
        double g = fu;
        for (int q = 0; q < N; ++q) {
            if (a[q] == 1.0 && bq[q] == 1.0) continue;
            const cd m[4] = {bq[q] * g, 0.0, 0.0, a[q] * g};
            g = 1.0;
            prog.push_back(gate_1q(q, m));
        }
        if (g != 1.0) {  // (no population decay: the uniform factor alone)
            const cd m[4] = {g, 0.0, 0.0, g};
            prog.push_back(gate_1q(0, m));
        }
    }
    GateIR dec;
    dec.special = OPK_REALTAB;
    dec.aux = d_tabs;
    dec.aux2 = fold_decay ? 0 : ntab;
    dec.diag = true;
    prog.push_back(dec);

    Epilogue ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.npop = (int)popq.size();
    for (size_t k = 0; k < popq.size(); ++k) ep.popq[k] = popq[k];
    void* handle = nullptr;
    if (smoq_status s = smoq_internal_prepare(ctx, st, prog, OPK_REALTAB, true, &handle)) return s;
    std::unique_ptr<void, void (*)(void*)> hold(handle, smoq_internal_free_prog);
    const int64_t tps = smoq_internal_tiles_per_state(handle);
    MCK(buf.alloc(&d_part, (size_t)B * tps * (1 + ep.npop)));
    ep.partials = d_part;

    // records: Z-string chunks of <= 31 observables plus the squared norm
    std::vector<uint64_t> masks(nobs);
    for (int i = 0; i < N; ++i) masks[i] = 1ull << i;
    for (int i = 0; i + 1 < N; ++i) masks[N + i] = 3ull << i;
    auto record = [&](int r) -> smoq_status {
        for (int o0 = 0; o0 < nobs; o0 += 31) {
            const int k = std::min(31, nobs - o0);
            uint64_t zm[32];
            zm[0] = 0;
            for (int j = 0; j < k; ++j) zm[1 + j] = masks[o0 + j];
            if (smoq_status s = smoq_internal_zreduce(ctx, st, zm, k + 1, d_tmp)) return s;
            mcwf_record_kernel<<<(B * k + 255) / 256, 256, 0, ctx->stream>>>(B, k, d_tmp, d_rec + (size_t)r * B * nobs,
                                                                           nobs, o0);
            ctx->launches++;
        }
        mcwf_mean_kernel<<<(nobs + 127) / 128, 128, 0, ctx->stream>>>(B, nobs, d_rec + (size_t)r * B * nobs,
                                                                      d_mean + (size_t)r * nobs);
        ctx->launches++;
        MCK(cudaGetLastError());
        return SMOQ_OK;
    };

    if (smoq_status s = record(0)) return s;
    const int jump_grid = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)1 << N) / 512, 64));
    int r = 1;
    for (int s = 0; s < steps; ++s) {
        if (smoq_status e = smoq_internal_rerun(ctx, st, handle, &ep)) return e;
        MCK(cudaMemsetAsync(d_njump, 0, sizeof(int32_t), ctx->stream));
        mcwf_decide_kernel<<<(B + 127) / 128, 128, 0, ctx->stream>>>(B, tps, ep.npop, d_part, d_ops, nops, dt, seed,
                                                                     traj_offset, (uint64_t)s, d_jump, d_scale,
                                                                     d_counts, d_jumpers, d_njump);
        dim3 jg(jump_grid, std::min(B, kJumpRows));
        if (dtype == SMOQ_C64)
            mcwf_jump_kernel<float><<<jg, 256, 0, ctx->stream>>>((float2*)st->ptr, N, d_jump, d_ops, d_jumpers,
                                                                 d_njump, B);
        else
            mcwf_jump_kernel<double><<<jg, 256, 0, ctx->stream>>>((double2*)st->ptr, N, d_jump, d_ops, d_jumpers,
                                                                  d_njump, B);
        ctx->launches += 2;
        MCK(cudaGetLastError());
        if ((s + 1) % record_every == 0) {
            if (smoq_status e = record(r)) return e;
            ++r;
        }
    }
    // leave every trajectory normalised
    MCK(launch_scale(st, d_scale, 1.0));

    std::vector<double> mean((size_t)nrec * nobs);
    MCK(cudaMemcpyAsync(mean.data(), d_mean, mean.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<double> rec;
    if (z_traj || zz_traj) {
        rec.resize((size_t)nrec * B * nobs);
        MCK(cudaMemcpyAsync(rec.data(), d_rec, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    std::vector<int32_t> cnt(B);
    MCK(cudaMemcpyAsync(cnt.data(), d_counts, B * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    MCK(cudaStreamSynchronize(ctx->stream));
    for (int rr = 0; rr < nrec; ++rr) {
        for (int i = 0; i < N; ++i) z_mean[(size_t)rr * N + i] = mean[(size_t)rr * nobs + i];
        for (int i = 0; i + 1 < N; ++i) zz_mean[(size_t)rr * (N - 1) + i] = mean[(size_t)rr * nobs + N + i];
        for (int b = 0; b < B && !rec.empty(); ++b) {
            const double* src = rec.data() + ((size_t)rr * B + b) * nobs;
            if (z_traj)
                for (int i = 0; i < N; ++i) z_traj[((size_t)rr * B + b) * N + i] = src[i];
            if (zz_traj)
                for (int i = 0; i + 1 < N; ++i) zz_traj[((size_t)rr * B + b) * (N - 1) + i] = src[N + i];
        }
    }
    if (jumps)
        for (int b = 0; b < B; ++b) jumps[b] = cnt[b];
    return SMOQ_OK;
}

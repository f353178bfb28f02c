// noisy_grad.cu -- the energy and its adjoint gradient along fixed noisy
// trajectories, with checkpoints at the non-invertible steps.
//
// A trajectory of a noisy circuit (smoq_apply_circuit_mcwf: the same draws, the
// same rules, circuit_common.cuh) is a product of maps: gates U_k(theta)
// (unitary), drawn Paulis P (unitary), and the normalised branch maps
// psi' = K psi of amplitude damping, measurement and reset (K real on the
// qubit's pairs, its normalisation folded in).  With the draws fixed the
// branches are piecewise constant in theta, so E(theta) = <psi_T|H|psi_T> has
// the path-wise gradient
//     dE/dtheta_k = Im <lambda_k| G_k |phi_k>          (U_k = exp(-i theta_k G_k / 2))
// where lambda is carried backwards from lambda_T = H psi_T: through a unitary
// by U^dag, through a branch map by
//     lambda <- K^T (lambda - Re<psi'|lambda> psi')
// (the second term removes the change of the normalisation).  Unitary steps
// are uncomputed (phi <- U^dag phi); a branch map cannot be inverted, so the
// forward pass stores phi in front of every k-th branch op (a checkpoint) and
// the backward pass restores phi from the nearest checkpoint, replaying the
// recorded steps from there.  Memory: ceil(branches / k) + 2 states.
//
// The reference's gradient treats noise as identity (the Enzyme wrapper,
// utils/cpu/cpuVQCEnzymeWrapper.jl:160-170); this is the gradient of the
// trajectory the noise actually produced, whose mean over trajectories is the
// gradient of the mean energy.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <functional>
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

constexpr int kNgThreads = 256;

// per block FP64 partials of <a|P|b> = sum_j conj(a_{j^x}) i^ny (-1)^popc(j & z) b_j:
// part[2 blk] = real part, part[2 blk + 1] = imaginary part
template <typename R>
__global__ void __launch_bounds__(kNgThreads) cross_pauli_kernel(const typename CT<R>::T* a,
                                                                 const typename CT<R>::T* b, int N, uint64_t x,
                                                                 uint64_t z, int ny, double* part) {
    const uint64_t len = (uint64_t)1 << N;
    double re = 0, im = 0;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x) {
        const typename CT<R>::T u = a[j ^ x], v = b[j];
        // conj(u) v
        double pr = (double)u.x * v.x + (double)u.y * v.y, pi = (double)u.x * v.y - (double)u.y * v.x;
        if (__popcll(j & z) & 1) pr = -pr, pi = -pi;
        re += pr;
        im += pi;
    }
    // times i^ny (the same for every j)
    for (int k = 0; k < (ny & 3); ++k) {
        const double t = re;
        re = -im;
        im = t;
    }
    __shared__ double red[kNgThreads / 32][2];
    for (int d = 16; d > 0; d >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, d);
        im += __shfl_down_sync(0xffffffffu, im, d);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][0] = re, red[threadIdx.x >> 5][1] = im;
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0;
        for (int w = 0; w < kNgThreads / 32; ++w) s += red[w][threadIdx.x];
        part[2 * blockIdx.x + threadIdx.x] = s;
    }
}

// (a0, a1) -> (k00 a0 + k01 a1, k10 a0 + k11 a1) on the pairs of qubit q
template <typename R>
__global__ void __launch_bounds__(kNgThreads) pair_map_kernel(typename CT<R>::T* s, int N, int q, double k00,
                                                              double k01, double k10, double k11) {
    using C = typename CT<R>::T;
    const uint64_t npairs = (uint64_t)1 << (N - 1), bit = (uint64_t)1 << q;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ins0<uint64_t>(g, q), i1 = i0 | bit;
        const C a0 = s[i0], a1 = s[i1];
        C n0, n1;
        n0.x = (R)(k00 * a0.x + k01 * a1.x);
        n0.y = (R)(k00 * a0.y + k01 * a1.y);
        n1.x = (R)(k10 * a0.x + k11 * a1.x);
        n1.y = (R)(k10 * a0.y + k11 * a1.y);
        s[i0] = n0;
        s[i1] = n1;
    }
}

// y <- y + c x (real c)
template <typename R>
__global__ void __launch_bounds__(kNgThreads) axpy_kernel(typename CT<R>::T* y, const typename CT<R>::T* x,
                                                          int N, double c) {
    const uint64_t len = (uint64_t)1 << N;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x) {
        typename CT<R>::T v = y[j];
        v.x = (R)(v.x + c * x[j].x);
        v.y = (R)(v.y + c * x[j].y);
        y[j] = v;
    }
}

// one recorded step of a trajectory's forward pass
struct Rec {
    enum Kind { GATE, PAULI, BRANCH } kind;
    int op = -1;          // GATE: the op index (its gate IR in gates[]); PAULI / BRANCH: the op index
    int gate = -1;        // GATE: index into the trajectory's gate list
    int q = 0;            // PAULI / BRANCH: the qubit
    int code = 0;         // PAULI: 1 X, 2 Y, 3 Z
    double K[4] = {1, 0, 0, 1};  // BRANCH: the applied map
    int ckpt = -1;        // BRANCH: checkpoint slot of the state in front of it, or -1
};

struct Ctx {
    smoq_ctx* ctx;
    int N;
    int dtype;
    int grid;
    double* d_part;
    int64_t len() const { return (int64_t)1 << N; }
    size_t bytes() const { return (size_t)len() * (dtype == SMOQ_C64 ? 8 : 16); }
};

smoq_state view(const Ctx& c, void* ptr) {
    smoq_state s;
    s.ctx = c.ctx;
    s.N = c.N;
    s.dtype = c.dtype;
    s.batch = 1;
    s.ptr = ptr;
    s.owned = false;
    return s;
}

cudaError_t cross(const Ctx& c, const void* a, const void* b, uint64_t x, uint64_t z, int ny, double* re, double* im) {
    if (c.dtype == SMOQ_C64)
        cross_pauli_kernel<float><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((const float2*)a, (const float2*)b, c.N, x,
                                                                            z, ny, c.d_part);
    else
        cross_pauli_kernel<double><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((const double2*)a, (const double2*)b, c.N,
                                                                             x, z, ny, c.d_part);
    c.ctx->launches++;
    std::vector<double> h(2 * (size_t)c.grid);
    cudaError_t e = cudaMemcpyAsync(h.data(), c.d_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                    c.ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.ctx->stream);
    double r = 0, i = 0;
    for (int k = 0; k < c.grid; ++k) r += h[2 * k], i += h[2 * k + 1];
    if (re) *re = r;
    if (im) *im = i;
    return e;
}

cudaError_t pair_map(const Ctx& c, void* s, int q, const double K[4]) {
    if (c.dtype == SMOQ_C64)
        pair_map_kernel<float><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((float2*)s, c.N, q, K[0], K[1], K[2], K[3]);
    else
        pair_map_kernel<double><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((double2*)s, c.N, q, K[0], K[1], K[2],
                                                                          K[3]);
    c.ctx->launches++;
    return cudaGetLastError();
}

cudaError_t axpy(const Ctx& c, void* y, const void* x, double a) {
    if (c.dtype == SMOQ_C64)
        axpy_kernel<float><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((float2*)y, (const float2*)x, c.N, a);
    else
        axpy_kernel<double><<<c.grid, kNgThreads, 0, c.ctx->stream>>>((double2*)y, (const double2*)x, c.N, a);
    c.ctx->launches++;
    return cudaGetLastError();
}

cudaError_t apply_ir(const Ctx& c, void* s, const GateIR& g) {
    DevOp op;
    build_devop(g, nullptr, op);
    smoq_state v = view(c, s);
    return launch_direct_op(&v, op);
}

GateIR dagger(const GateIR& g) {
    GateIR d = g;
    const int dim = 1 << g.nq;
    for (int r = 0; r < dim; ++r)
        for (int k = 0; k < dim; ++k) d.m[r * dim + k] = std::conj(g.m[k * dim + r]);
    return d;
}

GateIR pauli_ir(int code, int q) {
    const int type = code == 1 ? SMOQ_G_X : code == 2 ? SMOQ_G_Y : SMOQ_G_Z;
    return gate_named(type, &q, 0.0);
}

// the generator of a parameterised gate as Pauli strings (coef, x, z, ny), U = exp(-i theta G / 2)
bool generator_terms(const smoq_op& o, std::vector<HamTerm>& t) {
    const uint64_t a = 1ull << o.q[0], b = 1ull << o.q[1];
    auto add = [&](double c, uint64_t x, uint64_t z) {
        HamTerm h;
        h.coef = c;
        h.x = x;
        h.z = z;
        h.ny = __builtin_popcountll(x & z);
        h.pad = 0;
        t.push_back(h);
    };
    switch (o.type) {
        case SMOQ_G_RX: add(1, a, 0); return true;
        case SMOQ_G_RY: add(1, a, a); return true;
        case SMOQ_G_RZ: add(1, 0, a); return true;
        case SMOQ_G_RXX: add(1, a | b, 0); return true;
        case SMOQ_G_RYY: add(1, a | b, a | b); return true;
        case SMOQ_G_RZZ: add(1, 0, a | b); return true;
        case SMOQ_G_CRY: add(0.5, b, b), add(-0.5, b, a | b); return true;  // |1><1|_c (x) Y_t = (Y_t - Z_c Y_t) / 2
        default: return false;
    }
}

bool is_branch(int t) {
    return t == SMOQ_N_AMPLITUDE_DAMPING || t == SMOQ_M_MEASURE_Z || t == SMOQ_M_MEASURE_X || t == SMOQ_M_MEASURE_Y ||
           t == SMOQ_R_RESET;
}
bool is_pauli_noise(int t) {
    return t == SMOQ_N_DEPOLARIZING || t == SMOQ_N_DEPHASING || t == SMOQ_N_BIT_FLIP || t == SMOQ_N_PHASE_FLIP ||
           t == SMOQ_N_PHASE_DAMPING;
}

}  // namespace
}  // namespace smoq

using namespace smoq;

#define NG_CK(x)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess) return smoq_internal_cuda(ctx, e_, "noisy gradient");    \
    } while (0)

extern "C" smoq_status smoq_energy_grad_mcwf(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n,
                                             int n_params, const smoq_pauli_term* H, int nterms, const double* theta,
                                             uint64_t seed, uint64_t traj_offset, int n_traj, int checkpoint_every,
                                             double* energies, double* grads) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    if (N < 1 || N > 34) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "N must be in 1..34");
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad dtype");
    if (n < 0 || (n > 0 && !ops) || n_params < 0 || (n_params > 0 && !theta) || nterms < 1 || !H || n_traj < 1 ||
        !energies || checkpoint_every < 1)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad noisy-gradient arguments");
    const uint64_t lim = (1ull << N) - 1;
    for (int t = 0; t < nterms; ++t)
        if ((H[t].xmask | H[t].zmask) & ~lim)
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "Hamiltonian term acts beyond N");
    // the gate IR of every gate op, and the generators of the parameterised ones
    std::vector<GateIR> gate_ir(n);
    std::vector<std::vector<HamTerm>> gen(n);
    int n_branch_ops = 0;
    for (int i = 0; i < n; ++i) {
        const smoq_op& o = ops[i];
        if (o.if_outcome < 0) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "if_outcome < 0");
        if (o.type >= SMOQ_G_RX && o.type <= SMOQ_G_U2) {
            smoq_op one = o;
            one.if_outcome = 0;
            std::vector<GateIR> ir;
            if (smoq_status s = smoq_internal_ops_to_ir(N, &one, 1, theta, ir)) return s;
            gate_ir[i] = ir[0];
            if (o.param >= 0) {
                if (o.param >= n_params) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "op param index >= n_params");
                if (!generator_terms(o, gen[i]))
                    return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED,
                                              "noisy gradient: parameterised gate type has no generator");
            }
        } else if (is_branch(o.type) || is_pauli_noise(o.type)) {
            if (o.q[0] < 0 || o.q[0] >= N) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "op qubit out of range");
            if (is_branch(o.type)) ++n_branch_ops;
            if ((o.type >= SMOQ_M_MEASURE_Z && o.type <= SMOQ_M_MEASURE_Y) && o.if_outcome != 0)
                return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, "a conditional measurement is not supported");
        } else if (!(o.type == SMOQ_N_THERMAL_RELAXATION || o.type == SMOQ_T_TRACE_OUT ||
                     o.type == SMOQ_L_LINDBLAD_STEP)) {
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "unknown op type");
        }
    }
    // the Hamiltonian, device buffers: phi, lambda, checkpoints, partials
    std::vector<HamTerm> ht(nterms);
    for (int t = 0; t < nterms; ++t) {
        ht[t].coef = H[t].coef;
        ht[t].x = H[t].xmask;
        ht[t].z = H[t].zmask;
        ht[t].ny = __builtin_popcountll(H[t].xmask & H[t].zmask);
        ht[t].pad = 0;
    }
    Ctx c{ctx, N, dtype, 1, nullptr};
    c.grid = (int)std::max<int64_t>(1, std::min<int64_t>((c.len() + 1023) / 1024, (int64_t)ctx->num_sms * 4));
    const int n_ckpt = (n_branch_ops + checkpoint_every - 1) / checkpoint_every;
    std::vector<void*> owned;
    std::unique_ptr<void, std::function<void(void*)>> hold(&owned, [ctx](void* p) {
        for (void* q : *static_cast<std::vector<void*>*>(p)) cudaFreeAsync(q, ctx->stream);
    });
    auto dalloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMallocAsync(&p, bytes, ctx->stream) != cudaSuccess) return nullptr;
        owned.push_back(p);
        return p;
    };
    void* phi = dalloc(c.bytes());
    void* lam = dalloc(c.bytes());
    std::vector<void*> ckpt(n_ckpt);
    for (int k = 0; k < n_ckpt; ++k) ckpt[k] = dalloc(c.bytes());
    c.d_part = (double*)dalloc(2 * (size_t)std::max(c.grid, (int)std::min<int64_t>((c.len() + 255) / 256,
                                                                                    (int64_t)ctx->num_sms * 8)) *
                               sizeof(double));
    HamTerm* d_terms = (HamTerm*)dalloc(ht.size() * sizeof(HamTerm));
    if (!phi || !lam || !c.d_part || !d_terms || std::find(ckpt.begin(), ckpt.end(), nullptr) != ckpt.end()) {
        (void)cudaGetLastError();
        return smoq_internal_fail(ctx, SMOQ_ERR_OOM, "noisy gradient: device memory for the states and checkpoints");
    }
    NG_CK(cudaMemcpyAsync(d_terms, ht.data(), ht.size() * sizeof(HamTerm), cudaMemcpyHostToDevice, ctx->stream));
    const int eblocks = (int)std::max<int64_t>(1, std::min<int64_t>((c.len() + 255) / 256, (int64_t)ctx->num_sms * 8));
    smoq_state sphi = view(c, phi);

    for (int tr = 0; tr < n_traj; ++tr) {
        const uint64_t traj = traj_offset + (uint64_t)tr;
        // ---- forward, recording every applied step
        std::vector<Rec> rec;
        std::vector<int> outcomes;
        int branch_no = 0;
        NG_CK(launch_set_basis(&sphi, 0));
        for (int i = 0; i < n; ++i) {
            const smoq_op& o = ops[i];
            if (o.if_outcome > 0 && (o.if_outcome > (int)outcomes.size() || outcomes[o.if_outcome - 1] != 1)) continue;
            const int q = o.q[0];
            if (o.type >= SMOQ_G_RX && o.type <= SMOQ_G_U2) {
                NG_CK(apply_ir(c, phi, gate_ir[i]));
                Rec r;
                r.kind = Rec::GATE;
                r.op = i;
                rec.push_back(r);
            } else if (is_pauli_noise(o.type)) {
                const int code = pauli_code(o.type, o.angle, circuit_draw(seed, (uint32_t)i, traj));
                if (!code) continue;
                NG_CK(apply_ir(c, phi, pauli_ir(code, q)));
                Rec r;
                r.kind = Rec::PAULI;
                r.op = i;
                r.q = q;
                r.code = code;
                rec.push_back(r);
            } else if (is_branch(o.type)) {
                // basis changes of projective_measurement! as fixed gates
                auto fixed = [&](int type) -> smoq_status {
                    Rec r;
                    r.kind = Rec::GATE;
                    r.op = -1 - type;                       // a fixed gate: -1 - its type
                    r.q = q;
                    rec.push_back(r);
                    NG_CK(apply_ir(c, phi, gate_named(type, &q, 0.0)));
                    return SMOQ_OK;
                };
                if (o.type == SMOQ_M_MEASURE_X)
                    if (smoq_status s = fixed(SMOQ_G_H)) return s;
                if (o.type == SMOQ_M_MEASURE_Y) {
                    if (smoq_status s = fixed(SMOQ_G_SDG)) return s;
                    if (smoq_status s = fixed(SMOQ_G_H)) return s;
                }
                Rec r;
                r.kind = Rec::BRANCH;
                r.op = i;
                r.q = q;
                if (branch_no % checkpoint_every == 0) {
                    r.ckpt = branch_no / checkpoint_every;
                    NG_CK(cudaMemcpyAsync(ckpt[r.ckpt], phi, c.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
                }
                ++branch_no;
                double nrm = 0, zq = 0;
                NG_CK(cross(c, phi, phi, 0, 0, 0, &nrm, nullptr));
                NG_CK(cross(c, phi, phi, 0, 1ull << q, 0, &zq, nullptr));
                const int kind = o.type == SMOQ_N_AMPLITUDE_DAMPING ? BR_AMPDAMP
                                                                    : (o.type == SMOQ_R_RESET ? BR_RESET : BR_MEASURE);
                int m = -1;
                branch_map(kind, o.type == SMOQ_R_RESET ? o.q[1] : 0, o.angle, 0.5 * (nrm + zq), 0.5 * (nrm - zq),
                           circuit_draw(seed, (uint32_t)i, traj), r.K, &m);
                if (m >= 0) outcomes.push_back(m);
                NG_CK(pair_map(c, phi, q, r.K));
                rec.push_back(r);
                if (o.type == SMOQ_M_MEASURE_X)
                    if (smoq_status s = fixed(SMOQ_G_H)) return s;
                if (o.type == SMOQ_M_MEASURE_Y) {
                    if (smoq_status s = fixed(SMOQ_G_H)) return s;
                    if (smoq_status s = fixed(SMOQ_G_S)) return s;
                }
            }
        }
        // ---- energy, lambda = H phi
        smoq_state sp = view(c, phi);
        NG_CK(launch_ham_apply(ctx, &sp, lam, d_terms, nterms, c.d_part, eblocks));
        std::vector<double> ep(2 * (size_t)eblocks);
        NG_CK(cudaMemcpyAsync(ep.data(), c.d_part, ep.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        NG_CK(cudaStreamSynchronize(ctx->stream));
        double e = 0, nrm2 = 0;
        for (int k = 0; k < eblocks; ++k) e += ep[k], nrm2 += ep[eblocks + k];
        if (!(nrm2 > 0)) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "noisy gradient: zero-norm trajectory");
        energies[tr] = e / nrm2;
        if (!grads) continue;
        double* g = grads + (size_t)tr * n_params;
        for (int p = 0; p < n_params; ++p) g[p] = 0.0;
        // replay of the recorded forward steps [from, to) onto phi
        auto replay = [&](size_t from, size_t to) -> smoq_status {
            for (size_t k = from; k < to; ++k) {
                const Rec& r = rec[k];
                if (r.kind == Rec::GATE)
                    NG_CK(apply_ir(c, phi, r.op >= 0 ? gate_ir[r.op] : gate_named(-1 - r.op, &r.q, 0.0)));
                else if (r.kind == Rec::PAULI)
                    NG_CK(apply_ir(c, phi, pauli_ir(r.code, r.q)));
                else
                    NG_CK(pair_map(c, phi, r.q, r.K));
            }
            return SMOQ_OK;
        };
        // ---- backward
        for (size_t k = rec.size(); k-- > 0;) {
            const Rec& r = rec[k];
            if (r.kind == Rec::GATE) {
                if (r.op >= 0 && !gen[r.op].empty()) {
                    double acc = 0;
                    for (const HamTerm& t : gen[r.op]) {
                        double im = 0;
                        NG_CK(cross(c, lam, phi, t.x, t.z, t.ny, nullptr, &im));
                        acc += t.coef * im;
                    }
                    g[ops[r.op].param] += acc / nrm2;
                }
                const GateIR d = dagger(r.op >= 0 ? gate_ir[r.op] : gate_named(-1 - r.op, &r.q, 0.0));
                NG_CK(apply_ir(c, phi, d));
                NG_CK(apply_ir(c, lam, d));
            } else if (r.kind == Rec::PAULI) {
                const GateIR d = dagger(pauli_ir(r.code, r.q));
                NG_CK(apply_ir(c, phi, d));
                NG_CK(apply_ir(c, lam, d));
            } else {
                // lambda <- K^T (lambda - Re<psi'|lambda> psi'), psi' = phi (the state after the map)
                double proj = 0;
                NG_CK(cross(c, phi, lam, 0, 0, 0, &proj, nullptr));
                NG_CK(axpy(c, lam, phi, -proj));
                const double KT[4] = {r.K[0], r.K[2], r.K[1], r.K[3]};
                NG_CK(pair_map(c, lam, r.q, KT));
                // phi in front of the map: its checkpoint, or the nearest earlier one replayed forward
                size_t from = k;
                while (rec[from].kind != Rec::BRANCH || rec[from].ckpt < 0) --from;
                NG_CK(cudaMemcpyAsync(phi, ckpt[rec[from].ckpt], c.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
                if (smoq_status s = replay(from, k)) return s;
            }
        }
    }
    NG_CK(cudaStreamSynchronize(ctx->stream));
    return SMOQ_OK;
}

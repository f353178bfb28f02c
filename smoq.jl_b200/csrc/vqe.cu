// vqe.cu -- VQE energy and adjoint gradient.
//
// E(theta) = <phi|H|phi>, phi = U_P ... U_1 |0>, H = sum_t c_t P_t (Pauli strings).
// For a rotation U_k = exp(-i theta G_k / 2) (RX/RY/RZ/RXX/RYY/RZZ, and CRY
// with G = |1><1| (x) Y), dE/dtheta_k = Im <lambda_k| G_k |phi_k>, where
// phi_k = U_k ... U_1 |0> and lambda_k = U_{k+1}^dag ... U_P^dag H phi.
// The gradient therefore needs one forward sweep, one application of H and
// ONE backward sweep that carries the pair (phi, lambda): walking the gates
// in reverse, measure Im<lambda|G|phi> at a parameterised gate, then apply
// U_k^dag to both.  Nothing is stored per layer (the gates are unitary and
// are uncomputed), so memory is three states whatever the depth.
//
//  * ham_apply_kernel: lambda = H phi and the energy partials in one read of
//    phi per term;
//  * adj_tile_kernel: the backward sweep as fused passes over (phi, lambda)
//    tile pairs: both tiles come into shared memory by bulk copy, the pass's
//    program (U^dag ops and OPK_INNER measurements, in order) runs on both.
//    Generators are signed Pauli monomials, so a measurement is a few FMAs
//    per amplitude pair in the state's precision; a U^dag op directly before
//    a measurement on the same qubits is applied in the same sweep, and runs
//    of real-diagonal measurements (RZ, RZZ) share one read of the tiles.
//    Each warp adds its FP64 sum of a measurement to its own row of the
//    partials; adj_colsum_kernel reduces the rows.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

namespace smoq {

// lambda_k = sum_t c_t i^{ny} (-1)^{popc((k ^ x) & z)} phi_{k ^ x}; per block
// the FP64 partial sums of Re(conj(phi_k) lambda_k) (partials[blockIdx.x])
// and of |phi_k|^2 (partials[gridDim.x + blockIdx.x]), so the caller can
// divide the energy by the norm of the state it was measured on
template <typename R>
__global__ void __launch_bounds__(256) ham_apply_kernel(const typename CT<R>::T* phi, typename CT<R>::T* lam, int N,
                                                        const HamTerm* terms, int nterms, double* partials) {
    using C = typename CT<R>::T;
    const int64_t len = (int64_t)1 << N;
    double acc = 0, nrm = 0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < len; k += (int64_t)gridDim.x * blockDim.x) {
        double lr = 0, li = 0;
        for (int t = 0; t < nterms; ++t) {
            const uint64_t j = (uint64_t)k ^ terms[t].x;
            const C p = phi[j];
            double s = terms[t].coef * ((__popcll(j & terms[t].z) & 1) ? -1.0 : 1.0);
            const int yk = terms[t].ny & 3;
            double pr = p.x, pi = p.y;
            // multiply by i^yk
            if (yk == 1) { const double tr = -pi; pi = pr; pr = tr; }
            else if (yk == 2) { pr = -pr; pi = -pi; }
            else if (yk == 3) { const double tr = pi; pi = -pr; pr = tr; }
            lr += s * pr;
            li += s * pi;
        }
        C o;
        o.x = (R)lr;
        o.y = (R)li;
        lam[k] = o;
        const C f = phi[k];
        acc += (double)f.x * lr + (double)f.y * li;  // Re(conj(phi) lambda)
        nrm += (double)f.x * f.x + (double)f.y * f.y;
    }
    __shared__ double red[2][8];
    for (int d = 16; d > 0; d >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, d);
        nrm += __shfl_down_sync(0xffffffffu, nrm, d);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = acc, red[1][threadIdx.x >> 5] = nrm;
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

cudaError_t launch_ham_apply(smoq_ctx* ctx, const smoq_state* st, void* lam, const HamTerm* d_terms, int nterms,
                             double* d_part, int eblocks) {
    if (st->dtype == SMOQ_C64)
        ham_apply_kernel<float><<<eblocks, 256, 0, ctx->stream>>>((const float2*)st->ptr, (float2*)lam, st->N, d_terms,
                                                                  nterms, d_part);
    else
        ham_apply_kernel<double><<<eblocks, 256, 0, ctx->stream>>>((const double2*)st->ptr, (double2*)lam, st->N,
                                                                   d_terms, nterms, d_part);
    ctx->launches++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------- backward sweep
// The adjoint pass works on a PAIR of tiles in shared memory: P (phi) and Q
// (lambda), 2^T amplitudes each, and applies every U^dag op to both in the
// same loop iteration (one index decode, one coefficient load for both).

// U^dag op on both tiles; dco: 16 shared-memory slots for diagonal tables
template <typename R>
__device__ __forceinline__ void dual_apply(const DevOp& op, typename CT<R>::T* P, typename CT<R>::T* Q, int T,
                                           uint64_t base, typename CT<R>::T* dco) {
    using C = typename CT<R>::T;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    if (op.kind == OPK_DENSE1 && (op.flags & OPF_REAL)) {
        // real 2x2 (Ry and its products): real scalars times complex amplitudes
        const int a = op.lb[0];
        const int f = lane_flip<R>(tid, a, -1);
        const R m0 = coef<R>(op, 3 * f).x, m1 = coef<R>(op, 1 + f).x, m2 = coef<R>(op, 2 - f).x,
                m3 = coef<R>(op, 3 - 3 * f).x;
        for (uint32_t g = tid; g < (1u << (T - 1)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(g, a) ^ ((uint32_t)f << a), i1 = i0 ^ (1u << a);
            const C x = P[i0], y = P[i1], u = Q[i0], v = Q[i1];
            P[i0] = rmix(m0, x, m1, y);
            P[i1] = rmix(m2, x, m3, y);
            Q[i0] = rmix(m0, u, m1, v);
            Q[i1] = rmix(m2, u, m3, v);
        }
    } else if (op.kind == OPK_DENSE2 && (op.flags & OPF_REAL)) {
        const int a = op.lb[0], b = op.lb[1];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int f = lane_flip<R>(tid, a, b);
        const uint32_t fb = flip_bits(f, a, b);
        R m[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) m[k] = coef<R>(op, (((k >> 2) ^ f) << 2) | ((k & 3) ^ f)).x;
        for (uint32_t g = tid; g < (1u << (T - 2)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(ins0<uint32_t>(g, lo), hi) ^ fb;
            const uint32_t ix[4] = {i0, i0 ^ (1u << a), i0 ^ (1u << b), i0 ^ (1u << a) ^ (1u << b)};
            C x[4], y[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = P[ix[k]], y[k] = Q[ix[k]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C s, t;
                s.x = m[4 * r] * x[0].x, s.y = m[4 * r] * x[0].y;
                t.x = m[4 * r] * y[0].x, t.y = m[4 * r] * y[0].y;
#pragma unroll
                for (int c = 1; c < 4; ++c) {
                    s.x = fma(m[4 * r + c], x[c].x, s.x), s.y = fma(m[4 * r + c], x[c].y, s.y);
                    t.x = fma(m[4 * r + c], y[c].x, t.x), t.y = fma(m[4 * r + c], y[c].y, t.y);
                }
                P[ix[r]] = s;
                Q[ix[r]] = t;
            }
        }
    } else if (op.kind == OPK_DENSE1) {
        const int a = op.lb[0];
        const int f = lane_flip<R>(tid, a, -1);  // 0 or 1: M' = M with both indices flipped
        const C m0 = coef<R>(op, 3 * f), m1 = coef<R>(op, 1 + f), m2 = coef<R>(op, 2 - f), m3 = coef<R>(op, 3 - 3 * f);
        for (uint32_t g = tid; g < (1u << (T - 1)); g += nthr) {
            const uint32_t i0 = ins0<uint32_t>(g, a) ^ ((uint32_t)f << a), i1 = i0 ^ (1u << a);
            const C x = P[i0], y = P[i1], u = Q[i0], v = Q[i1];
            P[i0] = cfma(m0, x, cmul(m1, y));
            P[i1] = cfma(m2, x, cmul(m3, y));
            Q[i0] = cfma(m0, u, cmul(m1, v));
            Q[i1] = cfma(m2, u, cmul(m3, v));
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
            C x[4], y[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = P[ix[k]], y[k] = Q[ix[k]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C s = cmul(m[4 * r], x[0]), t = cmul(m[4 * r], y[0]);
#pragma unroll
                for (int c = 1; c < 4; ++c) s = cfma(m[4 * r + c], x[c], s), t = cfma(m[4 * r + c], y[c], t);
                P[ix[r]] = s;
                Q[ix[r]] = t;
            }
        }
    } else if (op.kind == OPK_PARITY2) {
        const int a = op.lb[0], b = op.lb[1];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        // flipped members: s = 1, 2 exchange the even (00, 11) and odd (01, 10)
        // blocks, s = 2, 3 reverse each block
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
            C v0 = P[i0], v1 = P[i1], v2 = P[i2], v3 = P[i3];
            P[i0] = cfma(e0, v0, cmul(e1, v3));
            P[i3] = cfma(e2, v0, cmul(e3, v3));
            P[i1] = cfma(o0, v1, cmul(o1, v2));
            P[i2] = cfma(o2, v1, cmul(o3, v2));
            v0 = Q[i0], v1 = Q[i1], v2 = Q[i2], v3 = Q[i3];
            Q[i0] = cfma(e0, v0, cmul(e1, v3));
            Q[i3] = cfma(e2, v0, cmul(e3, v3));
            Q[i1] = cfma(o0, v1, cmul(o1, v2));
            Q[i2] = cfma(o2, v1, cmul(o3, v2));
        }
    } else if (op.kind == OPK_DIAG) {
        // table index m = the op's qubit bits; qubits outside the tile are fixed by base
        int sh[4] = {0, 0, 0, 0}, in = 0, cm = 0;
        for (int t = 0; t < op.nq; ++t) {
            if (op.lb[t] >= 0) sh[t] = op.lb[t], in |= 1 << t;
            else cm |= (int)((base >> op.gb[t]) & 1) << t;
        }
        if (tid < 16) dco[tid] = coef<R>(op, (int)tid);
        __syncthreads();
        for (uint32_t j = tid; j < (1u << T); j += nthr) {
            int m = cm;
#pragma unroll
            for (int t = 0; t < 4; ++t) m |= (int)((j >> sh[t]) & (uint32_t)(in >> t) & 1u) << t;
            const C c = dco[m];
            P[j] = cmul(c, P[j]);
            Q[j] = cmul(c, Q[j]);
        }
    } else {  // OPK_MONO
        sweep_op<R, uint32_t>(op, P, T, op.lb, tid, nthr);
        sweep_op<R, uint32_t>(op, Q, T, op.lb, tid, nthr);
    }
}

// weights of a monomial entry i^code: Im(conj(l) i^code p) = wi Im z + wr Re z, z = conj(l) p
template <typename R>
__device__ __forceinline__ void code_weights(int code, R& wr, R& wi) {
    wi = code == 0 ? R(1) : code == 2 ? R(-1) : R(0);
    wr = code == 1 ? R(1) : code == 3 ? R(-1) : R(0);
}

template <typename R>
__device__ __forceinline__ R im_term(typename CT<R>::T l, typename CT<R>::T p, R wr, R wi) {
    const R zr = fma(l.x, p.x, l.y * p.y);
    const R zi = fma(l.x, p.y, -l.y * p.x);
    return fma(wi, zi, wr * zr);
}

template <typename C>
__device__ __forceinline__ C pick4(const C* v, int c) {
    return (c & 2) ? ((c & 1) ? v[3] : v[2]) : ((c & 1) ? v[1] : v[0]);
}

// this thread's share of Im<lambda|G|phi> over the tile pair, G a signed
// monomial on 1 or 2 tile bits; PRE: the op's dense matrix is applied to both
// tiles first (and written back)
template <typename R, int NQ, bool PRE, bool PREDIAG = false>
__device__ __forceinline__ R inner_pairs(const DevOp& op, typename CT<R>::T* P, typename CT<R>::T* Q, int T) {
    using C = typename CT<R>::T;
    constexpr int D = 1 << NQ;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const int a = op.lb[0], b = NQ == 2 ? op.lb[1] : 0;
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    // member k of this thread's groups is logical member k ^ f (bank spreading)
    const int f = lane_flip<R>(tid, a, NQ == 2 ? b : -1);
    const uint32_t fb = flip_bits(f, a, b);
    R wr[D], wi[D];
    int col[D];
#pragma unroll
    for (int r = 0; r < D; ++r) code_weights<R>(op.slot[r ^ f], wr[r], wi[r]), col[r] = op.perm[1 + (r ^ f)] ^ f;
    C m[D * D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) m[k] = PRE ? coef<R>(op, (((k / D) ^ f) * D) + ((k % D) ^ f)) : C{};
    R acc = 0;
    for (uint32_t g = tid; g < (1u << (T - NQ)); g += nthr) {
        uint32_t ix[D];
        if (NQ == 1) {
            ix[0] = ins0<uint32_t>(g, a) ^ fb;
            ix[D - 1] = ix[0] ^ (1u << a);
        } else {
            const uint32_t i0 = ins0<uint32_t>(ins0<uint32_t>(g, lo), hi) ^ fb;
            ix[0] = i0;
            ix[1 % D] = i0 ^ (1u << a);
            ix[2 % D] = i0 ^ (1u << b);
            ix[D - 1] = i0 ^ (1u << a) ^ (1u << b);
        }
        C p[D], l[D];
#pragma unroll
        for (int k = 0; k < D; ++k) p[k] = P[ix[k]], l[k] = Q[ix[k]];
        if (PRE) {
            C x[D], y[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                if (PREDIAG) {  // (a phase per member: the off-diagonal products are zero)
                    x[r] = cmul(m[r * D + r], p[r]);
                    y[r] = cmul(m[r * D + r], l[r]);
                    continue;
                }
                x[r] = cmul(m[r * D], p[0]);
                y[r] = cmul(m[r * D], l[0]);
#pragma unroll
                for (int c = 1; c < D; ++c) x[r] = cfma(m[r * D + c], p[c], x[r]), y[r] = cfma(m[r * D + c], l[c], y[r]);
            }
#pragma unroll
            for (int k = 0; k < D; ++k) p[k] = x[k], l[k] = y[k], P[ix[k]] = x[k], Q[ix[k]] = y[k];
        }
#pragma unroll
        for (int r = 0; r < D; ++r) {
            const C pc = D == 2 ? (col[r] ? p[D - 1] : p[0]) : pick4(p, col[r]);
            acc += im_term<R>(l[r], pc, wr[r], wi[r]);
        }
    }
    return acc;
}

// warp sum of one measurement, added to this warp's row of the partials
template <typename R>
__device__ __forceinline__ void inner_flush(R acc, const AdjArgs& A, int col) {
    double x = (double)acc;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
    if ((threadIdx.x & 31) == 0) {
        const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (SMOQ_INBOUNDS(col >= 0 && col < A.n_cols && row < A.n_rows, A.a.err, 4))
            atomicAdd(&A.partials[row * A.n_cols + col], x);
    }
}

// descriptor of a real-diagonal measurement for the run sweep: lb0 | lb1 << 5 |
// negative rows << 10 | zero rows << 14, rows indexed b(lb0) + 2 b(lb1) (a
// 1-qubit op uses lb1 = lb0: rows 0 and 3)
__device__ __forceinline__ uint32_t diag_desc(const DevOp& op) {
    const uint32_t l0 = (uint32_t)op.lb[0], l1 = op.nq == 2 ? (uint32_t)op.lb[1] : l0;
    uint32_t neg = 0, zero = 0;
    for (int r = 0; r < (1 << op.nq); ++r) {
        const int row = op.nq == 2 ? r : 3 * r;
        if (op.slot[r] == 2) neg |= 1u << row;
        if (op.slot[r] == INNER_ZERO) zero |= 1u << row;
    }
    return l0 | l1 << 5 | neg << 10 | zero << 14;
}

constexpr int kDiagRun = 8;  // real-diagonal measurements folded into one sweep

// The backward program of one tile pair (phi in tP, lambda in tL, 2^T amplitudes
// each, in shared memory): U^dag ops on both, measurements through flush(acc, column)
template <typename R, typename Flush>
__device__ __forceinline__ void adj_program(const DevOp* ops, int nops, typename CT<R>::T* tP, typename CT<R>::T* tL,
                                            int T, uint64_t base, typename CT<R>::T* dco, Flush flush) {
    using C = typename CT<R>::T;
    const int tid = threadIdx.x;
    const uint32_t amps = 1u << T;
    for (int o = 0; o < nops;) {
        const DevOp& op = ops[o];
        bool writes = true;
        if (op.kind == OPK_INNER && op.flags == INNER_DIAGG) {
            // a run of real-diagonal measurements (RZ, RZZ generators): one read
            // of both tiles, Im(conj(l) p) signed per measurement
            int k = 1;
            while (k < kDiagRun && o + k < nops && ops[o + k].kind == OPK_INNER &&
                   ops[o + k].flags == INNER_DIAGG)
                ++k;
            uint32_t d[kDiagRun];
            R acc[kDiagRun];
#pragma unroll
            for (int u = 0; u < kDiagRun; ++u) acc[u] = 0, d[u] = u < k ? diag_desc(ops[o + u]) : 0u;
            for (uint32_t j = tid; j < amps; j += blockDim.x) {
                const C p = tP[j], l = tL[j];
                const R zi = fma(l.x, p.y, -l.y * p.x);
#pragma unroll
                for (int u = 0; u < kDiagRun; ++u) {
                    if (u < k) {
                        const uint32_t r = ((j >> (d[u] & 31)) & 1) | (((j >> ((d[u] >> 5) & 31)) & 1) << 1);
                        const R x = ((d[u] >> (10 + r)) & 1) ? -zi : zi;
                        acc[u] += ((d[u] >> (14 + r)) & 1) ? R(0) : x;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kDiagRun; ++u)
                if (u < k) flush(acc[u], ops[o + u].perm[0]);
            o += k;
            writes = false;
        } else if (op.kind == OPK_INNER) {
            const bool pre = op.flags & INNER_PRE, pd = op.flags & INNER_PREDIAG;
            R acc;
            if (op.nq == 1)
                acc = !pre ? inner_pairs<R, 1, false>(op, tP, tL, T)
                           : pd ? inner_pairs<R, 1, true, true>(op, tP, tL, T) : inner_pairs<R, 1, true>(op, tP, tL, T);
            else
                acc = !pre ? inner_pairs<R, 2, false>(op, tP, tL, T)
                           : pd ? inner_pairs<R, 2, true, true>(op, tP, tL, T) : inner_pairs<R, 2, true>(op, tP, tL, T);
            flush(acc, op.perm[0]);
            writes = pre;
            ++o;
        } else {
            dual_apply<R>(op, tP, tL, T, base, dco);
            ++o;
        }
        // consecutive read-only measurements need no barrier between them
        const bool next_writes = o < nops && !(ops[o].kind == OPK_INNER && !(ops[o].flags & INNER_PRE));
        if (writes || next_writes) __syncthreads();
    }
}

// 2 (complex128) or 3 (complex64) CTAs per SM: one CTA's bulk copies overlap another's sweeps
template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 2) adj_tile_kernel(const AdjArgs A) {
    using C = typename CT<R>::T;
    const TileArgs& a = A.a;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int T = a.g.T, L = a.g.L, H = a.g.H;
    const uint32_t amps = 1u << T;
    C* tP = reinterpret_cast<C*>(smem_raw);
    C* tL = tP + amps;
    __shared__ __align__(8) uint64_t bar;
    __shared__ C dco[16];
    const int tid = threadIdx.x;
    const uint32_t nseg = 1u << H;
    const uint32_t seg_bytes = (uint32_t)sizeof(C) << L;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        uint64_t base = (uint64_t)t << L;
        for (int m = 0; m < H; ++m) base = ins0<uint64_t>(base, a.g.hb[m]);
        C* gP = reinterpret_cast<C*>(a.psi);
        C* gL = reinterpret_cast<C*>(A.lam);
        if (tid == 0) mbar_arrive_expect_tx(&bar, 2u * amps * (uint32_t)sizeof(C));
        for (uint32_t s = tid; s < 2 * nseg; s += blockDim.x) {
            const uint32_t sg = s < nseg ? s : s - nseg;
            uint64_t off = base;
            for (int m = 0; m < H; ++m) off |= (uint64_t)((sg >> m) & 1) << a.g.hb[m];
            if (!SMOQ_INBOUNDS(off + (1ull << L) <= (uint64_t)a.state_len, a.err, 3)) continue;
            if (s < nseg) bulk_g2s(tP + ((size_t)sg << L), gP + off, seg_bytes, &bar);
            else bulk_g2s(tL + ((size_t)sg << L), gL + off, seg_bytes, &bar);
        }
        const bool ok = mbar_wait_bounded(&bar, phase, a.err);
        if (!__syncthreads_and(ok)) {
            mbar_wait_bounded(&bar, phase, nullptr);
            return;
        }
        phase ^= 1;
        adj_program<R>(a.ops, a.nops, tP, tL, T, base, dco,
                       [&](R acc, int col) { inner_flush<R>(acc, A, col); });
        fence_proxy_async_smem();
        __syncthreads();
        for (uint32_t s = tid; s < 2 * nseg; s += blockDim.x) {
            const uint32_t sg = s < nseg ? s : s - nseg;
            uint64_t off = base;
            for (int m = 0; m < H; ++m) off |= (uint64_t)((sg >> m) & 1) << a.g.hb[m];
            if (!SMOQ_INBOUNDS(off + (1ull << L) <= (uint64_t)a.state_len, a.err, 5)) continue;
            if (s < nseg) bulk_s2g(gP + off, tP + ((size_t)sg << L), seg_bytes);
            else bulk_s2g(gL + off, tL + ((size_t)sg << L), seg_bytes);
        }
        bulk_commit();
        bulk_wait_read0();
        __syncthreads();
    }
    bulk_wait0();
}

// partial columns summed over rows: out[c] = sum_r part[r][c]; a block of
// 32 x 32 threads takes 32 columns, its 32 row lanes stride over the rows
__global__ void __launch_bounds__(1024) adj_colsum_kernel(const double* part, int64_t rows, int32_t cols, double* out) {
    __shared__ double red[32][33];
    const int lane = threadIdx.x & 31, rl = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    double s = 0;
    if (c < cols)
#pragma unroll 4
        for (int64_t r = rl; r < rows; r += 32) s += part[r * cols + c];
    red[rl][lane] = s;
    __syncthreads();
    if (rl == 0 && c < cols) {
        double t = 0;
        for (int k = 0; k < 32; ++k) t += red[k][lane];
        out[c] = t;
    }
}

// ---------------------------------------------------------------- many small circuits, one launch
// A circuit whose two states (phi, lambda) fit one CTA's shared memory runs
// entirely there: forward program, lambda = H phi and the energy, then the
// backward program; one CTA per circuit.  The CTAs are persistent and take
// circuits off a device work queue (an atomic counter over the jobs, sorted by
// cost, largest first), so uneven circuits balance across the SMs.
struct ResJob {
    int32_t N;
    int32_t fwd_off, fwd_n;  // forward ops (whole-state tile)
    int32_t bwd_off, bwd_n;  // backward ops (whole-state tile pair)
    int32_t term_off, nterms;
    int32_t col_off;         // first gradient column of the job
};
struct ResArgs {
    const ResJob* jobs;
    const DevOp* ops;
    const HamTerm* terms;
    double* energy;  // [njobs], <phi|H|phi> / <phi|phi>
    double* norm2;   // [njobs], <phi|phi>
    double* cols;    // [columns of all jobs], zeroed
    const int32_t* order;  // the queue: job indices, largest cost first
    int32_t* next;         // queue head, zeroed
    int32_t njobs;
};

template <typename R>
__device__ __forceinline__ void res_apply(const DevOp& op, typename CT<R>::T* psi, int N, typename CT<R>::T* dco) {
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
        sweep_op_spread<R>(op, psi, N, tid, nthr);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) vqe_resident_kernel(const ResArgs A) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ C dco[16];
    __shared__ double red[2][8];
    __shared__ int32_t s_job;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_job = atomicAdd(A.next, 1);
        __syncthreads();  // (the job's last barrier keeps thread 0 from overwriting s_job early)
        if (s_job >= A.njobs) break;
        const int j = A.order[s_job];
        const ResJob J = A.jobs[j];
        const uint32_t dim = 1u << J.N;
        C* P = reinterpret_cast<C*>(smem_raw);
        C* Q = P + dim;
        for (uint32_t a = tid; a < dim; a += blockDim.x) {
            C z;
            z.x = (R)(a == 0 ? 1 : 0);
            z.y = (R)0;
            P[a] = z;
        }
        __syncthreads();
        for (int o = 0; o < J.fwd_n; ++o) {
            res_apply<R>(A.ops[J.fwd_off + o], P, J.N, dco);
            __syncthreads();
        }
        // lambda = H phi, Re <phi|lambda> and <phi|phi> (the pull rule of ham_apply_kernel)
        double acc = 0, nrm = 0;
        for (uint32_t k = tid; k < dim; k += blockDim.x) {
            double lr = 0, li = 0;
            for (int t = 0; t < J.nterms; ++t) {
                const HamTerm& h = A.terms[J.term_off + t];
                const uint32_t i = k ^ (uint32_t)h.x;
                const C p = P[i];
                const double sg = h.coef * ((__popc(i & (uint32_t)h.z) & 1) ? -1.0 : 1.0);
                const int yk = h.ny & 3;
                double pr = p.x, pi = p.y;
                if (yk == 1) { const double tr = -pi; pi = pr; pr = tr; }
                else if (yk == 2) { pr = -pr; pi = -pi; }
                else if (yk == 3) { const double tr = pi; pi = -pr; pr = tr; }
                lr += sg * pr;
                li += sg * pi;
            }
            C o;
            o.x = (R)lr;
            o.y = (R)li;
            Q[k] = o;
            const C f = P[k];
            acc += (double)f.x * lr + (double)f.y * li;
            nrm += (double)f.x * f.x + (double)f.y * f.y;
        }
        for (int d = 16; d > 0; d >>= 1) {
            acc += __shfl_xor_sync(0xffffffffu, acc, d);
            nrm += __shfl_xor_sync(0xffffffffu, nrm, d);
        }
        if (lane == 0) red[0][warp] = acc, red[1][warp] = nrm;
        __syncthreads();
        if (tid == 0) {
            // E = <phi|H|phi> / <phi|phi>; the host divides the gradient columns by <phi|phi>
            double e = 0, n = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) e += red[0][w], n += red[1][w];
            A.energy[j] = e / n;
            A.norm2[j] = n;
        }
        adj_program<R>(A.ops + J.bwd_off, J.bwd_n, P, Q, J.N, 0, dco, [&](R a, int col) {
            double x = (double)a;
            for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
            if (lane == 0) atomicAdd(&A.cols[J.col_off + col], x);
        });
        __syncthreads();
    }
}

}  // namespace smoq

using namespace smoq;

smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg);
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where);
smoq_status smoq_internal_ops_to_ir(int N, const smoq_op* ops, int n, const double* theta, std::vector<GateIR>& out);
smoq_status smoq_internal_prepare(smoq_ctx* ctx, smoq_state* st, const std::vector<GateIR>& gates,
                                  int epilogue_special, bool reusable, void** prog_handle,
                                  bool variational = false);
std::vector<Pass> smoq_internal_plan(smoq_ctx* ctx, int N, int dtype, const std::vector<GateIR>& gates,
                                     bool variational);
smoq_status smoq_internal_prepare_planned(smoq_ctx* ctx, std::vector<Pass>&& passes, void** handle);
void smoq_internal_cap_fusion_depth(std::vector<Pass>& pl, int cap);
smoq_status smoq_internal_rerun(smoq_ctx* ctx, smoq_state* st, void* prog_handle, const Epilogue* ep);
void smoq_internal_free_prog(void* prog_handle);
int smoq_internal_tile_bits(smoq_ctx* ctx, int dtype);
int smoq_internal_low_bits(smoq_ctx* ctx, int dtype);

#define VCK(call)                                                         \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return smoq_internal_cuda(ctx, e_, #call); \
    } while (0)

namespace {

// generator G of a parameterised gate, as a dense matrix on the gate's qubits
// (index bit t = the gate's qubit t); false if the gate type has no generator
bool generator(int type, GateIR& g) {
    const cd I(0.0, 1.0);
    const int dim = g.nq == 1 ? 2 : 4;
    for (int k = 0; k < dim * dim; ++k) g.m[k] = 0.0;
    switch (type) {
        case SMOQ_G_RX: g.m[1] = 1; g.m[2] = 1; return true;
        case SMOQ_G_RY: g.m[1] = -I; g.m[2] = I; return true;
        case SMOQ_G_RZ: g.m[0] = 1; g.m[3] = -1; return true;
        case SMOQ_G_RXX:
            for (int m = 0; m < 4; ++m) g.m[m * 4 + (m ^ 3)] = 1;
            return true;
        case SMOQ_G_RYY:
            g.m[0 * 4 + 3] = -1; g.m[3 * 4 + 0] = -1; g.m[1 * 4 + 2] = 1; g.m[2 * 4 + 1] = 1;
            return true;
        case SMOQ_G_RZZ:
            g.m[0] = 1; g.m[5] = -1; g.m[10] = -1; g.m[15] = 1;
            return true;
        case SMOQ_G_CRY:  // |1><1| on the control (bit 0) times Y on the target (bit 1)
            g.m[1 * 4 + 3] = -I; g.m[3 * 4 + 1] = I;
            return true;
        default: return false;
    }
}

// d = g^dag, written into a freshly constructed d (only the 2^nq x 2^nq block of
// the 256-entry matrix is touched: a gate list holds thousands of these)
void dagger_into(const GateIR& g, GateIR& d) {
    d.nq = g.nq;
    for (int t = 0; t < 4; ++t) d.q[t] = g.q[t];
    d.diag = g.diag;
    d.special = g.special;
    d.aux = g.aux;
    d.aux2 = g.aux2;
    d.tag = g.tag;
    const int dim = 1 << g.nq;
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) d.m[r * dim + c] = std::conj(g.m[c * dim + r]);
}

// shared memory of the widest adjoint tile: two states of 2^13 complex64 or 2^12
// complex128 amplitudes (tile widths up to 14 / 13, one bit narrower for two states)
constexpr size_t kAdjMaxSmem = (size_t)2 * 8 << 13;
static_assert(((size_t)2 * 16 << 12) == kAdjMaxSmem, "same limit for both precisions");

struct Work {
    smoq_state phi, lam;
    std::vector<void*> owned;
    cudaStream_t s;
    ~Work() {
        for (void* p : owned) cudaFreeAsync(p, s);
    }
};

constexpr int kAdjThreads = 256;  // the adjoint kernel's __launch_bounds__
// circuits with both states in one CTA's shared memory: 2 x 2^13 complex64 or
// 2 x 2^12 complex128 = 128 KB
constexpr int kResMaxN64 = 13, kResMaxN128 = 12;
constexpr size_t kResMaxSmem = (size_t)2 * 8 << kResMaxN64;
static_assert(((size_t)2 * 16 << kResMaxN128) == kResMaxSmem, "same limit for both precisions");

// dense row-major matrix of a 1- or 2-qubit U^dag op (false: not a dense/diagonal kind)
bool op_dense(const DevOp& op, cd* M) {
    const int dim = 1 << op.nq;
    for (int k = 0; k < dim * dim; ++k) M[k] = 0.0;
    auto c = [&](int k) { return cd(op.cd[k].x, op.cd[k].y); };
    switch (op.kind) {
        case OPK_DENSE1:
        case OPK_DENSE2:
            for (int k = 0; k < dim * dim; ++k) M[k] = c(k);
            return true;
        case OPK_DIAG:
            for (int k = 0; k < dim; ++k) M[k * dim + k] = c(k);
            return true;
        case OPK_PARITY2:  // even block on local indices (0, 3), odd block on (1, 2)
            M[0] = c(0); M[3] = c(1); M[12] = c(2); M[15] = c(3);
            M[5] = c(4); M[6] = c(5); M[9] = c(6); M[10] = c(7);
            return true;
        default: return false;
    }
}

// Fold a U^dag op that directly precedes a measurement on the same tile bits
// into the measurement (INNER_PRE): one sweep of both tiles instead of two.
smoq_status fuse_measurements(std::vector<DevOp>& ops, std::string& err) {
    for (const DevOp& op : ops) {
        const bool ok = op.kind == OPK_DENSE1 || op.kind == OPK_DENSE2 || op.kind == OPK_PARITY2 ||
                        op.kind == OPK_MONO || op.kind == OPK_DIAG || op.kind == OPK_INNER;
        if (!ok) {
            err = "adjoint pass holds an unsupported op kind";
            return SMOQ_ERR_UNSUPPORTED;
        }
        if (op.kind == OPK_INNER)
            for (int t = 0; t < op.nq; ++t)
                if (op.lb[t] < 0) {
                    err = "measurement qubit outside the tile";
                    return SMOQ_ERR_BADINPUT;
                }
    }
    std::vector<DevOp> out;
    out.reserve(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) {
        if (i + 1 < ops.size() && ops[i + 1].kind == OPK_INNER && ops[i].nq == ops[i + 1].nq) {
            const DevOp& u = ops[i];
            DevOp m = ops[i + 1];
            const int nq = m.nq;
            const bool same = u.lb[0] == m.lb[0] && (nq == 1 || u.lb[1] == m.lb[1]);
            const bool swapped = nq == 2 && u.lb[0] == m.lb[1] && u.lb[1] == m.lb[0];
            cd M[16];
            if ((same || swapped) && u.lb[0] >= 0 && op_dense(u, M)) {
                const int dim = 1 << nq;
                auto sw = [&](int k) { return swapped ? (((k & 1) << 1) | (k >> 1)) : k; };
                for (int r = 0; r < dim; ++r)
                    for (int c = 0; c < dim; ++c) {
                        const cd x = M[sw(r) * dim + sw(c)];
                        m.cd[r * dim + c] = make_double2(x.real(), x.imag());
                        m.cf[r * dim + c] = make_float2((float)x.real(), (float)x.imag());
                    }
                bool diag = true;
                for (int r = 0; r < dim; ++r)
                    for (int c = 0; c < dim; ++c)
                        if (r != c && std::abs(M[r * dim + c]) != 0.0) diag = false;
                m.flags = INNER_PRE | (diag ? INNER_PREDIAG : 0);
                out.push_back(m);
                ++i;
                continue;
            }
        }
        out.push_back(ops[i]);
    }
    ops.swap(out);
    return SMOQ_OK;
}

}  // namespace

// CTAs of the adjoint kernel: persistent grid, as many per SM as fit
static int64_t adj_grid(smoq_ctx* ctx, smoq_dtype dtype, int64_t ntiles, size_t smem) {
    int per_sm = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, dtype == SMOQ_C64 ? (const void*)adj_tile_kernel<float> : (const void*)adj_tile_kernel<double>,
        kAdjThreads, smem);
    if (e != cudaSuccess) (void)cudaGetLastError();
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    return std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)ctx->num_sms * per_sm));
}

static smoq_status check_vqe_args(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n, int n_params,
                                  const smoq_pauli_term* H, int nterms, int batch, const double* theta) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    if (N < 1 || N > 34) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "N must be in 1..34");
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad dtype");
    if (n < 0 || (n > 0 && !ops) || n_params < 0 || (n_params > 0 && !theta) || nterms < 1 || !H || batch < 1)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad VQE arguments");
    const uint64_t lim = (1ull << N) - 1;
    for (int t = 0; t < nterms; ++t)
        if ((H[t].xmask | H[t].zmask) & ~lim)
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "Hamiltonian term acts beyond N");
    for (int i = 0; i < n; ++i)
        if (ops[i].param >= n_params) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "op param index >= n_params");
    return SMOQ_OK;
}

// forward state into w.phi, lambda = H phi into w.lam; returns
// E = <phi|H|phi> / <phi|phi> and the FP64 <phi|phi> it divided by (a unitary
// circuit keeps the norm at 1 in exact arithmetic; dividing removes the
// complex64 norm drift of a deep circuit from the energy at first order).
// compiled: the forward runs compiled kernels with run-time coefficients (one
// compile per circuit structure, for repeated calls on one circuit); fwd: the
// forward passes when a planning thread made them already (moved from)
static smoq_status forward_and_h(smoq_ctx* ctx, Work& w, const std::vector<GateIR>& ir, const std::vector<HamTerm>& ht,
                                 HamTerm* d_terms, double* d_epart, int eblocks, double* E, double* nrm2,
                                 bool compiled, std::vector<Pass>* fwd = nullptr) {
    VCK(launch_set_basis(&w.phi, 0));
    if (!ir.empty()) {
        void* h = nullptr;
        if (smoq_status s = fwd ? smoq_internal_prepare_planned(ctx, std::move(*fwd), &h)
                                : smoq_internal_prepare(ctx, &w.phi, ir, -1, false, &h, compiled))
            return s;
        std::unique_ptr<void, void (*)(void*)> hold(h, smoq_internal_free_prog);
        if (smoq_status s = smoq_internal_rerun(ctx, &w.phi, h, nullptr)) return s;
        VCK(cudaStreamSynchronize(ctx->stream));  // the program is freed at scope exit
    }
    if (w.phi.dtype == SMOQ_C64)
        ham_apply_kernel<float><<<eblocks, 256, 0, ctx->stream>>>((const float2*)w.phi.ptr, (float2*)w.lam.ptr,
                                                                  w.phi.N, d_terms, (int)ht.size(), d_epart);
    else
        ham_apply_kernel<double><<<eblocks, 256, 0, ctx->stream>>>((const double2*)w.phi.ptr, (double2*)w.lam.ptr,
                                                                   w.phi.N, d_terms, (int)ht.size(), d_epart);
    ctx->launches++;
    VCK(cudaGetLastError());
    std::vector<double> ep(2 * (size_t)eblocks);
    VCK(cudaMemcpyAsync(ep.data(), d_epart, ep.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    double e = 0, n = 0;
    for (int k = 0; k < eblocks; ++k) e += ep[k], n += ep[eblocks + k];
    if (!(n > 0)) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "VQE: the circuit's state has zero norm");
    *E = e / n;
    *nrm2 = n;
    return SMOQ_OK;
}

// The backward program of a circuit: for k = n-1 .. 0, [the measurement of
// G_k when gate k is parameterised] then U_k^dag.  inner_param[m] = the
// parameter of measurement m.  False (with err) for a parameterised gate type
// that has no generator.
static bool build_backward(const std::vector<GateIR>& ir, const smoq_op* ops, int n, std::vector<GateIR>& back,
                           std::vector<int>& inner_param, std::string& err) {
    back.reserve(2 * (size_t)n);
    for (int k = n - 1; k >= 0; --k) {
        if (ops[k].param >= 0) {
            back.emplace_back();
            GateIR& gi = back.back();
            gi.nq = ir[k].nq;
            for (int t = 0; t < gi.nq; ++t) gi.q[t] = ir[k].q[t];
            if (!generator(ops[k].type, gi)) {
                err = "adjoint gradient: parameterised gate type has no generator";
                return false;
            }
            gi.special = OPK_INNER;
            gi.aux2 = (int64_t)inner_param.size();
            inner_param.push_back(ops[k].param);
        }
        back.emplace_back();
        dagger_into(ir[k], back.back());
    }
    return true;
}

// Host-only preparation of one parameter set: the gate IR and, for a gradient,
// the backward program planned into fused tile passes.  Touches no context
// state, so the many-circuit call prepares several circuits on host threads.
struct GradPlan {
    std::vector<GateIR> ir;
    std::vector<Pass> fwd;       // the forward passes, when planned ahead (fwd_ready)
    bool fwd_ready = false;
    std::vector<Pass> passes;    // the backward passes, measurements fused
    std::vector<Pass> staged;    // per pass: its stage schedule when the compiled adjoint
                                 // kernel runs it (staged[i].staged false: the shared-memory kernel)
    std::vector<std::vector<int32_t>> sig;   // ... that kernel's signature
    std::vector<std::string> src;            // ... and source (empty when it is loaded already)
    std::vector<std::vector<float2>> coefs;  // ... and its run-time coefficients
    std::vector<int> inner_param;  // measurement -> parameter
    smoq_status status = SMOQ_OK;
    std::string error;
};
// jit (1, 2): complex64 backward passes of tile width 12 get the compiled adjoint
// kernel (4-bit register stages on both states, coefficients read at run time, so
// the NVRTC compile of the first parameter set serves all later ones); with jit = 1
// they are compiled here, on the planning thread, and loaded by the caller
// fwd_ctx: also plan the forward (on fwd_ctx's options; a variational forward with jit 1);
// max_ops: at most that many fused ops per backward pass (0: as many as fit)
static void plan_gradient_impl(int N, smoq_dtype dtype, int tile_bits, int low_bits, const smoq_op* ops, int n,
                               const double* th, bool grad, GradPlan& gp, int jit, smoq_ctx* fwd_ctx, int max_ops) {
    if ((gp.status = smoq_internal_ops_to_ir(N, ops, n, th, gp.ir))) {
        gp.error = "bad op list";
        return;
    }
    if (fwd_ctx && !gp.ir.empty()) {
        try {
            gp.fwd = smoq_internal_plan(fwd_ctx, N, dtype, gp.ir, jit == 1);
            gp.fwd_ready = true;
        } catch (const std::exception& ex) {
            gp.status = SMOQ_ERR_BADINPUT;
            gp.error = ex.what();
            return;
        }
    }
    if (!grad) return;
    std::vector<GateIR> back;
    if (!build_backward(gp.ir, ops, n, back, gp.inner_param, gp.error)) {
        gp.status = SMOQ_ERR_UNSUPPORTED;
        return;
    }
    if (gp.inner_param.empty()) return;
    // tiles for two states in shared memory: one qubit narrower than the single-state passes
    const int T = std::max(tile_bits - 1, 6);
    try {
        gp.passes = plan_passes(back, N, T, low_bits, -1, dtype == SMOQ_C64 ? 1 : 0);
        smoq_internal_cap_fusion_depth(gp.passes, max_ops);
    } catch (const std::exception& ex) {
        gp.status = SMOQ_ERR_BADINPUT;
        gp.error = ex.what();
        return;
    }
    gp.staged.assign(gp.passes.size(), Pass());
    gp.src.assign(gp.passes.size(), std::string());
    gp.sig.assign(gp.passes.size(), std::vector<int32_t>());
    gp.coefs.assign(gp.passes.size(), std::vector<float2>());
    if (jit && dtype == SMOQ_C64) {
        std::vector<const std::string*> todo;
        for (size_t i = 0; i < gp.passes.size(); ++i) {
            Pass q = gp.passes[i];  // (before the measurements are fused)
            q.rtc = true;
            schedule_stages(q, 8, true);
            if (!q.staged || q.g.T != 12) continue;
            std::vector<float2> blk;  // the coefficients must fit the kernel parameter space
            jit_rtc_block(q, blk);
            if (sizeof(AdjArgs) + sizeof(float2) * blk.size() > kMaxKernelParamBytes) continue;
            std::vector<int32_t> sig = jit_pass_signature(q);
            if (jit == 1 && jit_sig_find(sig)) {  // a later parameter set of a known circuit
                gp.staged[i] = std::move(q);
                gp.sig[i] = std::move(sig);
                gp.coefs[i] = std::move(blk);
                continue;
            }
            std::string err;
            std::string src = jit_adjoint_source(q, err);
            if (src.empty()) continue;  // (an op the compiled kernel does not take)
            gp.staged[i] = std::move(q);
            gp.sig[i] = std::move(sig);
            gp.src[i] = std::move(src);
            gp.coefs[i] = std::move(blk);
            todo.push_back(&gp.src[i]);
        }
        if (jit == 1) jit_precompile_sources(todo);
    }
    for (Pass& p : gp.passes)
        if ((gp.status = fuse_measurements(p.ops, gp.error))) return;
}
// (planning threads and the C entry points: a failure is a status, never an exception)
static void plan_gradient(int N, smoq_dtype dtype, int tile_bits, int low_bits, const smoq_op* ops, int n,
                          const double* th, bool grad, GradPlan& gp, int jit = 0, smoq_ctx* fwd_ctx = nullptr,
                          int max_ops = 0) {
    try {
        plan_gradient_impl(N, dtype, tile_bits, low_bits, ops, n, th, grad, gp, jit, fwd_ctx, max_ops);
    } catch (const std::exception& ex) {
        gp.status = SMOQ_ERR_BADINPUT;
        gp.error = ex.what();
    }
}

static smoq_status vqe_run(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n, int n_params,
                           const smoq_pauli_term* H, int nterms, int batch, const double* theta, double* energies,
                           double* grads, GradPlan* pre = nullptr) {
    if (smoq_status s = check_vqe_args(ctx, N, dtype, ops, n, n_params, H, nterms, batch, theta)) return s;
    Work w;
    w.s = ctx->stream;
    for (smoq_state* st : {&w.phi, &w.lam}) {
        st->ctx = ctx;
        st->N = N;
        st->dtype = dtype;
        st->batch = 1;
        st->owned = false;
        VCK(cudaMallocAsync(&st->ptr, st->bytes(), ctx->stream));
        w.owned.push_back(st->ptr);
    }
    std::vector<HamTerm> ht(nterms);
    for (int t = 0; t < nterms; ++t) {
        ht[t].coef = H[t].coef;
        ht[t].x = H[t].xmask;
        ht[t].z = H[t].zmask;
        ht[t].ny = __builtin_popcountll(H[t].xmask & H[t].zmask);
    }
    HamTerm* d_terms;
    VCK(cudaMallocAsync((void**)&d_terms, ht.size() * sizeof(HamTerm), ctx->stream));
    w.owned.push_back(d_terms);
    VCK(cudaMemcpyAsync(d_terms, ht.data(), ht.size() * sizeof(HamTerm), cudaMemcpyHostToDevice, ctx->stream));
    const int64_t len = (int64_t)1 << N;
    const int eblocks = (int)std::max<int64_t>(1, std::min<int64_t>((len + 255) / 256, (int64_t)ctx->num_sms * 8));
    double* d_epart;  // energy partials, then norm partials
    VCK(cudaMallocAsync((void**)&d_epart, 2 * (size_t)eblocks * sizeof(double), ctx->stream));
    w.owned.push_back(d_epart);

    // the next parameter set is prepared on a host thread while this one runs
    const int tb = smoq_internal_tile_bits(ctx, dtype), lbits = smoq_internal_low_bits(ctx, dtype);
    const int jit = (ctx->engine == 3 || (ctx->engine < 0 && jit_available())) ? 1 : 0;
    auto theta_of = [&](int b) { return theta ? theta + (size_t)b * n_params : nullptr; };
    const bool use_pre = pre && batch == 1;
    // Parameter sets are planned (forward and backward) on host threads, up to
    // `window` sets ahead of the one the GPU runs; each plan holds one set's gate IR
    // and pass lists and is freed once its set ran
    const int window = std::max(1, std::min(batch, (int)std::min<unsigned>(8, std::thread::hardware_concurrency())));
    std::vector<std::unique_ptr<GradPlan>> plans(batch);
    std::vector<std::future<void>> planned(batch);  // (declared after `plans`: joined first)
    const bool want_grad = grads != nullptr;
    const int depth = ctx->fusion_depth;
    auto start = [&](int b) {
        plans[b].reset(new GradPlan);
        GradPlan* np = plans[b].get();
        const double* th = theta_of(b);
        planned[b] = std::async(std::launch::async,
                                [=]() { plan_gradient(N, dtype, tb, lbits, ops, n, th, want_grad, *np, jit, ctx, depth); });
    };
    // set 0 alone first: a new circuit structure is compiled once, by its planning
    if (!use_pre) start(0);
    for (int b = 0; b < batch; ++b) {
        if (!use_pre) {
            planned[b].get();
            if (b > 0) plans[b - 1].reset();
            for (int k = b == 0 ? 1 : b + window; k <= b + window && k < batch; ++k) start(k);
        }
        GradPlan& gp = use_pre ? *pre : *plans[b];
        if (gp.status) return smoq_internal_fail(ctx, gp.status, gp.error.c_str());
        double E = 0, nrm2 = 1;
        // (the many-circuit call keeps its distinct circuits off the compiler)
        if (smoq_status s = forward_and_h(ctx, w, gp.ir, ht, d_terms, d_epart, eblocks, &E, &nrm2, jit && !use_pre,
                                          gp.fwd_ready ? &gp.fwd : nullptr))
            return s;
        energies[b] = E;
        if (!grads) continue;
        double* g = grads + (size_t)b * n_params;
        for (int p = 0; p < n_params; ++p) g[p] = 0.0;
        if (gp.inner_param.empty()) continue;
        const std::vector<int>& inner_param = gp.inner_param;
        std::vector<Pass>& passes = gp.passes;
        std::vector<size_t> opoff(passes.size() + 1, 0);
        std::vector<int64_t> grid(passes.size(), 0);
        std::vector<const JitKernel*> kern(passes.size(), nullptr);
        std::vector<DevOp> all;
        int64_t max_rows = 1;
        for (size_t i = 0; i < passes.size(); ++i) {
            const int64_t ntiles = (int64_t)1 << (N - passes[i].g.T);
            if (gp.staged[i].staged) {  // the compiled adjoint kernel of this pass
                std::string why;
                kern[i] = jit_adjoint_load(gp.staged[i], gp.src[i], gp.sig[i], why);
                if (!kern[i]) return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, ("compiled adjoint kernel: " + why).c_str());
                const std::vector<DevOp>& so = gp.staged[i].ops;
                opoff[i + 1] = opoff[i] + so.size();
                all.insert(all.end(), so.begin(), so.end());
                grid[i] = std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)ctx->num_sms * kern[i]->per_sm[0]));
                max_rows = std::max(max_rows, grid[i] * (kern[i]->threads / 32));
                continue;
            }
            opoff[i + 1] = opoff[i] + passes[i].ops.size();
            all.insert(all.end(), passes[i].ops.begin(), passes[i].ops.end());
            const size_t smem = (size_t)2 * w.phi.amp_bytes() << passes[i].g.T;
            if (smem > kAdjMaxSmem) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "adjoint tile too wide");
            grid[i] = adj_grid(ctx, dtype, ntiles, smem);
            max_rows = std::max(max_rows, grid[i] * (kAdjThreads / 32));
        }
        // partials: one row per warp of the widest launch, one column per measurement
        const int32_t ncols = (int32_t)inner_param.size();
        const int64_t nrows = max_rows;
        double *d_part, *d_sum;
        DevOp* d_ops;
        VCK(cudaMallocAsync((void**)&d_part, (size_t)nrows * ncols * sizeof(double), ctx->stream));
        VCK(cudaMallocAsync((void**)&d_sum, (size_t)ncols * sizeof(double), ctx->stream));
        VCK(cudaMallocAsync((void**)&d_ops, std::max<size_t>(1, all.size()) * sizeof(DevOp), ctx->stream));
        VCK(cudaMemsetAsync(d_part, 0, (size_t)nrows * ncols * sizeof(double), ctx->stream));
        VCK(cudaMemcpyAsync(d_ops, all.data(), all.size() * sizeof(DevOp), cudaMemcpyHostToDevice, ctx->stream));
        for (size_t i = 0; i < passes.size(); ++i) {
            const Pass& p = passes[i];
            if (p.ops.empty()) continue;
            AdjArgs A;
            A.a.psi = w.phi.ptr;
            A.a.state_len = len;
            A.a.tiles_per_state = (int64_t)1 << (N - p.g.T);
            A.a.ntiles = A.a.tiles_per_state;
            A.a.ops = d_ops + opoff[i];
            A.a.nops = (int32_t)(opoff[i + 1] - opoff[i]);
            A.a.err = ctx->d_err;
            A.a.g = p.g;
            A.a.ep.partials = nullptr;
            A.a.ep.npop = 0;
            A.lam = w.lam.ptr;
            A.partials = d_part;
            A.n_rows = nrows;
            A.n_cols = ncols;
            const size_t smem = (size_t)2 * w.phi.amp_bytes() << p.g.T;
            if (kern[i]) {
                void* params[] = {&A, gp.coefs[i].data()};  // (the angles of this parameter set)
                VCK(cudaLaunchKernel(kern[i]->fn[0], dim3((unsigned)grid[i]), dim3((unsigned)kern[i]->threads), params,
                                     kern[i]->smem, ctx->stream));
                ctx->launches++;
                ctx->tile_passes++;
                continue;
            }
            // (the kernels' shared-memory limit is set once per context, vqe_kernels_init:
            // setting it per launch would race between contexts driven from several threads)
            if (dtype == SMOQ_C64) adj_tile_kernel<float><<<(unsigned)grid[i], kAdjThreads, smem, ctx->stream>>>(A);
            else adj_tile_kernel<double><<<(unsigned)grid[i], kAdjThreads, smem, ctx->stream>>>(A);
            ctx->launches++;
            ctx->tile_passes++;
            VCK(cudaGetLastError());
        }
        adj_colsum_kernel<<<(unsigned)((ncols + 31) / 32), 1024, 0, ctx->stream>>>(d_part, nrows, ncols, d_sum);
        ctx->launches++;
        VCK(cudaGetLastError());
        std::vector<double> colsum(ncols);
        VCK(cudaMemcpyAsync(colsum.data(), d_sum, (size_t)ncols * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        VCK(cudaFreeAsync(d_part, ctx->stream));
        VCK(cudaFreeAsync(d_sum, ctx->stream));
        VCK(cudaFreeAsync(d_ops, ctx->stream));
        VCK(cudaStreamSynchronize(ctx->stream));
        int32_t herr = 0;
        VCK(cudaMemcpy(&herr, ctx->d_err, sizeof(herr), cudaMemcpyDeviceToHost));
        if (herr) {
            VCK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream));
            if ((herr & 255) == DEVERR_BOUNDS)
                return smoq_internal_fail(ctx, SMOQ_ERR_CUDA,
                                          ("device bounds check failed at site " + std::to_string(herr >> 8)).c_str());
            return smoq_internal_fail(ctx, SMOQ_ERR_TIMEOUT, "a bounded device wait ran out");
        }
        // the gradient of <phi|H|phi> / <phi|phi>: the norm is constant in theta for a
        // unitary circuit, so the raw adjoint sums are divided by the same <phi|phi>
        for (int32_t c = 0; c < ncols; ++c) g[inner_param[c]] += colsum[c] / nrm2;
    }
    return SMOQ_OK;
}

extern "C" smoq_status smoq_debug_compile_adjoint(int N, const smoq_op* ops, int n, int n_params, const double* theta,
                                                  int tile_bits, int low_bits, int flags, int* n_passes,
                                                  int* n_compiled, char* msg, int msg_len) {
    if (N < 1 || N > 34 || n < 0 || (n > 0 && !ops) || n_params < 0 || (n_params > 0 && !theta) || !n_passes ||
        !n_compiled || tile_bits < 7 || tile_bits > 14 || (flags & ~3))
        return SMOQ_ERR_BADINPUT;
    for (int i = 0; i < n; ++i)
        if (ops[i].param >= n_params) return SMOQ_ERR_BADINPUT;
    auto say = [&](const std::string& m) {
        if (msg && msg_len > 0) {
            std::strncpy(msg, m.c_str(), (size_t)msg_len - 1);
            msg[msg_len - 1] = 0;
        }
    };
    *n_passes = *n_compiled = 0;
    if (!jit_available()) {
        say("NVRTC not available");
        return SMOQ_ERR_UNSUPPORTED;
    }
    GradPlan gp;
    plan_gradient(N, SMOQ_C64, tile_bits, low_bits, ops, n, theta, true, gp, 2);
    if (gp.status) {
        say(gp.error);
        return gp.status;
    }
    *n_passes = (int)gp.passes.size();
    std::string report;
    for (size_t i = 0; i < gp.staged.size(); ++i) {
        const Pass& q = gp.staged[i];
        if (!q.staged) continue;
        std::string why, info;
        if (flags & 2) {  // the generated source of the first compiled pass
            *n_compiled = 1;
            say(gp.src[i]);
            return SMOQ_OK;
        }
        if (!jit_check_adjoint(q, why, (flags & 1) ? &info : nullptr)) {
            say(why);
            return SMOQ_ERR_BADINPUT;
        }
        report += info;
        ++*n_compiled;
    }
    say((flags & 1) ? report : std::string("ok"));
    return SMOQ_OK;
}

extern "C" smoq_status smoq_energy_grad(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n,
                                        int n_params, const smoq_pauli_term* H, int nterms, int batch,
                                        const double* theta, double* energies, double* grads) {
    if (!energies || !grads) return ctx ? smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "null output") : SMOQ_ERR_BADINPUT;
    return vqe_run(ctx, N, dtype, ops, n, n_params, H, nterms, batch, theta, energies, grads);
}

extern "C" smoq_status smoq_energy(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n, int n_params,
                                   const smoq_pauli_term* H, int nterms, int batch, const double* theta,
                                   double* energies) {
    if (!energies) return ctx ? smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "null output") : SMOQ_ERR_BADINPUT;
    return vqe_run(ctx, N, dtype, ops, n, n_params, H, nterms, batch, theta, energies, nullptr);
}

// once per context, before any launch (and never during capture)
cudaError_t smoq::vqe_kernels_init(smoq_ctx* ctx) {
    (void)ctx;
    cudaError_t e = cudaFuncSetAttribute(adj_tile_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kAdjMaxSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(adj_tile_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdjMaxSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(vqe_resident_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kResMaxSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(vqe_resident_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kResMaxSmem);
}

// ---------------------------------------------------------------- many small circuits
// the whole-state program of a circuit (one tile spanning every qubit), appended to out
static smoq_status whole_state_ops(smoq_ctx* ctx, const std::vector<GateIR>& gates, int N, int dtype, bool backward,
                                   std::vector<DevOp>& out) {
    if (gates.empty()) return SMOQ_OK;
    std::vector<Pass> passes;
    try {
        passes = plan_passes(gates, N, N, std::min(N, smoq_internal_low_bits(ctx, dtype)), -1, 0);
    } catch (const std::exception& ex) {
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, ex.what());
    }
    for (Pass& p : passes) {
        std::string err;
        if (backward)
            if (smoq_status s = fuse_measurements(p.ops, err)) return smoq_internal_fail(ctx, s, err.c_str());
        for (const DevOp& op : p.ops) {
            const bool kind_ok = op.kind == OPK_DENSE1 || op.kind == OPK_DENSE2 || op.kind == OPK_PARITY2 ||
                                 op.kind == OPK_MONO || op.kind == OPK_DIAG || (backward && op.kind == OPK_INNER);
            bool bits_ok = op.nq >= 0 && op.nq <= 4;
            for (int t = 0; bits_ok && t < op.nq; ++t) bits_ok = op.lb[t] == op.gb[t] && op.lb[t] >= 0 && op.lb[t] < N;
            if (!kind_ok || !bits_ok)
                return smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, "whole-state program: op outside the tile");
            out.push_back(op);
        }
    }
    return SMOQ_OK;
}

// jobs[idx[*]] in one launch of vqe_resident_kernel
static smoq_status run_resident(smoq_ctx* ctx, smoq_dtype dtype, const smoq_vqe_job* jobs, const std::vector<int>& idx) {
    std::vector<ResJob> rj;
    std::vector<DevOp> ops;
    std::vector<HamTerm> terms;
    std::vector<std::vector<int>> inner_param(idx.size());
    int32_t ncols = 0;
    int nmax = 1;
    for (size_t u = 0; u < idx.size(); ++u) {
        const smoq_vqe_job& J = jobs[idx[u]];
        auto job_fail = [&](smoq_status s) {
            const std::string why = "job " + std::to_string(idx[u]) + ": " + smoq_last_error(ctx);
            return smoq_internal_fail(ctx, s, why.c_str());
        };
        if (smoq_status s = check_vqe_args(ctx, J.N, dtype, J.ops, J.n, J.n_params, J.H, J.nterms, 1, J.theta))
            return job_fail(s);
        std::vector<GateIR> ir;
        if (smoq_status s = smoq_internal_ops_to_ir(J.N, J.ops, J.n, J.theta, ir))
            return job_fail(smoq_internal_fail(ctx, s, "bad op list"));
        ResJob r;
        r.N = J.N;
        nmax = std::max(nmax, J.N);
        r.fwd_off = (int32_t)ops.size();
        if (smoq_status s = whole_state_ops(ctx, ir, J.N, dtype, false, ops)) return job_fail(s);
        r.fwd_n = (int32_t)ops.size() - r.fwd_off;
        r.bwd_off = (int32_t)ops.size();
        if (J.grad) {
            std::vector<GateIR> back;
            std::string err;
            if (!build_backward(ir, J.ops, J.n, back, inner_param[u], err))
                return job_fail(smoq_internal_fail(ctx, SMOQ_ERR_UNSUPPORTED, err.c_str()));
            if (!inner_param[u].empty())
                if (smoq_status s = whole_state_ops(ctx, back, J.N, dtype, true, ops)) return job_fail(s);
        }
        r.bwd_n = (int32_t)ops.size() - r.bwd_off;
        r.term_off = (int32_t)terms.size();
        r.nterms = J.nterms;
        for (int t = 0; t < J.nterms; ++t) {
            HamTerm h;
            h.coef = J.H[t].coef;
            h.x = J.H[t].xmask;
            h.z = J.H[t].zmask;
            h.ny = __builtin_popcountll(J.H[t].xmask & J.H[t].zmask);
            h.pad = 0;
            terms.push_back(h);
        }
        r.col_off = ncols;
        ncols += (int32_t)inner_param[u].size();
        rj.push_back(r);
    }
    const int n = (int)rj.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_jobs = al(rj.size() * sizeof(ResJob)), b_ops = al(std::max<size_t>(1, ops.size()) * sizeof(DevOp)),
                 b_terms = al(terms.size() * sizeof(HamTerm)), b_e = al((size_t)n * 8),
                 b_c = al((size_t)std::max(1, ncols) * 8);
    // the queue order: estimated cost (ops x amplitudes), largest first
    std::vector<int32_t> order(rj.size());
    for (size_t u = 0; u < rj.size(); ++u) order[u] = (int32_t)u;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return ((int64_t)rj[a].fwd_n + rj[a].bwd_n + 1) << rj[a].N > ((int64_t)rj[b].fwd_n + rj[b].bwd_n + 1) << rj[b].N;
    });
    const size_t b_q = al((order.size() + 1) * sizeof(int32_t));
    char* buf = nullptr;
    VCK(cudaMallocAsync((void**)&buf, b_jobs + b_ops + b_terms + 2 * b_e + b_c + b_q, ctx->stream));
    std::unique_ptr<char, std::function<void(char*)>> hold(buf, [ctx](char* q) { cudaFreeAsync(q, ctx->stream); });
    ResArgs A;
    char* c = buf;
    A.jobs = (const ResJob*)c;
    VCK(cudaMemcpyAsync(c, rj.data(), rj.size() * sizeof(ResJob), cudaMemcpyHostToDevice, ctx->stream));
    c += b_jobs;
    A.ops = (const DevOp*)c;
    if (!ops.empty()) VCK(cudaMemcpyAsync(c, ops.data(), ops.size() * sizeof(DevOp), cudaMemcpyHostToDevice, ctx->stream));
    c += b_ops;
    A.terms = (const HamTerm*)c;
    VCK(cudaMemcpyAsync(c, terms.data(), terms.size() * sizeof(HamTerm), cudaMemcpyHostToDevice, ctx->stream));
    c += b_terms;
    A.energy = (double*)c;
    c += b_e;
    A.norm2 = (double*)c;
    c += b_e;
    A.cols = (double*)c;
    VCK(cudaMemsetAsync(c, 0, (size_t)std::max(1, ncols) * 8, ctx->stream));
    c += b_c;
    A.next = (int32_t*)c;
    A.order = (const int32_t*)c + 1;
    VCK(cudaMemsetAsync(c, 0, sizeof(int32_t), ctx->stream));
    VCK(cudaMemcpyAsync(c + sizeof(int32_t), order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                        ctx->stream));
    A.njobs = n;
    const size_t amp = dtype == SMOQ_C64 ? 8 : 16;
    const size_t smem = 2 * amp << nmax;
    const void* fn = dtype == SMOQ_C64 ? (const void*)vqe_resident_kernel<float> : (const void*)vqe_resident_kernel<double>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess || per_sm < 1) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    const int grid = (int)std::min<int64_t>(n, (int64_t)ctx->num_sms * per_sm);
    if (dtype == SMOQ_C64) vqe_resident_kernel<float><<<grid, 256, smem, ctx->stream>>>(A);
    else vqe_resident_kernel<double><<<grid, 256, smem, ctx->stream>>>(A);
    ctx->launches++;
    VCK(cudaGetLastError());
    std::vector<double> e(n), nrm(n), cols((size_t)std::max(1, ncols));
    VCK(cudaMemcpyAsync(e.data(), A.energy, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaMemcpyAsync(nrm.data(), A.norm2, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaMemcpyAsync(cols.data(), A.cols, cols.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    for (size_t u = 0; u < idx.size(); ++u) {
        const smoq_vqe_job& J = jobs[idx[u]];
        J.energy[0] = e[u];
        if (!J.grad) continue;
        for (int p = 0; p < J.n_params; ++p) J.grad[p] = 0.0;
        for (size_t k = 0; k < inner_param[u].size(); ++k)
            J.grad[inner_param[u][k]] += cols[rj[u].col_off + k] / nrm[u];
    }
    return SMOQ_OK;
}

// ---------------------------------------------------------------- many circuits
// Worker contexts of a context (own stream and error word, the parent's options):
// the many-circuit call runs its larger circuits on them from host threads, so the
// small grids of several circuits share the GPU
static smoq_status job_workers(smoq_ctx* ctx, size_t k) {
    while (ctx->workers.size() < k) {
        smoq_ctx* w = nullptr;
        if (smoq_status s = smoq_ctx_create(ctx->device, &w)) return s;
        ctx->workers.push_back(w);
    }
    for (smoq_ctx* w : ctx->workers) {
        w->tile_bits_c64 = ctx->tile_bits_c64;
        w->tile_bits_c128 = ctx->tile_bits_c128;
        w->low_bits_c64 = ctx->low_bits_c64;
        w->low_bits_c128 = ctx->low_bits_c128;
        w->engine = ctx->engine;
        w->jit_buffers = ctx->jit_buffers;
        w->jit_groups = ctx->jit_groups;
        w->autotune = ctx->autotune;
        w->fusion_depth = ctx->fusion_depth;
        w->kernel_timing = 0;
    }
    return SMOQ_OK;
}

// Independent VQE jobs (each its own circuit, size and Hamiltonian).  Circuits
// whose two states fit one CTA's shared memory run in one launch off a device
// work queue (run_resident); the others are taken off a host queue by up to 8
// worker threads, each planning a circuit and running it on its own worker
// context's stream, while the calling thread runs the resident launch.
extern "C" smoq_status smoq_energy_grad_jobs(smoq_ctx* ctx, smoq_dtype dtype, const smoq_vqe_job* jobs, int njobs) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    if (njobs < 0 || (njobs > 0 && !jobs)) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "bad job list");
    for (int j = 0; j < njobs; ++j)
        if (!jobs[j].energy) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "job without energy output");
    std::vector<int> small, large;
    for (int j = 0; j < njobs; ++j) {
        const smoq_vqe_job& J = jobs[j];
        if (ctx->vqe_resident && J.N >= 1 && J.N <= (dtype == SMOQ_C64 ? kResMaxN64 : kResMaxN128)) {
            small.push_back(j);
            continue;
        }
        if (smoq_status s = check_vqe_args(ctx, J.N, dtype, J.ops, J.n, J.n_params, J.H, J.nterms, 1, J.theta)) {
            const std::string why = "job " + std::to_string(j) + ": " + smoq_last_error(ctx);
            return smoq_internal_fail(ctx, s, why.c_str());
        }
        large.push_back(j);
    }
    const size_t nworkers =
        std::min(large.size(), std::max<size_t>(1, std::min<size_t>(8, std::thread::hardware_concurrency() / 2)));
    if (nworkers > 0)
        if (smoq_status s = job_workers(ctx, nworkers)) return smoq_internal_fail(ctx, s, "worker context");
    const int tb = smoq_internal_tile_bits(ctx, dtype), lb = smoq_internal_low_bits(ctx, dtype);
    std::atomic<size_t> next(0);
    std::atomic<bool> failed(false);
    std::mutex mu;
    smoq_status first = SMOQ_OK;
    std::string why;
    std::vector<long long> launches0(nworkers);
    for (size_t w = 0; w < nworkers; ++w) launches0[w] = ctx->workers[w]->launches;
    auto work = [&](size_t w) {
        smoq_ctx* wc = ctx->workers[w];
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            if (first == SMOQ_OK) first = SMOQ_ERR_CUDA, why = "worker thread: cudaSetDevice failed";
            failed = true;
            return;
        }
        for (size_t i; !failed && (i = next++) < large.size();) {
            const smoq_vqe_job& J = jobs[large[i]];
            GradPlan gp;  // (host planning overlaps the other workers' GPU work)
            plan_gradient(J.N, dtype, tb, lb, J.ops, J.n, J.theta, J.grad != nullptr, gp, 0, wc, wc->fusion_depth);
            const smoq_status s =
                vqe_run(wc, J.N, dtype, J.ops, J.n, J.n_params, J.H, J.nterms, 1, J.theta, J.energy, J.grad, &gp);
            if (s != SMOQ_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (first == SMOQ_OK) {
                    first = s;
                    why = "job " + std::to_string(large[i]) + ": " + smoq_last_error(wc);
                }
                failed = true;
            }
        }
    };
    std::vector<std::thread> pool;
    for (size_t w = 0; w < nworkers; ++w) pool.emplace_back(work, w);
    smoq_status rs = SMOQ_OK;
    if (!small.empty()) rs = run_resident(ctx, dtype, jobs, small);
    for (std::thread& t : pool) t.join();
    for (size_t w = 0; w < nworkers; ++w) ctx->launches += ctx->workers[w]->launches - launches0[w];
    if (rs != SMOQ_OK) return rs;
    if (first != SMOQ_OK) return smoq_internal_fail(ctx, first, why.c_str());
    return SMOQ_OK;
}

// ---------------------------------------------------------------- HamiltonianParams -> Pauli terms
// apply_hamiltonian_bitwise! (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55) sums, per row,
// the bonds' ZZ, XX, YY and the fields' Z, X, Y terms with nonzero coefficients
static void params_to_terms(const double* x_bonds, int nx, const double* y_bonds, int ny, const double* fields,
                            int nf, std::vector<smoq_pauli_term>& t) {
    auto add = [&](double c, uint64_t x, uint64_t z) {
        if (c == 0.0) return;
        smoq_pauli_term p;
        p.coef = c;
        p.xmask = x;
        p.zmask = z;
        t.push_back(p);
    };
    for (int set = 0; set < 2; ++set) {
        const double* rows = set ? y_bonds : x_bonds;
        for (int r = 0; r < (set ? ny : nx); ++r) {
            const double* b = rows + 5 * r;
            const uint64_t m = (1ull << (int)b[0]) | (1ull << (int)b[1]);
            add(b[4], 0, m);   // ZZ
            add(b[2], m, 0);   // XX
            add(b[3], m, m);   // YY
        }
    }
    for (int r = 0; r < nf; ++r) {
        const double* f = fields + 4 * r;
        const uint64_t m = 1ull << (int)f[0];
        add(f[3], 0, m);   // Z
        add(f[1], m, 0);   // X
        add(f[2], m, m);   // Y
    }
}

extern "C" smoq_status smoq_apply_pauli_sum(smoq_state* in, smoq_state* out, const smoq_pauli_term* H, int nterms,
                                            double* expect);

extern "C" smoq_status smoq_apply_hamiltonian_bitwise(smoq_state* out, smoq_state* in, const double* x_bonds, int nx,
                                                      const double* y_bonds, int ny, const double* fields, int nf) {
    if (!in || !out || !in->ctx) return SMOQ_ERR_BADINPUT;
    if (nx < 0 || ny < 0 || nf < 0 || (nx && !x_bonds) || (ny && !y_bonds) || (nf && !fields))
        return smoq_internal_fail(in->ctx, SMOQ_ERR_BADINPUT, "apply_hamiltonian_bitwise: bad term arrays");
    for (int r = 0; r < nx + ny; ++r) {
        const double* b = r < nx ? x_bonds + 5 * r : y_bonds + 5 * (r - nx);
        if (b[0] < 0 || b[0] >= in->N || b[1] < 0 || b[1] >= in->N || (int)b[0] == (int)b[1])
            return smoq_internal_fail(in->ctx, SMOQ_ERR_BADINPUT, "apply_hamiltonian_bitwise: bond site out of range");
    }
    for (int r = 0; r < nf; ++r)
        if (fields[4 * r] < 0 || fields[4 * r] >= in->N)
            return smoq_internal_fail(in->ctx, SMOQ_ERR_BADINPUT, "apply_hamiltonian_bitwise: field site out of range");
    std::vector<smoq_pauli_term> t;
    params_to_terms(x_bonds, nx, y_bonds, ny, fields, nf, t);
    if (t.empty()) {  // H = 0
        smoq_pauli_term z;
        z.coef = 0.0;
        z.xmask = z.zmask = 0;
        t.push_back(z);
    }
    return smoq_apply_pauli_sum(in, out, t.data(), (int)t.size(), nullptr);
}

extern "C" smoq_status smoq_apply_h_xxz(smoq_state* psi, smoq_state* out, double Jx, double Jy, double Jz, double h) {
    if (!psi) return SMOQ_ERR_BADINPUT;
    const int N = psi->N;
    std::vector<double> bonds, fields;
    for (int i = 0; i + 1 < N; ++i) bonds.insert(bonds.end(), {(double)i, (double)(i + 1), Jx, Jy, Jz});
    for (int i = 0; i < N; ++i) fields.insert(fields.end(), {(double)i, h, 0.0, 0.0});
    return smoq_apply_hamiltonian_bitwise(out, psi, bonds.data(), N - 1, nullptr, 0, fields.data(), N);
}

// ---------------------------------------------------------------- H psi
// out = H in for every state of the batch, H = sum_t c_t P_t (Pauli strings);
// expect[b] = Re <in_b|H|in_b> when expect != NULL.  The pull-pattern
// Hamiltonian apply of apply_hamiltonian_bitwise!
// (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55) and apply_H_xxz! /
// apply_H_ising! (cpuQuantumStateLanczos.jl:157,220), for any Pauli sum.
extern "C" smoq_status smoq_apply_pauli_sum(smoq_state* in, smoq_state* out, const smoq_pauli_term* H, int nterms,
                                            double* expect) {
    if (!in || !out || !in->ctx) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = in->ctx;
    if (out->ctx != ctx || out->N != in->N || out->dtype != in->dtype || out->batch != in->batch)
        return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "apply_pauli_sum: in/out states differ in shape");
    if (out->ptr == in->ptr) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "apply_pauli_sum: out must not alias in");
    if (nterms < 1 || !H) return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "apply_pauli_sum: no terms");
    const int N = in->N;
    const uint64_t lim = (N >= 64) ? ~0ull : ((1ull << N) - 1);
    std::vector<HamTerm> ht(nterms);
    for (int t = 0; t < nterms; ++t) {
        if ((H[t].xmask | H[t].zmask) & ~lim)
            return smoq_internal_fail(ctx, SMOQ_ERR_BADINPUT, "Hamiltonian term acts beyond N");
        ht[t].coef = H[t].coef;
        ht[t].x = H[t].xmask;
        ht[t].z = H[t].zmask;
        ht[t].ny = __builtin_popcountll(H[t].xmask & H[t].zmask);
    }
    const int64_t len = (int64_t)1 << N;
    const int eblocks = (int)std::max<int64_t>(1, std::min<int64_t>((len + 255) / 256, (int64_t)ctx->num_sms * 8));
    void* buf = nullptr;
    const size_t tbytes = ht.size() * sizeof(HamTerm);
    // per state: eblocks energy partials, then eblocks norm partials (unused here)
    VCK(cudaMallocAsync(&buf, ((tbytes + 15) / 16) * 16 + 2 * (size_t)eblocks * in->batch * sizeof(double),
                        ctx->stream));
    HamTerm* d_terms = (HamTerm*)buf;
    double* d_part = (double*)((char*)buf + ((tbytes + 15) / 16) * 16);
    VCK(cudaMemcpyAsync(d_terms, ht.data(), tbytes, cudaMemcpyHostToDevice, ctx->stream));
    const size_t amp = in->amp_bytes();
    for (int b = 0; b < in->batch; ++b) {
        const char* src = (const char*)in->ptr + (size_t)b * len * amp;
        char* dst = (char*)out->ptr + (size_t)b * len * amp;
        if (in->dtype == SMOQ_C64)
            ham_apply_kernel<float><<<eblocks, 256, 0, ctx->stream>>>((const float2*)src, (float2*)dst, N, d_terms,
                                                                      nterms, d_part + 2 * (size_t)b * eblocks);
        else
            ham_apply_kernel<double><<<eblocks, 256, 0, ctx->stream>>>((const double2*)src, (double2*)dst, N,
                                                                       d_terms, nterms, d_part + 2 * (size_t)b * eblocks);
        ctx->launches++;
    }
    cudaError_t e = cudaGetLastError();
    std::vector<double> part;
    if (e == cudaSuccess && expect) {
        part.resize(2 * (size_t)eblocks * in->batch);
        e = cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    }
    cudaFreeAsync(buf, ctx->stream);
    if (e != cudaSuccess) return smoq_internal_cuda(ctx, e, "apply_pauli_sum");
    VCK(cudaStreamSynchronize(ctx->stream));
    if (expect)
        for (int b = 0; b < in->batch; ++b) {
            double s = 0;
            for (int k = 0; k < eblocks; ++k) s += part[2 * (size_t)b * eblocks + k];
            expect[b] = s;
        }
    return SMOQ_OK;
}

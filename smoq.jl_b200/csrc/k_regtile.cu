// k_regtile.cu -- the register-tile fused pass (sm_100a).
//
// Same contract as tile_pass_kernel (one HBM read + one HBM write of every
// tile, the pass's whole op program applied in between), but the tile lives
// in registers while the program runs:
//   * the tile's 2^T amplitudes arrive in shared memory by bulk copy
//     (cp.async.bulk + mbarrier, one copy per contiguous segment, no multicast);
//   * 256 threads pick them up: tile-local bits 0..4 = lane, KR = T - 8
//     register bits (2^KR amplitudes per thread), 3 warp bits;
//   * an op on lane bits exchanges values with __shfl (parity-block 4x4 and
//     1-qubit ops: one shuffle per amplitude); an op on register bits is a
//     fully unrolled update of the thread's own registers (the bit positions
//     are dispatched to compile-time constants); a mixed lane/register op uses
//     both; diagonal ops read any bit (lane, register, warp, or the tile's base
//     index for qubits outside the tile);
//   * when the next op needs a warp bit, the tile makes one round trip
//     through shared memory into a new register/warp assignment (OPK_LAYOUT),
//     planned on the host (schedule_regtile);
//   * at the end the registers go back to shared memory and out by bulk store.
// Shared-memory traffic is therefore ~2 tile sweeps per layout instead of 2
// per op, and every shared-memory access is 32 consecutive amplitudes per
// warp (conflict-free).
#include <cuda_runtime.h>
#include <stdint.h>
#include "k_common.cuh"

namespace smoq {

__device__ __forceinline__ float2 shfl_xor_c(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ double2 shfl_xor_c(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float2 shfl_c(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 shfl_c(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// matrix element (r, c) of a fused op, whatever its encoding
template <typename R>
__device__ __forceinline__ typename CT<R>::T op_elem(const DevOp& op, int r, int c) {
    using C = typename CT<R>::T;
    const int k = op.kind;
    if (k == OPK_DENSE1) return coef<R>(op, r * 2 + c);
    if (k == OPK_DENSE2) return coef<R>(op, r * 4 + c);
    if (k == OPK_PARITY2) {
        // even block {0,3}: c0 c1 / c2 c3 ; odd block {1,2}: c4 c5 / c6 c7
        if (((r == 0) || (r == 3)) != ((c == 0) || (c == 3))) return czero(C());
        if (r == 0) return coef<R>(op, c == 0 ? 0 : 1);
        if (r == 3) return coef<R>(op, c == 0 ? 2 : 3);
        if (r == 1) return coef<R>(op, c == 1 ? 4 : 5);
        return coef<R>(op, c == 1 ? 6 : 7);
    }
    if (k == OPK_MONO) return op.perm[r] == c ? coef<R>(op, r) : czero(C());
    return r == c ? coef<R>(op, r) : czero(C());
}

struct Layout {
    int regb[5];    // tile-local bit of register bit k
    int warpb[3];   // tile-local bit of warp bit k
    uint32_t wpart; // this thread's local-index bits from lane and warp
};

template <int KR>
__device__ __forceinline__ uint32_t rpart(const Layout& L, int r) {
    uint32_t j = 0;
#pragma unroll
    for (int k = 0; k < KR; ++k)
        if ((r >> k) & 1) j |= 1u << L.regb[k];
    return j;
}

template <int KR>
__device__ __forceinline__ void set_layout(Layout& L, const DevOp& op, int lane, int warp) {
#pragma unroll
    for (int k = 0; k < 5; ++k) L.regb[k] = k < KR ? op.perm[k] : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) L.warpb[k] = op.perm[5 + k];
    uint32_t j = (uint32_t)lane;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if ((warp >> k) & 1) j |= 1u << L.warpb[k];
    L.wpart = j;
}

template <typename C, int KR>
__device__ __forceinline__ void regs_to_smem(const C* v, C* tile, const Layout& L) {
#pragma unroll
    for (int r = 0; r < (1 << KR); ++r) tile[L.wpart | rpart<KR>(L, r)] = v[r];
}
template <typename C, int KR>
__device__ __forceinline__ void regs_from_smem(C* v, const C* tile, const Layout& L) {
#pragma unroll
    for (int r = 0; r < (1 << KR); ++r) v[r] = tile[L.wpart | rpart<KR>(L, r)];
}

// ---------------------------------------------------------------- 1 qubit
template <typename R, int KR, int P>
__device__ __forceinline__ void reg1(typename CT<R>::T* v, const DevOp& op) {
    if constexpr (P < KR) {
        using C = typename CT<R>::T;
        const C m00 = op_elem<R>(op, 0, 0), m01 = op_elem<R>(op, 0, 1);
        const C m10 = op_elem<R>(op, 1, 0), m11 = op_elem<R>(op, 1, 1);
#pragma unroll
        for (int e = 0; e < (1 << KR); ++e) {
            if (e & (1 << P)) continue;
            const int f = e | (1 << P);
            const C a = v[e], b = v[f];
            v[e] = cfma(m00, a, cmul(m01, b));
            v[f] = cfma(m10, a, cmul(m11, b));
        }
    }
}

template <typename R, int KR>
__device__ __forceinline__ void op1(typename CT<R>::T* v, const DevOp& op, int lane) {
    using C = typename CT<R>::T;
    const int s = op.slot[0];
    const int ty = s >> 8, ix = s & 255;
    if (ty == SLOT_LANE) {
        const int lm = 1 << ix;
        const int me = (lane >> ix) & 1;
        const C cs = op_elem<R>(op, me, me), cp = op_elem<R>(op, me, me ^ 1);
#pragma unroll
        for (int e = 0; e < (1 << KR); ++e) {
            const C p = shfl_xor_c(v[e], lm);
            v[e] = cfma(cs, v[e], cmul(cp, p));
        }
    } else {
        switch (ix) {
            case 0: reg1<R, KR, 0>(v, op); break;
            case 1: reg1<R, KR, 1>(v, op); break;
            case 2: reg1<R, KR, 2>(v, op); break;
            case 3: reg1<R, KR, 3>(v, op); break;
            case 4: reg1<R, KR, 4>(v, op); break;
            default: break;
        }
    }
}

// ---------------------------------------------------------------- 2 qubits
// both register bits: op qubit 0 on register bit P0, qubit 1 on P1
template <typename R, int KR, int P0, int P1>
__device__ __forceinline__ void reg2(typename CT<R>::T* v, const DevOp& op) {
    if constexpr (P0 < KR && P1 < KR && P0 != P1) {
        using C = typename CT<R>::T;
        if (op.kind == OPK_PARITY2) {
            // parity-block encoding read directly: e0 e1 / e2 e3 on (00, 11), o0 o1 / o2 o3 on (01, 10)
            const C e0 = coef<R>(op, 0), e3 = coef<R>(op, 3), o0 = coef<R>(op, 4), o1 = coef<R>(op, 5);
            const C o2 = coef<R>(op, 6), o3 = coef<R>(op, 7);
            if (op.flags & 1) {
                // even block diagonal (XX+YY+ZZ bonds with fields): two complex products fewer per quartet
#pragma unroll
                for (int e = 0; e < (1 << KR); ++e) {
                    if (e & ((1 << P0) | (1 << P1))) continue;
                    const int i1 = e | (1 << P0), i2 = e | (1 << P1), i3 = e | (1 << P0) | (1 << P1);
                    const C a1 = v[i1], a2 = v[i2];
                    v[e] = cmul(e0, v[e]);
                    v[i3] = cmul(e3, v[i3]);
                    v[i1] = cfma(o0, a1, cmul(o1, a2));
                    v[i2] = cfma(o2, a1, cmul(o3, a2));
                }
                return;
            }
            const C e1 = coef<R>(op, 1), e2 = coef<R>(op, 2);
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) {
                if (e & ((1 << P0) | (1 << P1))) continue;
                const int i1 = e | (1 << P0), i2 = e | (1 << P1), i3 = e | (1 << P0) | (1 << P1);
                const C a0 = v[e], a1 = v[i1], a2 = v[i2], a3 = v[i3];
                v[e] = cfma(e0, a0, cmul(e1, a3));
                v[i3] = cfma(e2, a0, cmul(e3, a3));
                v[i1] = cfma(o0, a1, cmul(o1, a2));
                v[i2] = cfma(o2, a1, cmul(o3, a2));
            }
            return;
        }
        C M[16];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) M[r * 4 + c] = op_elem<R>(op, r, c);
        const bool parity = false;
#pragma unroll
        for (int e = 0; e < (1 << KR); ++e) {
            if (e & ((1 << P0) | (1 << P1))) continue;
            const int i1 = e | (1 << P0), i2 = e | (1 << P1), i3 = e | (1 << P0) | (1 << P1);
            const C a0 = v[e], a1 = v[i1], a2 = v[i2], a3 = v[i3];
            if (parity) {
            } else {
                v[e] = cfma(M[0], a0, cfma(M[1], a1, cfma(M[2], a2, cmul(M[3], a3))));
                v[i1] = cfma(M[4], a0, cfma(M[5], a1, cfma(M[6], a2, cmul(M[7], a3))));
                v[i2] = cfma(M[8], a0, cfma(M[9], a1, cfma(M[10], a2, cmul(M[11], a3))));
                v[i3] = cfma(M[12], a0, cfma(M[13], a1, cfma(M[14], a2, cmul(M[15], a3))));
            }
        }
    }
}

// one lane bit (op qubit tl, lane bit la) and one register bit (op qubit 1-tl, register bit P)
template <typename R, int KR, int P>
__device__ __forceinline__ void mixed2(typename CT<R>::T* v, const DevOp& op, int tl, int la, int lane) {
    if constexpr (P < KR) {
        using C = typename CT<R>::T;
        const int tr = 1 - tl;
        const int bl = (lane >> la) & 1;
        const int lm = 1 << la;
        // matrix index of (lane bit value x, register bit value y)
        auto mi = [&](int x, int y) { return (x << tl) | (y << tr); };
        // rows for this thread's two elements (y = 0, 1); inputs: own y=0, own y=1, remote y=0, remote y=1
        C A[2][4];
#pragma unroll
        for (int y = 0; y < 2; ++y) {
            const int row = mi(bl, y);
            A[y][0] = op_elem<R>(op, row, mi(bl, 0));
            A[y][1] = op_elem<R>(op, row, mi(bl, 1));
            A[y][2] = op_elem<R>(op, row, mi(bl ^ 1, 0));
            A[y][3] = op_elem<R>(op, row, mi(bl ^ 1, 1));
        }
        if (op.kind == OPK_PARITY2) {
            // only the element with both bits flipped couples: (bl, y) <-> (bl^1, y^1)
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) {
                if (e & (1 << P)) continue;
                const int f = e | (1 << P);
                const C o0 = v[e], o1 = v[f];
                const C s0 = shfl_xor_c(o0, lm), s1 = shfl_xor_c(o1, lm);
                v[e] = cfma(A[0][0], o0, cmul(A[0][3], s1));
                v[f] = cfma(A[1][1], o1, cmul(A[1][2], s0));
            }
            return;
        }
#pragma unroll
        for (int e = 0; e < (1 << KR); ++e) {
            if (e & (1 << P)) continue;
            const int f = e | (1 << P);
            const C o0 = v[e], o1 = v[f];
            const C s0 = shfl_xor_c(o0, lm), s1 = shfl_xor_c(o1, lm);
            v[e] = cfma(A[0][0], o0, cfma(A[0][1], o1, cfma(A[0][2], s0, cmul(A[0][3], s1))));
            v[f] = cfma(A[1][0], o0, cfma(A[1][1], o1, cfma(A[1][2], s0, cmul(A[1][3], s1))));
        }
    }
}

template <typename R, int KR>
__device__ __forceinline__ void op2(typename CT<R>::T* v, const DevOp& op, int lane) {
    using C = typename CT<R>::T;
    const int t0 = op.slot[0] >> 8, i0 = op.slot[0] & 255;
    const int t1 = op.slot[1] >> 8, i1 = op.slot[1] & 255;
    if (t0 == SLOT_LANE && t1 == SLOT_LANE) {
        const int m0 = ((lane >> i0) & 1) | (((lane >> i1) & 1) << 1);
        const int l0 = 1 << i0, l1 = 1 << i1;
        if (op.kind == OPK_PARITY2) {
            const C cs = op_elem<R>(op, m0, m0), cp = op_elem<R>(op, m0, m0 ^ 3);
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) {
                const C p = shfl_xor_c(v[e], l0 | l1);
                v[e] = cfma(cs, v[e], cmul(cp, p));
            }
        } else if (op.kind == OPK_MONO) {
            const int src_m = op.perm[m0];
            const int src = (lane & ~(l0 | l1)) | ((src_m & 1) ? l0 : 0) | ((src_m & 2) ? l1 : 0);
            const C ph = coef<R>(op, m0);
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) v[e] = cmul(ph, shfl_c(v[e], src));
        } else {
            const C c0 = op_elem<R>(op, m0, m0), c1 = op_elem<R>(op, m0, m0 ^ 1);
            const C c2 = op_elem<R>(op, m0, m0 ^ 2), c3 = op_elem<R>(op, m0, m0 ^ 3);
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) {
                const C x1 = shfl_xor_c(v[e], l0), x2 = shfl_xor_c(v[e], l1), x3 = shfl_xor_c(v[e], l0 | l1);
                v[e] = cfma(c0, v[e], cfma(c1, x1, cfma(c2, x2, cmul(c3, x3))));
            }
        }
        return;
    }
    if (t0 == SLOT_REG && t1 == SLOT_REG) {
#define SMOQ_R2(A, B) \
    case (A) * 8 + (B): reg2<R, KR, A, B>(v, op); break;
        // the host puts qubit 0 on the lower register bit (schedule_regtile)
        switch (i0 * 8 + i1) {
            SMOQ_R2(0, 1) SMOQ_R2(0, 2) SMOQ_R2(0, 3) SMOQ_R2(0, 4)
            SMOQ_R2(1, 2) SMOQ_R2(1, 3) SMOQ_R2(1, 4)
            SMOQ_R2(2, 3) SMOQ_R2(2, 4)
            SMOQ_R2(3, 4)
            default: break;
        }
#undef SMOQ_R2
        return;
    }
    // mixed: one lane bit, one register bit
    const int tl = (t0 == SLOT_LANE) ? 0 : 1;
    const int la = tl == 0 ? i0 : i1;
    const int P = tl == 0 ? i1 : i0;
    switch (P) {
        case 0: mixed2<R, KR, 0>(v, op, tl, la, lane); break;
        case 1: mixed2<R, KR, 1>(v, op, tl, la, lane); break;
        case 2: mixed2<R, KR, 2>(v, op, tl, la, lane); break;
        case 3: mixed2<R, KR, 3>(v, op, tl, la, lane); break;
        case 4: mixed2<R, KR, 4>(v, op, tl, la, lane); break;
        default: break;
    }
}

// diagonal op on any bits: phase index from lane / warp / base bits (per
// thread) and register bits (per element)
template <typename R, int KR>
__device__ __forceinline__ void opdiag(typename CT<R>::T* v, const DevOp& op, const Layout& L, int lane,
                                       int warp, uint64_t base) {
    int mu = 0;
    int rpos[4] = {-1, -1, -1, -1};
    for (int t = 0; t < op.nq; ++t) {
        const int ty = op.slot[t] >> 8, ix = op.slot[t] & 255;
        if (ty == SLOT_LANE) mu |= ((lane >> ix) & 1) << t;
        else if (ty == SLOT_WARP) mu |= ((warp >> ix) & 1) << t;
        else if (ty == SLOT_REG) rpos[t] = ix;
        else mu |= (int)((base >> op.gb[t]) & 1) << t;
    }
#pragma unroll
    for (int e = 0; e < (1 << KR); ++e) {
        int m = mu;
#pragma unroll
        for (int t = 0; t < 4; ++t)
            if (rpos[t] >= 0) m |= ((e >> rpos[t]) & 1) << t;
        v[e] = cmul(coef<R>(op, m), v[e]);
    }
    (void)L;
}

template <int KR>
__device__ __forceinline__ uint64_t global_index(const Layout& L, int r, const TileGeom& g, uint64_t base) {
    const uint32_t j = L.wpart | rpart<KR>(L, r);
    uint64_t gi = base | (j & ((1u << g.L) - 1));
    const uint32_t h = j >> g.L;
    for (int m = 0; m < g.H; ++m) gi |= (uint64_t)((h >> m) & 1) << g.hb[m];
    return gi;
}

// Two tile buffers: while the registers work on tile k (buffer k&1, also used
// for its layout changes and its store), the bulk-copy engine brings tile k+1
// into the other buffer, and tile k's store drains behind tile k+1's compute.
template <typename R, int KR, bool EPI>
__global__ void __launch_bounds__(RT_THREADS, 2) regtile_kernel(const TileArgs a) {
    using C = typename CT<R>::T;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ double red[RT_THREADS / 32][16];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int T = a.g.T, L = a.g.L, H = a.g.H;
    const uint32_t amps = 1u << T;
    const uint32_t nseg = 1u << H;
    const uint32_t seg_bytes = (uint32_t)sizeof(C) << L;
    C* bufs[2] = {reinterpret_cast<C*>(smem_raw), reinterpret_cast<C*>(smem_raw) + amps};
    C v[1 << KR];

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phases = 0;  // bit i: parity of buffer i's next completion

    if ((int64_t)blockIdx.x < a.ntiles) issue_tile_load<C>(a, blockIdx.x, bufs[0], &bars[0]);
    int k = 0;
    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++k) {
        const int cur = k & 1;
        C* tile = bufs[cur];
        // prefetch the next tile into the other buffer (its previous store has
        // finished reading it: every thread waited on its bulk groups below)
        const int64_t tn = t + gridDim.x;
        const bool have_next = tn < a.ntiles;
        if (have_next) issue_tile_load<C>(a, tn, bufs[cur ^ 1], &bars[cur ^ 1]);

        int64_t b;
        const uint64_t base = tile_base(a, t, b);
        C* gs = reinterpret_cast<C*>(a.psi) + b * a.state_len;
        const bool ok = mbar_wait_bounded(&bars[cur], (phases >> cur) & 1, a.err);
        if (!__syncthreads_and(ok)) {
            // let the copies in flight land before the block exits
            mbar_wait_bounded(&bars[cur], (phases >> cur) & 1, nullptr);
            if (have_next) mbar_wait_bounded(&bars[cur ^ 1], (phases >> (cur ^ 1)) & 1, nullptr);
            return;
        }
        phases ^= 1u << cur;

        Layout Ly;
        set_layout<KR>(Ly, a.ops[0], lane, warp);
        regs_from_smem<C, KR>(v, tile, Ly);

        for (int o = 1; o < a.nops; ++o) {
            const DevOp& op = a.ops[o];
            const int kind = op.kind;
            if (kind == OPK_LAYOUT) {
                __syncthreads();
                regs_to_smem<C, KR>(v, tile, Ly);
                __syncthreads();
                set_layout<KR>(Ly, op, lane, warp);
                regs_from_smem<C, KR>(v, tile, Ly);
            } else if (op.mode == 1) {
                __syncthreads();
                regs_to_smem<C, KR>(v, tile, Ly);
                __syncthreads();
                if (kind == OPK_DIAG) {
                    // not scheduled this way, kept for completeness
                } else {
                    sweep_op<R, uint32_t>(op, tile, T, op.lb, (uint32_t)tid, (uint32_t)blockDim.x);
                }
                __syncthreads();
                regs_from_smem<C, KR>(v, tile, Ly);
            } else if (kind == OPK_DIAG) {
                opdiag<R, KR>(v, op, Ly, lane, warp, base);
            } else if (kind == OPK_STATESCALE) {
                const R s = (R)((const double*)op.aux)[b];
#pragma unroll
                for (int e = 0; e < (1 << KR); ++e) v[e] = cscale(v[e], s);
            } else if (kind == OPK_REALTAB) {
                const double* tab = (const double*)op.aux;
                const int ntab = (int)op.aux2;
#pragma unroll
                for (int e = 0; e < (1 << KR); ++e) {
                    const uint64_t gi = global_index<KR>(Ly, e, a.g, base);
                    double f = 1.0;
                    for (int k = 0; k < ntab; ++k) f *= tab[k * 256 + ((gi >> (8 * k)) & 255)];
                    v[e] = cscale(v[e], (R)f);
                }
            } else if (op.nq == 1) {
                op1<R, KR>(v, op, lane);
            } else {
                op2<R, KR>(v, op, lane);
            }
        }

        if (EPI) {
            // |psi|^2 total and per tile-local bit, for this tile
            double tot = 0, rs[5] = {0, 0, 0, 0, 0};
#pragma unroll
            for (int e = 0; e < (1 << KR); ++e) {
                const double p = cabs2d(v[e]);
                tot += p;
#pragma unroll
                for (int k = 0; k < KR; ++k)
                    if ((e >> k) & 1) rs[k] += p;
            }
            double vals[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) vals[j] = 0.0;
            vals[0] = tot;
#pragma unroll
            for (int j = 0; j < 15; ++j) {
                if (j >= T) continue;
                double x = 0;
                if ((Ly.wpart >> j) & 1) x = tot;  // lane and warp bits
#pragma unroll
                for (int k = 0; k < KR; ++k)
                    if (Ly.regb[k] == j) x = rs[k];
                vals[1 + j] = x;
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                double x = vals[k];
                for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
                if (lane == 0) red[warp][k] = x;
            }
            __syncthreads();
            if (tid < 16) {
                double s = 0;
                for (int w = 0; w < RT_THREADS / 32; ++w) s += red[w][tid];
                red[0][tid] = s;
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
        }

        __syncthreads();
        regs_to_smem<C, KR>(v, tile, Ly);
        fence_proxy_async_smem();
        __syncthreads();
        for (uint32_t s = tid; s < nseg; s += blockDim.x) {
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
template <typename R, bool EPI, int KR>
static cudaError_t rt_init_one(smoq_ctx* ctx, int dt) {
    auto kern = regtile_kernel<R, KR, EPI>;
    const size_t smem = (size_t)2 * sizeof(typename CT<R>::T) << (RT_MIN_T + KR);  // two tile buffers
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RT_THREADS, smem);
    if (e != cudaSuccess) return e;
    ctx->rt_occ[dt][EPI ? 1 : 0][KR] = per_sm < 1 ? 1 : per_sm;
    return cudaSuccess;
}

template <typename R, bool EPI>
static cudaError_t rt_init_all(smoq_ctx* ctx, int dt) {
    cudaError_t e;
    if ((e = rt_init_one<R, EPI, 0>(ctx, dt)) != cudaSuccess) return e;
    if ((e = rt_init_one<R, EPI, 1>(ctx, dt)) != cudaSuccess) return e;
    if ((e = rt_init_one<R, EPI, 2>(ctx, dt)) != cudaSuccess) return e;
    if ((e = rt_init_one<R, EPI, 3>(ctx, dt)) != cudaSuccess) return e;
    if ((e = rt_init_one<R, EPI, 4>(ctx, dt)) != cudaSuccess) return e;
    if constexpr (sizeof(R) == 4)
        if ((e = rt_init_one<R, EPI, 5>(ctx, dt)) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t regtile_kernels_init(smoq_ctx* ctx) {
    cudaError_t e;
    if ((e = rt_init_all<float, false>(ctx, 0)) != cudaSuccess) return e;
    if ((e = rt_init_all<float, true>(ctx, 0)) != cudaSuccess) return e;
    if ((e = rt_init_all<double, false>(ctx, 1)) != cudaSuccess) return e;
    return rt_init_all<double, true>(ctx, 1);
}

template <typename R, bool EPI>
static cudaError_t rt_launch(smoq_ctx* ctx, const TileArgs& a, int dt) {
    const int KR = a.g.T - RT_MIN_T;
    const size_t smem = (size_t)2 * sizeof(typename CT<R>::T) << a.g.T;  // two tile buffers
    int per_sm = ctx->rt_occ[dt][EPI ? 1 : 0][KR];
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)ctx->num_sms * per_sm;
    if (grid > a.ntiles) grid = a.ntiles;
    const unsigned g = (unsigned)grid;
    switch (KR) {
        case 0: regtile_kernel<R, 0, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a); break;
        case 1: regtile_kernel<R, 1, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a); break;
        case 2: regtile_kernel<R, 2, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a); break;
        case 3: regtile_kernel<R, 3, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a); break;
        case 4: regtile_kernel<R, 4, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a); break;
        case 5:
            if constexpr (sizeof(R) == 4) {
                regtile_kernel<R, 5, EPI><<<g, RT_THREADS, smem, ctx->stream>>>(a);
                break;
            }
            return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_regtile(smoq_ctx* ctx, const TileArgs& a, int dtype, bool epi) {
    if (dtype == SMOQ_C64) return epi ? rt_launch<float, true>(ctx, a, 0) : rt_launch<float, false>(ctx, a, 0);
    return epi ? rt_launch<double, true>(ctx, a, 1) : rt_launch<double, false>(ctx, a, 1);
}

}  // namespace smoq

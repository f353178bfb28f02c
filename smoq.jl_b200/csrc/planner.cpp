// planner.cpp -- gate IR, gate matrices, and the fused-pass planner.
//
// The planner turns an ordered gate list into tile passes.  It generalises
// the reference's own fusion (fuse_gates, SmoQ.jl_benchmarks/
// benchmark_random_circuit_sampling/run_benchmark_smoq_Float64.jl:167, which
// merges runs of single-qubit gates into one 2x2 and flushes at two-qubit
// gates) from "one qubit" to "one tile of T qubits":
//   1. greedy pass building: scan the remaining gates in order; a
//      non-diagonal gate joins the pass if none of its qubits is blocked and
//      the pass's tile (the low Lmin qubits + the qubits taken so far) can
//      hold its qubits within T; a diagonal gate joins whenever none of its
//      qubits is blocked by a skipped NON-diagonal gate (diagonals commute
//      with each other and need no tile membership: their phase depends only
//      on the amplitude's global index).  A skipped gate blocks its qubits
//      (hard for non-diagonal, soft for diagonal) so no later gate that does
//      not commute with it can overtake it.
//   2. fusion inside the pass: runs of 1-qubit gates on a qubit collapse to
//      one 2x2; a 2-qubit gate absorbs the pending 2x2s of its qubits;
//      consecutive 2-qubit gates on the same pair multiply into one 4x4.
//   3. classification of every fused matrix (diagonal, monomial, parity
//      block, dense) so the kernel runs the cheapest sweep for it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include "smoq_internal.h"

namespace smoq {

static const cd I1(0.0, 1.0);

GateIR gate_1q(int q, const cd m[4]) {
    GateIR g;
    g.nq = 1;
    g.q[0] = q;
    for (int k = 0; k < 4; ++k) g.m[k] = m[k];
    g.diag = (m[1] == 0.0 && m[2] == 0.0);
    return g;
}

GateIR gate_2q(int q0, int q1, const cd m[16]) {
    GateIR g;
    g.nq = 2;
    g.q[0] = q0;
    g.q[1] = q1;
    bool d = true;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            g.m[r * 4 + c] = m[r * 4 + c];
            if (r != c && m[r * 4 + c] != 0.0) d = false;
        }
    g.diag = d;
    return g;
}

static GateIR diag_nq(int nq, const int* q, const cd* d) {
    GateIR g;
    g.nq = nq;
    for (int t = 0; t < nq; ++t) g.q[t] = q[t];
    const int dim = 1 << nq;
    for (int k = 0; k < dim * dim; ++k) g.m[k] = 0.0;
    for (int k = 0; k < dim; ++k) g.m[k * dim + k] = d[k];
    g.diag = true;
    return g;
}

// Gate matrices as defined in utils/cpu/cpuQuantumChannelGates.jl:53-71
// (header) and in each apply_*_psi! body; two-qubit local index
// m = bit(q[0]) + 2 bit(q[1]).
GateIR gate_named(int type, const int* q, double th) {
    const double c = std::cos(th / 2), s = std::sin(th / 2);
    switch (type) {
        case SMOQ_G_RX: { cd m[4] = {c, -I1 * s, -I1 * s, c}; return gate_1q(q[0], m); }
        case SMOQ_G_RY: { cd m[4] = {c, -s, s, c}; return gate_1q(q[0], m); }
        case SMOQ_G_RZ: { cd m[4] = {std::exp(-I1 * th / 2.0), 0, 0, std::exp(I1 * th / 2.0)}; return gate_1q(q[0], m); }
        case SMOQ_G_H: { const double r = 1 / std::sqrt(2.0); cd m[4] = {r, r, r, -r}; return gate_1q(q[0], m); }
        case SMOQ_G_X: { cd m[4] = {0, 1, 1, 0}; return gate_1q(q[0], m); }
        case SMOQ_G_Y: { cd m[4] = {0, -I1, I1, 0}; return gate_1q(q[0], m); }
        case SMOQ_G_Z: { cd m[4] = {1, 0, 0, -1}; return gate_1q(q[0], m); }
        case SMOQ_G_S: { cd m[4] = {1, 0, 0, I1}; return gate_1q(q[0], m); }
        case SMOQ_G_SDG: { cd m[4] = {1, 0, 0, -I1}; return gate_1q(q[0], m); }
        case SMOQ_G_T: { cd m[4] = {1, 0, 0, std::exp(I1 * (M_PI / 4))}; return gate_1q(q[0], m); }
        case SMOQ_G_TDG: { cd m[4] = {1, 0, 0, std::exp(-I1 * (M_PI / 4))}; return gate_1q(q[0], m); }
        case SMOQ_G_CZ: { cd d[4] = {1, 1, 1, -1}; return diag_nq(2, q, d); }
        case SMOQ_G_RZZ: {
            const cd same = std::exp(-I1 * th / 2.0), diff = std::exp(I1 * th / 2.0);
            cd d[4] = {same, diff, diff, same};
            return diag_nq(2, q, d);
        }
        case SMOQ_G_CCZ: { cd d[8] = {1, 1, 1, 1, 1, 1, 1, -1}; return diag_nq(3, q, d); }
        case SMOQ_G_CNOT: {  // q[0] control, q[1] target: swap m=1 <-> m=3
            cd m[16] = {};
            m[0 * 4 + 0] = 1; m[2 * 4 + 2] = 1; m[1 * 4 + 3] = 1; m[3 * 4 + 1] = 1;
            return gate_2q(q[0], q[1], m);
        }
        case SMOQ_G_RXX: {  // c I - i s XX, XX: m -> m ^ 3
            cd m[16] = {};
            for (int k = 0; k < 4; ++k) { m[k * 4 + k] = c; m[k * 4 + (k ^ 3)] = -I1 * s; }
            return gate_2q(q[0], q[1], m);
        }
        case SMOQ_G_RYY: {  // c I - i s YY, YY: 00<->11 with -1, 01<->10 with +1
            cd m[16] = {};
            for (int k = 0; k < 4; ++k) m[k * 4 + k] = c;
            m[0 * 4 + 3] = I1 * s; m[3 * 4 + 0] = I1 * s;
            m[1 * 4 + 2] = -I1 * s; m[2 * 4 + 1] = -I1 * s;
            return gate_2q(q[0], q[1], m);
        }
        case SMOQ_G_CRY: {  // q[0] control, q[1] target; Ry on (m=1, m=3)
            cd m[16] = {};
            m[0] = 1; m[2 * 4 + 2] = 1;
            m[1 * 4 + 1] = c; m[1 * 4 + 3] = -s; m[3 * 4 + 1] = s; m[3 * 4 + 3] = c;
            return gate_2q(q[0], q[1], m);
        }
        case SMOQ_G_TOFFOLI: {  // q = (c1, c2, t): swap m=3 <-> m=7
            GateIR g;
            g.nq = 3;
            for (int t = 0; t < 3; ++t) g.q[t] = q[t];
            for (int k = 0; k < 64; ++k) g.m[k] = 0.0;
            for (int k = 0; k < 8; ++k) g.m[k * 8 + k] = 1;
            g.m[3 * 8 + 3] = 0; g.m[7 * 8 + 7] = 0;
            g.m[3 * 8 + 7] = 1; g.m[7 * 8 + 3] = 1;
            g.diag = false;
            return g;
        }
        default: throw std::invalid_argument("unknown gate type");
    }
}

// ---------------------------------------------------------------- matrices
static void matmul(int dim, const cd* A, const cd* B, cd* out) {  // out = A * B
    cd tmp[64];
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) {
            cd s = 0;
            for (int k = 0; k < dim; ++k) s += A[r * dim + k] * B[k * dim + c];
            tmp[r * dim + c] = s;
        }
    std::memcpy(out, tmp, sizeof(cd) * dim * dim);
}
// kron for the 2-qubit local basis m = bit(q0) + 2 bit(q1): (P1 (x) P0)
static void kron2(const cd* P0, const cd* P1, cd* out) {
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[r * 4 + c] = P1[(r >> 1) * 2 + (c >> 1)] * P0[(r & 1) * 2 + (c & 1)];
}
// the same 4x4 with its two qubits' roles exchanged
static void swap_roles(const cd* M, cd* out) {
    auto sw = [](int m) { return ((m & 1) << 1) | (m >> 1); };
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out[sw(r) * 4 + sw(c)] = M[r * 4 + c];
}

static void fill_coeffs(DevOp& op, const cd* v, int n) {
    for (int k = 0; k < 16; ++k) {
        cd x = k < n ? v[k] : cd(0.0);
        op.cd[k] = make_double2(x.real(), x.imag());
        op.cf[k] = make_float2((float)x.real(), (float)x.imag());
    }
}

// classify and encode a k-qubit matrix (k = 1..3; diagonals up to 4) as a DevOp
static void encode_matrix(int nq, const cd* M, DevOp& op) {
    const int dim = 1 << nq;
    bool diag = true, mono = nq <= 3;
    int perm[16];
    for (int r = 0; r < dim; ++r) {
        int nz = 0;
        perm[r] = r;
        for (int c = 0; c < dim; ++c)
            if (M[r * dim + c] != 0.0) {
                ++nz;
                perm[r] = c;
                if (r != c) diag = false;
            }
        if (nz > 1) { mono = false; diag = false; }
        if (nz == 0) diag = false, perm[r] = r;  // a zero row: monomial with phase 0
    }
    op.nq = nq;
    if (diag) {
        cd d[16];
        for (int k = 0; k < dim; ++k) d[k] = M[k * dim + k];
        op.kind = OPK_DIAG;
        fill_coeffs(op, d, dim);
        return;
    }
    if (mono) {
        cd ph[8];
        for (int r = 0; r < dim; ++r) {
            ph[r] = M[r * dim + perm[r]];
            op.perm[r] = perm[r];
        }
        op.kind = OPK_MONO;
        fill_coeffs(op, ph, dim);
        return;
    }
    auto all_real = [&](int n) {
        for (int k = 0; k < n; ++k)
            if (M[k].imag() != 0.0) return false;
        return true;
    };
    if (nq == 1) {
        op.kind = OPK_DENSE1;
        fill_coeffs(op, M, 4);
        op.flags = all_real(4) ? OPF_REAL : 0;
        return;
    }
    if (nq == 2) {
        const bool parity = M[0 * 4 + 1] == 0.0 && M[0 * 4 + 2] == 0.0 && M[3 * 4 + 1] == 0.0 &&
                            M[3 * 4 + 2] == 0.0 && M[1 * 4 + 0] == 0.0 && M[1 * 4 + 3] == 0.0 &&
                            M[2 * 4 + 0] == 0.0 && M[2 * 4 + 3] == 0.0;
        if (parity) {
            cd v[8] = {M[0], M[3], M[12], M[15], M[5], M[6], M[9], M[10]};
            op.kind = OPK_PARITY2;
            fill_coeffs(op, v, 8);
            // XX+YY+ZZ-type bonds (and anything fused with diagonal fields) leave
            // one block diagonal: the kernels skip its zero products
            op.flags = (M[3] == 0.0 && M[12] == 0.0 ? 1 : 0) | (M[6] == 0.0 && M[9] == 0.0 ? 2 : 0);
            return;
        }
        op.kind = OPK_DENSE2;
        fill_coeffs(op, M, 16);
        op.flags = all_real(16) ? OPF_REAL : 0;
        return;
    }
    throw std::invalid_argument("3-qubit gates must be diagonal or monomial");
}

static int local_bit(const TileGeom* g, int q) {
    if (!g) return q;
    if (q < g->L) return q;
    for (int m = 0; m < g->H; ++m)
        if (g->hb[m] == q) return g->L + m;
    return -1;
}

void build_devop(const GateIR& gt, const TileGeom* g, DevOp& op) {
    std::memset(&op, 0, sizeof(op));
    for (int t = 0; t < 4; ++t) {
        op.lb[t] = -1;
        op.gb[t] = 0;
    }
    for (int r = 0; r < 8; ++r) op.perm[r] = r;
    if (gt.special == OPK_INNER) {
        // generator G (dense row-major on the op's qubits) re-encoded as a signed
        // monomial: row r has at most one nonzero, i^code at column perm[1 + r]
        op.kind = OPK_INNER;
        op.nq = gt.nq;
        if (gt.nq < 1 || gt.nq > 2) throw std::runtime_error("adjoint generator must act on 1 or 2 qubits");
        for (int t = 0; t < gt.nq; ++t) {
            op.gb[t] = gt.q[t];
            op.lb[t] = local_bit(g, gt.q[t]);
        }
        const int dim = 1 << gt.nq;
        bool diag = true;
        for (int r = 0; r < dim; ++r) {
            int col = r, code = INNER_ZERO, nz = 0;
            for (int c = 0; c < dim; ++c) {
                const cd x = gt.m[r * dim + c];
                if (std::abs(x) == 0.0) continue;
                ++nz;
                col = c;
                if (x == cd(1.0, 0.0)) code = 0;
                else if (x == cd(0.0, 1.0)) code = 1;
                else if (x == cd(-1.0, 0.0)) code = 2;
                else if (x == cd(0.0, -1.0)) code = 3;
                else throw std::runtime_error("adjoint generator entries must be +-1 or +-i");
            }
            if (nz > 1) throw std::runtime_error("adjoint generator must be a signed Pauli monomial");
            op.perm[1 + r] = col;
            op.slot[r] = code;
            if (col != r || code == 1 || code == 3) diag = false;  // real diagonal only
        }
        op.flags = diag ? INNER_DIAGG : 0;
        op.perm[0] = (int32_t)gt.aux2;  // the caller's index of this measurement
        return;
    }
    if (gt.special) {
        op.kind = gt.special;
        op.aux = gt.aux;
        op.aux2 = gt.aux2;
        op.nq = 0;
        return;
    }
    for (int t = 0; t < gt.nq; ++t) {
        op.gb[t] = gt.q[t];
        op.lb[t] = local_bit(g, gt.q[t]);
    }
    encode_matrix(gt.nq, gt.m, op);
    op.nq = gt.nq;
}

// -------------------------------------------------------------------- plan
namespace {
// diagonal of a diagonal gate, index bit t = qubit q[t]
static void diag_of(const GateIR& g, cd* d) {
    const int dim = 1 << g.nq;
    for (int k = 0; k < dim; ++k) d[k] = g.m[k * dim + k];
}

// Fusion inside one pass.  Ops are kept in host (matrix) form until the pass
// is complete so that later gates can still be folded into earlier ops:
//  * 1-qubit gates on a tile qubit accumulate in a pending 2x2 per qubit;
//  * a 2-qubit gate absorbs the pending 2x2s of its qubits, and merges into
//    the last op on the same pair when no op since has touched either qubit;
//  * a pending 2x2 that is flushed (end of pass, or a diagonal on a non-tile
//    qubit) is folded into the last 2-qubit op on its qubit when nothing
//    after that op touched the qubit;
//  * a diagonal op merges into an earlier diagonal op (one phase table, up to 4
//    qubits) when every op in between commutes with it: diagonal ops, measurements
//    of a diagonal generator, and ops on other qubits (a backward program's Rz^dag
//    ops join the CZ tables across the Z measurements between them).
struct Fuser {
    const TileGeom* g;
    std::vector<GateIR> ops;
    bool have_pending[64] = {};
    cd pending[64][4];
    int last_touch[64];

    explicit Fuser(const TileGeom* geom) : g(geom) {
        for (int q = 0; q < 64; ++q) last_touch[q] = -1;
    }
    bool is_tile(int q) const { return local_bit(g, q) >= 0; }
    bool tile_2q(const GateIR& o) const {
        return o.nq == 2 && !o.special && is_tile(o.q[0]) && is_tile(o.q[1]);
    }
    void touch(int idx) {
        const GateIR& o = ops[idx];
        if (o.special == OPK_REALTAB) {
            for (int q = 0; q < 64; ++q) last_touch[q] = idx;
            return;
        }
        for (int t = 0; t < o.nq; ++t) last_touch[o.q[t]] = idx;
    }
    static bool merge_diag(GateIR& A, const GateIR& B) {
        int uq[4], u = 0;
        for (int t = 0; t < A.nq; ++t) uq[u++] = A.q[t];
        for (int t = 0; t < B.nq; ++t) {
            bool seen = false;
            for (int s = 0; s < u; ++s) seen |= (uq[s] == B.q[t]);
            if (!seen) {
                if (u == 4) return false;
                uq[u++] = B.q[t];
            }
        }
        cd da[16], db[16], d[16];
        diag_of(A, da);
        diag_of(B, db);
        for (int m = 0; m < (1 << u); ++m) {
            int ia = 0, ib = 0;
            for (int t = 0; t < A.nq; ++t)
                for (int s = 0; s < u; ++s)
                    if (uq[s] == A.q[t]) ia |= ((m >> s) & 1) << t;
            for (int t = 0; t < B.nq; ++t)
                for (int s = 0; s < u; ++s)
                    if (uq[s] == B.q[t]) ib |= ((m >> s) & 1) << t;
            d[m] = da[ia] * db[ib];
        }
        GateIR r;
        r.nq = u;
        for (int s = 0; s < u; ++s) r.q[s] = uq[s];
        const int dim = 1 << u;
        for (int k = 0; k < dim * dim; ++k) r.m[k] = 0.0;
        for (int k = 0; k < dim; ++k) r.m[k * dim + k] = d[k];
        r.diag = true;
        A = r;
        return true;
    }
    // does op o commute with the diagonal d?
    static bool commutes_with_diag(const GateIR& o, const GateIR& d) {
        if (o.special == OPK_REALTAB || o.special == OPK_STATESCALE) return true;  // diagonal
        bool diag = o.diag && !o.special;
        if (o.special == OPK_INNER) {  // a measurement: its generator's matrix is in m
            const int dim = 1 << o.nq;
            diag = true;
            for (int r = 0; r < dim && diag; ++r)
                for (int c = 0; c < dim; ++c)
                    if (r != c && std::abs(o.m[r * dim + c]) != 0.0) diag = false;
        } else if (o.special) {
            return false;
        }
        if (diag) return true;
        for (int t = 0; t < o.nq; ++t)
            for (int u = 0; u < d.nq; ++u)
                if (o.q[t] == d.q[u]) return false;
        return true;
    }
    void push(const GateIR& gt) {
        if (gt.diag && !gt.special) {
            int seen = 0;
            for (int i = (int)ops.size() - 1; i >= 0 && seen < 64; --i, ++seen) {
                GateIR& e = ops[i];
                if (e.diag && !e.special) {
                    // (a look-back merge only builds tables on tile qubits: a table
                    // with an off-tile qubit is indexed per register at run time)
                    bool tile_only = true;
                    for (int t = 0; t < e.nq; ++t) tile_only &= is_tile(e.q[t]);
                    for (int t = 0; t < gt.nq; ++t) tile_only &= is_tile(gt.q[t]);
                    if ((i == (int)ops.size() - 1 || tile_only) && merge_diag(e, gt)) {
                        // (ops after i that touched these qubits keep their later mark)
                        for (int t = 0; t < e.nq; ++t) last_touch[e.q[t]] = std::max(last_touch[e.q[t]], i);
                        return;
                    }
                    continue;  // diagonals commute: look further back for room
                }
                if (!commutes_with_diag(e, gt)) break;
            }
        }
        ops.push_back(gt);
        touch((int)ops.size() - 1);
    }
    void flush(int q) {
        if (!have_pending[q]) return;
        have_pending[q] = false;
        const int j = last_touch[q];
        if (j >= 0 && tile_2q(ops[j])) {
            static const cd Id[4] = {1, 0, 0, 1};
            cd P4[16], out[16];
            if (ops[j].q[0] == q) kron2(pending[q], Id, P4);
            else kron2(Id, pending[q], P4);
            matmul(4, P4, ops[j].m, out);  // the pending gates act after op j
            ops[j] = gate_2q(ops[j].q[0], ops[j].q[1], out);
            return;
        }
        push(gate_1q(q, pending[q]));
    }
    void flush_all() {
        for (int q = 0; q < 64; ++q) flush(q);
    }
    void add(const GateIR& gt) {
        if (gt.special) {
            if (gt.special == OPK_REALTAB) flush_all();  // diagonal over every qubit
            if (gt.special == OPK_INNER)                 // measures the state as it is at this point
                for (int t = 0; t < gt.nq; ++t) flush(gt.q[t]);
            ops.push_back(gt);
            touch((int)ops.size() - 1);
            return;
        }
        bool all_tile = true;
        for (int t = 0; t < gt.nq; ++t)
            if (!is_tile(gt.q[t])) all_tile = false;
        if (gt.nq == 1 && all_tile) {
            const int q = gt.q[0];
            if (have_pending[q]) {
                cd out[4];
                matmul(2, gt.m, pending[q], out);
                std::memcpy(pending[q], out, sizeof(out));
            } else {
                std::memcpy(pending[q], gt.m, sizeof(cd) * 4);
                have_pending[q] = true;
            }
            return;
        }
        if (gt.nq == 2 && all_tile) {
            const int a = gt.q[0], b = gt.q[1];
            cd M[16];
            std::memcpy(M, gt.m, sizeof(M));
            if (have_pending[a] || have_pending[b]) {
                static const cd Id[4] = {1, 0, 0, 1};
                cd K[16];
                kron2(have_pending[a] ? pending[a] : Id, have_pending[b] ? pending[b] : Id, K);
                matmul(4, M, K, M);
                have_pending[a] = have_pending[b] = false;
            }
            const int j = last_touch[a];
            if (j >= 0 && j == last_touch[b] && tile_2q(ops[j]) &&
                ((ops[j].q[0] == a && ops[j].q[1] == b) || (ops[j].q[0] == b && ops[j].q[1] == a))) {
                cd Mal[16], out[16];
                if (ops[j].q[0] == a) std::memcpy(Mal, M, sizeof(Mal));
                else swap_roles(M, Mal);
                matmul(4, Mal, ops[j].m, out);
                ops[j] = gate_2q(ops[j].q[0], ops[j].q[1], out);
                return;
            }
            push(gate_2q(a, b, M));
            return;
        }
        // diagonal gates touching non-tile qubits, and 3-qubit gates
        for (int t = 0; t < gt.nq; ++t)
            if (is_tile(gt.q[t])) flush(gt.q[t]);
        if (!all_tile && !gt.diag) throw std::logic_error("planner placed a non-diagonal gate off-tile");
        push(gt);
    }
    std::vector<DevOp> finish() {
        flush_all();
        std::vector<DevOp> out(ops.size());
        for (size_t i = 0; i < ops.size(); ++i) build_devop(ops[i], g, out[i]);
        return out;
    }
};
}  // namespace

std::vector<Pass> plan_passes(const std::vector<GateIR>& gates, int N, int T, int Lmin,
                              int epilogue_after_special, int Lreq) {
    // Lreq: contiguous low qubits every tile must hold (complex64 needs 1 so a
    // segment is >= 16 bytes, the bulk-copy granule).  A tile must keep room
    // for a 3-qubit gate next to its reserved low qubits, or some gates could
    // never be placed.
    if (T > N) T = N;
    if (Lreq > T) Lreq = T;
    if (T < N && T < Lreq + 3) throw std::invalid_argument("tile too narrow for 3-qubit gates");
    if (Lmin > T - 3) Lmin = T - 3;
    if (Lmin < Lreq) Lmin = Lreq;
    if (Lmin > T) Lmin = T;
    std::vector<int> remaining(gates.size());
    for (size_t i = 0; i < gates.size(); ++i) remaining[i] = (int)i;
    const uint64_t allq = (N >= 64) ? ~0ull : ((1ull << N) - 1);
    std::vector<Pass> passes;
    while (!remaining.empty()) {
        uint64_t tileset = (Lmin > 0) ? ((1ull << Lmin) - 1) : 0;
        uint64_t hard = 0, soft = 0;
        std::vector<int> taken, rest;
        for (int idx : remaining) {
            const GateIR& gt = gates[idx];
            uint64_t qm = 0;
            if (gt.special == OPK_REALTAB) qm = allq;
            for (int t = 0; t < gt.nq; ++t) qm |= 1ull << gt.q[t];
            // an inner-product op needs its generator's qubits in the tile, like a gate
            if (gt.diag || (gt.special && gt.special != OPK_INNER)) {
                if ((qm & hard) == 0) taken.push_back(idx);
                else { soft |= qm; rest.push_back(idx); }
            } else {
                const uint64_t ns = tileset | qm;
                if ((qm & (hard | soft)) == 0 && __builtin_popcountll(ns) <= T) {
                    tileset = ns;
                    taken.push_back(idx);
                } else {
                    hard |= qm;
                    rest.push_back(idx);
                }
            }
        }
        if (taken.empty()) throw std::logic_error("planner made no progress");
        // widen the tile with the lowest free qubits: longer contiguous segments
        for (int b = 0; b < N && __builtin_popcountll(tileset) < T; ++b) tileset |= 1ull << b;
        Pass p;
        std::memset(&p.g, 0, sizeof(p.g));
        p.g.N = N;
        p.g.T = __builtin_popcountll(tileset);
        int L = 0;
        while (L < N && ((tileset >> L) & 1)) ++L;
        p.g.L = L;
        p.g.H = 0;
        for (int b = L; b < N; ++b)
            if ((tileset >> b) & 1) p.g.hb[p.g.H++] = b;
        Fuser f(&p.g);
        f.ops.reserve(taken.size() + 64);  // (a flush adds at most one op per qubit)
        for (int idx : taken) {
            f.add(gates[idx]);
            if (epilogue_after_special >= 0 && gates[idx].special == epilogue_after_special) p.epilogue = true;
        }
        p.ops = f.finish();
        passes.push_back(std::move(p));
        remaining.swap(rest);
    }
    return passes;
}

// Exchange the roles of a 2-qubit op's qubits 0 and 1 (matrix index bits
// swapped: local index 1 <-> 2), in every encoding the kernels read.
static void swap_qubit_roles(DevOp& op) {
    auto sw = [](int m) { return ((m & 1) << 1) | ((m >> 1) & 1); };
    std::swap(op.lb[0], op.lb[1]);
    std::swap(op.gb[0], op.gb[1]);
    std::swap(op.slot[0], op.slot[1]);
    double2 d[16];
    float2 f[16];
    for (int k = 0; k < 16; ++k) d[k] = op.cd[k], f[k] = op.cf[k];
    if (op.kind == OPK_DENSE2) {
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) {
                op.cd[r * 4 + c] = d[sw(r) * 4 + sw(c)];
                op.cf[r * 4 + c] = f[sw(r) * 4 + sw(c)];
            }
    } else if (op.kind == OPK_PARITY2) {
        // even block (00, 11) is unchanged; the odd block (01, 10) is mirrored
        const int map[4] = {7, 6, 5, 4};
        for (int k = 0; k < 4; ++k) {  // (the diagonal flags of both blocks stay valid)
            op.cd[4 + k] = d[map[k]];
            op.cf[4 + k] = f[map[k]];
        }
    } else if (op.kind == OPK_MONO) {
        int perm[4];
        for (int r = 0; r < 4; ++r) perm[r] = op.perm[r];
        for (int r = 0; r < 4; ++r) {
            op.perm[r] = sw(perm[sw(r)]);
            op.cd[r] = d[sw(r)];
            op.cf[r] = f[sw(r)];
        }
    }
}

// ----------------------------------------------------------------------------
// Rotation splitting for the compiled pass kernels.  A unitary 2x2 block
// [[p, q], [r, t]] equals diag(1, l2) . [[c, -is], [-is, c]] . diag(r1, r2) with
// c = |p|, s = |q|, r1 = p / c, r2 = i q / s, l2 = t / (c r2) (unitarity gives the
// fourth entry).  The middle factor has one real and one imaginary coefficient per
// row: half the FP32 work of a general complex block.  The two diagonal factors sit
// on the op's own qubits, which the stage schedule keeps on stage bits, so the
// compiled kernel folds them with the stage's other diagonals into one literal
// phase per register.
namespace {
struct BlockSplit {
    cd r1, r2, l2;
    double c, s;
};
// false: the block is not reproduced to 1e-12 (not unitary): keep the op
bool split_block(cd p, cd q, cd r, cd t, BlockSplit& o) {
    const cd I(0.0, 1.0);
    const double c = std::abs(p), s = std::abs(q);
    if (s < 1e-13) o = BlockSplit{p, t, 1.0, 1.0, 0.0};               // diagonal block
    else if (c < 1e-13) o = BlockSplit{1.0, I * q, I * r, 0.0, 1.0};  // anti-diagonal block
    else {
        o.c = c;
        o.s = s;
        o.r1 = p / c;
        o.r2 = I * q / s;
        o.l2 = t / (c * o.r2);
    }
    const cd P = o.c * o.r1, Q = -I * o.s * o.r2, R = -I * o.s * o.l2 * o.r1, T = o.c * o.l2 * o.r2;
    return std::abs(P - p) + std::abs(Q - q) + std::abs(R - r) + std::abs(T - t) < 1e-12;
}

bool genuine(const BlockSplit& b) { return b.c > 1e-13 && b.s > 1e-13; }

DevOp diag_of(const DevOp& like, const cd* v, int n) {
    DevOp d = like;
    d.kind = OPK_DIAG;
    d.flags = DIAG_STAGED;
    for (int k = 0; k < 16; ++k) {
        d.cd[k] = make_double2(0.0, 0.0);
        d.cf[k] = make_float2(0.f, 0.f);
    }
    for (int k = 0; k < n; ++k) {
        d.cd[k] = make_double2(v[k].real(), v[k].imag());
        d.cf[k] = make_float2((float)v[k].real(), (float)v[k].imag());
    }
    return d;
}

bool is_one(cd z) { return std::abs(z - cd(1.0, 0.0)) < 1e-15; }

// DENSE1 / PARITY2 ops with a genuine complex rotation become R-diagonal, rotation,
// L-diagonal (a diagonal factor that is the identity is left out)
std::vector<DevOp> split_rotations(std::vector<DevOp> in) {
    const cd I(0.0, 1.0);
    std::vector<DevOp> out;
    out.reserve(in.size() * 2);
    for (const DevOp& op : in) {
        auto c = [&](int k) { return cd(op.cd[k].x, op.cd[k].y); };
        bool real = true;
        for (int k = 0; k < 8; ++k) real &= op.cd[k].y == 0.0;
        if (op.kind == OPK_DENSE1 && !(op.flags & OPF_REAL) && !real) {
            BlockSplit b;
            if (split_block(c(0), c(1), c(2), c(3), b) && genuine(b)) {
                const cd rd[2] = {b.r1, b.r2}, ld[2] = {1.0, b.l2};
                if (!is_one(b.r1) || !is_one(b.r2)) out.push_back(diag_of(op, rd, 2));
                DevOp m = op;
                const cd v[4] = {b.c, -I * b.s, -I * b.s, b.c};
                for (int k = 0; k < 4; ++k) {
                    m.cd[k] = make_double2(v[k].real(), v[k].imag());
                    m.cf[k] = make_float2((float)v[k].real(), (float)v[k].imag());
                }
                m.flags = 0;
                out.push_back(m);
                if (!is_one(b.l2)) out.push_back(diag_of(op, ld, 2));
                continue;
            }
        }
        if (op.kind == OPK_PARITY2 && !real) {
            BlockSplit e, o;
            if (split_block(c(0), c(1), c(2), c(3), e) && split_block(c(4), c(5), c(6), c(7), o) &&
                (genuine(e) || genuine(o))) {
                // local index 0 = 00, 1 = 01, 2 = 10, 3 = 11: even block (0, 3), odd block (1, 2)
                const cd rd[4] = {e.r1, o.r1, o.r2, e.r2}, ld[4] = {1.0, 1.0, o.l2, e.l2};
                if (!is_one(e.r1) || !is_one(e.r2) || !is_one(o.r1) || !is_one(o.r2))
                    out.push_back(diag_of(op, rd, 4));
                DevOp m = op;
                const cd v[8] = {e.c, -I * e.s, -I * e.s, e.c, o.c, -I * o.s, -I * o.s, o.c};
                for (int k = 0; k < 16; ++k) {
                    m.cd[k] = make_double2(0.0, 0.0);
                    m.cf[k] = make_float2(0.f, 0.f);
                }
                for (int k = 0; k < 8; ++k) {
                    m.cd[k] = make_double2(v[k].real(), v[k].imag());
                    m.cf[k] = make_float2((float)v[k].real(), (float)v[k].imag());
                }
                m.flags = (e.s == 0.0 ? 1 : 0) | (o.s == 0.0 ? 2 : 0);
                out.push_back(m);
                if (!is_one(e.l2) || !is_one(o.l2)) out.push_back(diag_of(op, ld, 4));
                continue;
            }
        }
        out.push_back(op);
    }
    return out;
}
}  // namespace

// ----------------------------------------------------------------------------
// Stage-sweep scheduling (engine 2).  The tile stays in shared memory; the
// pass's op list is cut into stages of consecutive ops whose non-diagonal
// qubits fit in 4 tile bits S.  A stage is one conflict-free sweep: every
// thread loads 16-amplitude groups (the 16 values of S for fixed other bits)
// into registers, applies all the stage's ops there and stores them back.
// Bank spreading: the tile bits below `LB` pick the shared-memory bank
// (8-byte amplitudes: 16 per 128-byte row, LB = 4; 16-byte amplitudes:
// LB = 3).  Lanes run over the lowest free (non-S) bits; every stage bit below
// LB is XOR-rotated by one lane bit (perm[4 + k]), so the 32 lanes of a warp
// always hit distinct banks.  The kernel folds the rotation into per-thread
// coefficients, once per op.
// ----------------------------------------------------------------------------
constexpr int kMaxBackwardStageOps = 24;

void schedule_stages(Pass& p, int amp_bytes, bool allow_inner, bool split) {
    const int T = p.g.T;
    constexpr int K = 4;
    if (T < 12 || T > 13) return;
    const int LB = amp_bytes == 8 ? 4 : 3;
    // adjoint measurements only for the compiled adjoint kernels, and only plain ones
    // (a U^dag folded into a measurement belongs to the shared-memory adjoint kernel)
    for (const DevOp& op : p.ops)
        if ((op.kind == OPK_INNER && (!allow_inner || (op.flags & (INNER_PRE | INNER_PREDIAG)))) ||
            op.kind == OPK_JUMP || op.kind == OPK_STAGE)
            return;
    std::vector<DevOp> in = std::move(p.ops);
    // 1- and 2-qubit permutations run as dense matrices on the stage registers
    for (DevOp& op : in) {
        if (op.kind != OPK_MONO || op.nq > 2) continue;
        const int dim = 1 << op.nq;
        double2 d[4];
        float2 f[4];
        for (int r = 0; r < dim; ++r) d[r] = op.cd[r], f[r] = op.cf[r];
        for (int k = 0; k < 16; ++k) {
            op.cd[k] = make_double2(0.0, 0.0);
            op.cf[k] = make_float2(0.f, 0.f);
        }
        for (int r = 0; r < dim; ++r) {
            op.cd[r * dim + op.perm[r]] = d[r];
            op.cf[r * dim + op.perm[r]] = f[r];
        }
        op.kind = op.nq == 1 ? OPK_DENSE1 : OPK_DENSE2;
    }
    if (split) in = split_rotations(std::move(in));
    std::vector<DevOp> out;
    auto needs = [](const DevOp& op) {
        std::vector<int> v;
        if ((op.kind == OPK_DIAG && !(op.flags & DIAG_STAGED)) || op.kind == OPK_STATESCALE ||
            op.kind == OPK_REALTAB)
            return v;
        for (int t = 0; t < op.nq; ++t) v.push_back(op.lb[t]);
        return v;
    };
    auto contains = [](const std::vector<int>& s, int b) { return std::find(s.begin(), s.end(), b) != s.end(); };
    auto header = [&](std::vector<int> S, int nmembers) {
        for (int b = LB; (int)S.size() < K && b < T; ++b)  // pad with bank-neutral bits first
            if (!contains(S, b)) S.push_back(b);
        for (int b = 0; (int)S.size() < K && b < T; ++b)
            if (!contains(S, b)) S.push_back(b);
        std::sort(S.begin(), S.end());
        DevOp h;
        std::memset(&h, 0, sizeof(h));
        h.kind = OPK_STAGE;
        h.nq = K;
        h.aux2 = nmembers;
        int c = 0;  // free bits below LB: the lowest lane bits
        for (int b = 0; b < LB; ++b)
            if (!contains(S, b)) ++c;
        int a = 0;
        for (int k = 0; k < 4; ++k) h.lb[k] = -1;
        for (int k = 0; k < K; ++k) {
            h.perm[k] = S[k];
            h.perm[4 + k] = S[k] < LB ? c + a++ : -1;
        }
        return h;
    };
    size_t i = 0;
    while (i < in.size()) {
        // a 3-qubit permutation (Toffoli) runs as a plain shared-memory sweep
        if (in[i].kind != OPK_DIAG && in[i].nq > 2) {
            DevOp h;
            std::memset(&h, 0, sizeof(h));
            h.kind = OPK_STAGE;
            h.nq = 0;
            h.aux2 = 1;
            out.push_back(h);
            out.push_back(in[i]);
            ++i;
            continue;
        }
        std::vector<int> S;
        size_t j = i;
        for (; j < in.size(); ++j) {
            if (in[j].kind != OPK_DIAG && in[j].nq > 2) break;
            // a backward stage holds two register sets: its length is capped, so the
            // compiled kernel's straight-line code per stage stays within registers
            if (allow_inner && (int)(j - i) >= kMaxBackwardStageOps) break;
            std::vector<int> U = S;
            for (int b : needs(in[j]))
                if (!contains(U, b)) U.push_back(b);
            if ((int)U.size() > K) break;
            S = U;
        }
        DevOp h = header(S, (int)(j - i));
        out.push_back(h);
        for (size_t k = i; k < j; ++k) {
            DevOp op = in[k];
            if (op.kind == OPK_INNER) {  // its slot[] holds the generator's i^k codes: keep them
                out.push_back(op);
                continue;
            }
            for (int t = 0; t < 4; ++t) op.slot[t] = -1;
            if (op.kind != OPK_DIAG && op.kind != OPK_STATESCALE && op.kind != OPK_REALTAB) {
                for (int t = 0; t < op.nq; ++t)
                    for (int q = 0; q < K; ++q)
                        if (h.perm[q] == op.lb[t]) op.slot[t] = q;
                if (op.nq == 2 && op.slot[0] > op.slot[1]) swap_qubit_roles(op);
            }
            out.push_back(op);
        }
        i = j;
    }
    p.ops = std::move(out);
    p.staged = true;
}

}  // namespace smoq

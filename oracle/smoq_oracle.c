/*
 * smoq_oracle.c -- CPU restatement of SmoQ.jl's state-vector hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product; see the header).
 * Each function names the reference file:line whose loop it restates.  The
 * loops deliberately keep the reference's shape (a scan over all 2^N
 * indices with a branch on the qubit bit, single-threaded per state) so the
 * CPU baseline built from this file times the work the Julia kernels do.
 */
#include "smoq_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <pthread.h>

#define I_ _Complex_I
typedef so_cplx C;

static inline C ld(const double* m, int idx) { return m[2 * idx] + I_ * m[2 * idx + 1]; }
/* column-major element (r, c) of an n x n matrix */
static inline C mat(const double* m, int n, int r, int c) { return ld(m, c * n + r); }

/* ---- threads over the amplitudes of ONE state ----
 * so_set_threads (default 1 = the reference's single-threaded loops).  Only
 * the parity tests at the measured sizes (N = 24..30) raise it, so that the
 * same loops finish in seconds.  run_range splits [0, 2^N) into contiguous
 * ranges, one per thread, and calls the loop body on each.  Every gate loop
 * below writes each amplitude from exactly one iteration (a pair or quartet
 * is updated by the iteration of its lowest index, the others skip), so the
 * split gives the same state; an observable's FP64 sum is the sum of the
 * ranges' partial sums in range order. */
static int so_nthreads = 1;
void so_set_threads(int n) { so_nthreads = n < 1 ? 1 : (n > 256 ? 256 : n); }
int so_get_threads(void) { return so_nthreads; }
typedef void (*range_fn)(int64_t lo, int64_t hi, const void* a, double* acc);
typedef struct {
    range_fn fn;
    const void* a;
    int64_t lo, hi;
    double acc;
} range_job;
static void* range_worker(void* p) {
    range_job* j = (range_job*)p;
    j->acc = 0;
    j->fn(j->lo, j->hi, j->a, &j->acc);
    return NULL;
}
static double run_range(int64_t dim, range_fn fn, const void* a) {
    int nt = so_nthreads;
    if (nt > dim / 4096) nt = (int)(dim / 4096);
    if (nt <= 1) {
        double acc = 0;
        fn(0, dim, a, &acc);
        return acc;
    }
    range_job jobs[256];
    pthread_t th[256];
    int started[256];
    for (int t = 0; t < nt; t++) {
        jobs[t].fn = fn;
        jobs[t].a = a;
        jobs[t].lo = dim / nt * t;
        jobs[t].hi = t == nt - 1 ? dim : dim / nt * (t + 1);
        jobs[t].acc = 0;
    }
    for (int t = 1; t < nt; t++) started[t] = pthread_create(&th[t], NULL, range_worker, &jobs[t]) == 0;
    range_worker(&jobs[0]);
    for (int t = 1; t < nt; t++) {
        if (started[t]) pthread_join(th[t], NULL);
        else range_worker(&jobs[t]);  /* no thread: run the range here */
    }
    double acc = 0;
    for (int t = 0; t < nt; t++) acc += jobs[t].acc;
    return acc;
}

double so_wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ========================================================================
 * Single-qubit gates -- utils/cpu/cpuQuantumChannelGates.jl
 * ======================================================================== */
typedef struct {
    C* psi;
    int k;
    int64_t step;
    double c, s;
    C is, ph[2];
} rot_args;
static void rx_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const rot_args* A = (const rot_args*)p;
    C* psi = A->psi;
    for (int64_t i = lo; i < hi; i++) {
        if (((i >> (A->k - 1)) & 1) == 0) {
            int64_t j = i + A->step;
            C a = psi[i], b = psi[j];
            psi[i] = A->c * a + A->is * b;
            psi[j] = A->is * a + A->c * b;
        }
    }
    (void)acc;
}
void so_apply_rx_psi(C* psi, int k, double theta, int N) { /* :142-161 */
    rot_args A = {psi, k, 1LL << (k - 1), cos(theta / 2), sin(theta / 2), 0, {0, 0}};
    A.is = -I_ * A.s;
    run_range(1LL << N, rx_range, &A);
}
static void ry_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const rot_args* A = (const rot_args*)p;
    C* psi = A->psi;
    for (int64_t i = lo; i < hi; i++) {
        if (((i >> (A->k - 1)) & 1) == 0) {
            int64_t j = i + A->step;
            C a = psi[i], b = psi[j];
            psi[i] = A->c * a - A->s * b;
            psi[j] = A->s * a + A->c * b;
        }
    }
    (void)acc;
}
void so_apply_ry_psi(C* psi, int k, double theta, int N) { /* :172-190 */
    rot_args A = {psi, k, 1LL << (k - 1), cos(theta / 2), sin(theta / 2), 0, {0, 0}};
    run_range(1LL << N, ry_range, &A);
}
static void rz_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const rot_args* A = (const rot_args*)p;
    for (int64_t i = lo; i < hi; i++) A->psi[i] *= A->ph[(i >> (A->k - 1)) & 1];
    (void)acc;
}
void so_apply_rz_psi(C* psi, int k, double theta, int N) { /* :201-212 */
    rot_args A = {psi, k, 0, 0, 0, 0, {cexp(-I_ * theta / 2), cexp(I_ * theta / 2)}};
    run_range(1LL << N, rz_range, &A);
}
void so_apply_hadamard_psi(C* psi, int k, int N) { /* :222-238 */
    double s = 1 / sqrt(2.0);
    int64_t step = 1LL << (k - 1), dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) {
        if (((i >> (k - 1)) & 1) == 0) {
            int64_t j = i + step;
            C a = psi[i], b = psi[j];
            psi[i] = s * (a + b);
            psi[j] = s * (a - b);
        }
    }
}
void so_apply_pauli_x_psi(C* psi, int k, int N) { /* :245-257 */
    int64_t step = 1LL << (k - 1), dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) {
        if (((i >> (k - 1)) & 1) == 0) {
            int64_t j = i + step;
            C t = psi[i]; psi[i] = psi[j]; psi[j] = t;
        }
    }
}
void so_apply_pauli_y_psi(C* psi, int k, int N) { /* :265-280 */
    int64_t step = 1LL << (k - 1), dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) {
        if (((i >> (k - 1)) & 1) == 0) {
            int64_t j = i + step;
            C v0 = psi[i], v1 = psi[j];
            psi[i] = -I_ * v1;
            psi[j] = I_ * v0;
        }
    }
}
static void phase_on_set_bit(C* psi, int k, int N, C ph) {
    int64_t dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++)
        if (((i >> (k - 1)) & 1) == 1) psi[i] *= ph;
}
void so_apply_pauli_z_psi(C* psi, int k, int N) { /* :286-296 */
    int64_t dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++)
        if (((i >> (k - 1)) & 1) == 1) psi[i] = -psi[i];
}
void so_apply_s_psi(C* psi, int k, int N) { phase_on_set_bit(psi, k, N, I_); }        /* :307 */
void so_apply_sdagger_psi(C* psi, int k, int N) { phase_on_set_bit(psi, k, N, -I_); } /* :328 */
void so_apply_t_psi(C* psi, int k, int N) { /* :360 */
    phase_on_set_bit(psi, k, N, cexp(I_ * M_PI / 4));
}
void so_apply_tdagger_psi(C* psi, int k, int N) { /* :380 */
    phase_on_set_bit(psi, k, N, cexp(-I_ * M_PI / 4));
}

/* ========================================================================
 * Multi-qubit gates
 * ======================================================================== */
void so_apply_ccz_psi(C* psi, int q1, int q2, int q3, int N) { /* :448-461 */
    int64_t dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) {
        int b1 = (i >> (q1 - 1)) & 1, b2 = (i >> (q2 - 1)) & 1, b3 = (i >> (q3 - 1)) & 1;
        if (b1 && b2 && b3) psi[i] = -psi[i];
    }
}
void so_apply_toffoli_psi(C* psi, int c1, int c2, int t, int N) { /* :471-489 */
    int64_t dim = 1LL << N, ts = 1LL << (t - 1);
    for (int64_t i = 0; i < dim; i++) {
        int b1 = (i >> (c1 - 1)) & 1, b2 = (i >> (c2 - 1)) & 1, bt = (i >> (t - 1)) & 1;
        if (b1 && b2 && !bt) {
            int64_t j = i + ts;
            C x = psi[i]; psi[i] = psi[j]; psi[j] = x;
        }
    }
}
void so_apply_cnot_psi(C* psi, int control, int target, int N) { /* :870-882 */
    int64_t dim = 1LL << N, ts = 1LL << (target - 1);
    for (int64_t i = 0; i < dim; i++) {
        if (((i >> (control - 1)) & 1) == 1 && ((i >> (target - 1)) & 1) == 0) {
            int64_t j = i + ts;
            C x = psi[i]; psi[i] = psi[j]; psi[j] = x;
        }
    }
}
typedef struct {
    C* psi;
    int qi, qj;
    C same, diff;
} pair_args;
static void cz_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const pair_args* A = (const pair_args*)p;
    for (int64_t idx = lo; idx < hi; idx++) {
        int bi = (idx >> (A->qi - 1)) & 1, bj = (idx >> (A->qj - 1)) & 1;
        A->psi[idx] *= (double)(1 - 2 * (bi & bj));
    }
    (void)acc;
}
void so_apply_cz_psi(C* psi, int qi, int qj, int N) { /* :889-900 (branchless sign) */
    pair_args A = {psi, qi, qj, 0, 0};
    run_range(1LL << N, cz_range, &A);
}
void so_apply_cry_psi(C* psi, int control, int target, double theta, int N) { /* :914-943 */
    double c = cos(theta / 2), s = sin(theta / 2);
    int64_t dim = 1LL << N, ts = 1LL << (target - 1);
    for (int64_t i = 0; i < dim; i++) {
        if (((i >> (control - 1)) & 1) == 1 && ((i >> (target - 1)) & 1) == 0) {
            int64_t j = i + ts;
            C a = psi[i], b = psi[j];
            psi[i] = c * a - s * b;
            psi[j] = s * a + c * b;
        }
    }
}
/* :992-1028 and :1039-1073: quartet loops over "base" with both bits 0 */
static void rpp_quartet(C* psi, int qi, int qj, C m00_11, C m01_10, C m10_01, C m11_00,
                        double c, int N) {
    int64_t dim = 1LL << N, si = 1LL << (qi - 1), sj = 1LL << (qj - 1);
    for (int64_t base = 0; base < dim; base++) {
        if (((base >> (qi - 1)) & 1) != 0 || ((base >> (qj - 1)) & 1) != 0) continue;
        int64_t i00 = base, i01 = base + sj, i10 = base + si, i11 = base + si + sj;
        C p00 = psi[i00], p01 = psi[i01], p10 = psi[i10], p11 = psi[i11];
        psi[i00] = c * p00 + m00_11 * p11;
        psi[i01] = c * p01 + m01_10 * p10;
        psi[i10] = m10_01 * p01 + c * p10;
        psi[i11] = m11_00 * p00 + c * p11;
    }
}
void so_apply_rxx_psi(C* psi, int qi, int qj, double theta, int N) { /* :992 */
    double c = cos(theta / 2), s = sin(theta / 2);
    C is = -I_ * s;
    rpp_quartet(psi, qi, qj, is, is, is, is, c, N);
}
void so_apply_ryy_psi(C* psi, int qi, int qj, double theta, int N) { /* :1039 */
    double c = cos(theta / 2), s = sin(theta / 2);
    C is = -I_ * s, isn = I_ * s;
    rpp_quartet(psi, qi, qj, isn, is, is, isn, c, N);
}
static void rzz_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const pair_args* A = (const pair_args*)p;
    for (int64_t idx = lo; idx < hi; idx++) {
        int bi = (idx >> (A->qi - 1)) & 1, bj = (idx >> (A->qj - 1)) & 1;
        A->psi[idx] *= (bi == bj) ? A->same : A->diff;
    }
    (void)acc;
}
void so_apply_rzz_psi(C* psi, int qi, int qj, double theta, int N) { /* :1084-1100 */
    pair_args A = {psi, qi, qj, cexp(-I_ * theta / 2), cexp(I_ * theta / 2)};
    run_range(1LL << N, rzz_range, &A);
}

/* ========================================================================
 * Jump operators
 * ======================================================================== */
void so_apply_sigma_minus_psi(C* psi, int k, int N) { /* :739-752 */
    int64_t dim = 1LL << N, mask = 1LL << (k - 1);
    for (int64_t i = 0; i < dim; i++) {
        if (i & mask) {
            int64_t j = i ^ mask;
            psi[j] = psi[i];
            psi[i] = 0;
        }
    }
}
void so_apply_sigma_plus_psi(C* psi, int k, int N) { /* :762-775 */
    int64_t dim = 1LL << N, mask = 1LL << (k - 1);
    for (int64_t i = 0; i < dim; i++) {
        if ((i & mask) == 0) {
            int64_t j = i | mask;
            psi[j] = psi[i];
            psi[i] = 0;
        }
    }
}
double so_population_excited_psi(const C* psi, int k, int N) { /* :784-796 */
    int64_t dim = 1LL << N, mask = 1LL << (k - 1);
    double r = 0;
    for (int64_t i = 0; i < dim; i++)
        if (i & mask) r += creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
    return r;
}

/* ========================================================================
 * Generic bitwise gates
 * ======================================================================== */
typedef struct {
    C* psi;
    int64_t s1, s2;
    C u[4][4];
} gate_args;
static void one_qubit_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const gate_args* A = (const gate_args*)p;
    C* psi = A->psi;
    const int64_t step = A->s1;
    for (int64_t b = lo; b < hi; b++) {
        if ((b & step) == 0) {
            C a0 = psi[b], a1 = psi[b + step];
            psi[b] = A->u[0][0] * a0 + A->u[0][1] * a1;
            psi[b + step] = A->u[1][0] * a0 + A->u[1][1] * a1;
        }
    }
    (void)acc;
}
void so_apply_one_qubit_gate(C* psi, const double* U, int qubit, int N) {
    /* cpuQuantumChannelUnitaryEvolutionTrotter.jl:77-99 */
    gate_args A;
    A.psi = psi;
    A.s1 = 1LL << (qubit - 1);
    A.s2 = 0;
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) A.u[r][c] = mat(U, 2, r, c);
    run_range(1LL << N, one_qubit_range, &A);
}
static void two_qubit_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    /* cpuQuantumChannelUnitaryEvolutionTrotter.jl:123-139: basis order
     * |00>, |q1=1>, |q2=1>, |11> with q1 < q2 */
    const gate_args* A = (const gate_args*)p;
    C* psi = A->psi;
    const int64_t s1 = A->s1, s2 = A->s2;
    for (int64_t b = lo; b < hi; b++) {
        if ((b & s1) == 0 && (b & s2) == 0) {
            int64_t i0 = b, i1 = b + s1, i2 = b + s2, i3 = b + s1 + s2;
            C a[4] = {psi[i0], psi[i1], psi[i2], psi[i3]};
            C o[4];
            for (int r = 0; r < 4; r++)
                o[r] = A->u[r][0] * a[0] + A->u[r][1] * a[1] + A->u[r][2] * a[2] + A->u[r][3] * a[3];
            psi[i0] = o[0]; psi[i1] = o[1]; psi[i2] = o[2]; psi[i3] = o[3];
        }
    }
    (void)acc;
}
static void two_qubit_core(C* psi, const C u[4][4], int q1, int q2, int N) {
    gate_args A;
    A.psi = psi;
    A.s1 = 1LL << (q1 - 1);
    A.s2 = 1LL << (q2 - 1);
    memcpy(A.u, u, sizeof(A.u));
    run_range(1LL << N, two_qubit_range, &A);
}
void so_apply_two_qubit_gate(C* psi, const double* U, int q1, int q2, int N) {
    /* :107-142 -- if q1 > q2 the qubits are swapped, U is NOT permuted */
    if (q1 > q2) { int t = q1; q1 = q2; q2 = t; }
    C u[4][4];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) u[r][c] = mat(U, 4, r, c);
    two_qubit_core(psi, u, q1, q2, N);
}
void so_apply_2qubit_gate_ru(C* psi, const double* U, int q1, int q2, int N) {
    /* cpuQuantumChannelRandomUnitaries.jl:317-360 -- if q1 > q2, U <- SWAP U SWAP */
    C u[4][4];
    int perm[4] = {0, 1, 2, 3};
    if (q1 > q2) {
        int t = q1; q1 = q2; q2 = t;
        perm[1] = 2; perm[2] = 1;
    }
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) u[r][c] = mat(U, 4, perm[r], perm[c]);
    two_qubit_core(psi, u, q1, q2, N);
}

/* ========================================================================
 * Observables -- utils/cpu/cpuQuantumStateObservables.jl
 * ======================================================================== */
static inline double abs2(C z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }
typedef struct {
    const C* psi;
    int64_t xmask, zmask;
    C iy;
} obs_args;
static void zstring_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const obs_args* A = (const obs_args*)p;
    double r = 0;
    for (int64_t i = lo; i < hi; i++) r += abs2(A->psi[i]) * (double)(1 - 2 * (__builtin_popcountll(i & A->zmask) & 1));
    *acc = r;
}
double so_expect_z(const C* psi, int k, int N) { /* :201-210 */
    /* sum_i |psi_i|^2 (1 - 2 bit_k(i)): the Z string of the one bit */
    obs_args A = {psi, 0, 1LL << (k - 1), 0};
    return run_range(1LL << N, zstring_range, &A);
}
double so_expect_x(const C* psi, int k, int N) { /* :230-240 */
    int64_t dim = 1LL << N, step = 1LL << (k - 1);
    double r = 0;
    for (int64_t i = 0; i < dim; i++)
        if (((i >> (k - 1)) & 1) == 0) r += 2 * creal(conj(psi[i]) * psi[i + step]);
    return r;
}
double so_expect_y(const C* psi, int k, int N) { /* :256-267 (code sign: +2 Im) */
    int64_t dim = 1LL << N, step = 1LL << (k - 1);
    double r = 0;
    for (int64_t i = 0; i < dim; i++)
        if (((i >> (k - 1)) & 1) == 0) r += 2 * cimag(conj(psi[i]) * psi[i + step]);
    return r;
}
double so_expect_zz(const C* psi, int i, int j, int N) { /* :341-352 */
    /* sum_s |psi_s|^2 (1 - 2 (bit_i xor bit_j)): the Z string of the two bits */
    obs_args A = {psi, 0, (1LL << (i - 1)) | (1LL << (j - 1)), 0};
    if (i == j) return so_norm2(psi, N);
    return run_range(1LL << N, zstring_range, &A);
}
static double corr_pairs(const C* psi, int i, int j, int N, double s0011) {
    int64_t dim = 1LL << N, si = 1LL << (i - 1), sj = 1LL << (j - 1);
    double r = 0;
    for (int64_t s = 0; s < dim; s++) {
        if (((s >> (i - 1)) & 1) == 0 && ((s >> (j - 1)) & 1) == 0) {
            r += s0011 * 2 * creal(conj(psi[s]) * psi[s + si + sj]);
            r += 2 * creal(conj(psi[s + sj]) * psi[s + si]);
        }
    }
    return r;
}
double so_expect_xx(const C* psi, int i, int j, int N) { return corr_pairs(psi, i, j, N, 1.0); }  /* :385 */
double so_expect_yy(const C* psi, int i, int j, int N) { return corr_pairs(psi, i, j, N, -1.0); } /* :427 */

double so_norm2(const C* psi, int N) {
    obs_args A = {psi, 0, 0, 0};
    return run_range(1LL << N, zstring_range, &A);
}

/* Pauli string expectation.  Z-only strings: _expect_pauli_Z_string (:900).
 * Mixed strings: _expect_pauli_mixed_string (:948) visits each base with all
 * X/Y bits 0 and each flip pattern once and adds Re(coeff psi_bra^* psi_ket),
 * i.e. only the (bra<ket) half of the Hermitian sum -- its own docstring
 * example (GHZ <XXX> = 1, :835) comes out 0.5 from that loop.  This oracle
 * (and the CUDA library) returns the full expectation
 *     <P> = sum_i conj(psi_i) * phase(i) * psi_{i ^ flipmask}
 * which equals _expect_X/_expect_XX/_expect_YY (:230/:385/:427) on 1- and
 * 2-body strings, where the reference is self-consistent. */
/* Re sum_i conj(psi_{i ^ xmask}) i^{ny} (-1)^{popc(i & zmask)} psi_i over a range */
static void mixed_range(int64_t lo, int64_t hi, const void* p, double* acc) {
    const obs_args* A = (const obs_args*)p;
    C r = 0;
    for (int64_t i = lo; i < hi; i++) {
        int64_t j = i ^ A->xmask;
        double sg = (double)(1 - 2 * (__builtin_popcountll(i & A->zmask) & 1));
        r += conj(A->psi[j]) * A->iy * sg * A->psi[i];
    }
    *acc = creal(r);
}
double so_expect_pauli_string(const C* psi, int n, const char* ops, const int* qubits, int N) {
    int64_t dim = 1LL << N, xmask = 0, zmask = 0;
    int ny = 0;
    for (int t = 0; t < n; t++) {
        int64_t b = 1LL << (qubits[t] - 1);
        char o = ops[t];
        if (o == 'X' || o == 'x') xmask |= b;
        else if (o == 'Y' || o == 'y') { xmask |= b; zmask |= b; ny++; }
        else if (o == 'Z' || o == 'z') zmask |= b;
    }
    obs_args A = {psi, xmask, zmask, 1};
    if (xmask == 0) /* :900-930 */
        return run_range(dim, zstring_range, &A);
    /* P|i> = i^{ny} (-1)^{popc(i & zmask)} |i ^ xmask>  with Y = i X Z */
    for (int t = 0; t < ny; t++) A.iy *= I_;
    return run_range(dim, mixed_range, &A);
}

/* ========================================================================
 * Trotter -- utils/cpu/cpuQuantumChannelUnitaryEvolutionTrotter.jl
 * ======================================================================== */
static void put(double* U, int n, int r, int c, C v) {
    U[2 * (c * n + r)] = creal(v);
    U[2 * (c * n + r) + 1] = cimag(v);
}
int so_precompute_trotter_gates(const double* bonds, int nb, const double* fields, int nf,
                                double dt, so_trotter_gate* out) {
    /* :322-354.  exp(-i dt (Jx XX + Jy YY + Jz ZZ)): XX, YY, ZZ commute, so the
     * exponential is the product of the three, and in the basis
     * |00>,|01>,|10>,|11> (kron(A_hi, B_lo), Julia's kron order) it is block
     * diagonal on {|00>,|11>} and {|01>,|10>}:
     *   XX: |00><->|11>, |01><->|10> with +1;  YY: |00><->|11> with -1,
     *   |01><->|10> with +1;  ZZ: +1 on 00/11, -1 on 01/10.
     * even block {00,11}: H = Jz I + (Jx - Jy) sx  -> e^{-i Jz dt}(cos a I - i sin a sx), a=(Jx-Jy)dt
     * odd  block {01,10}: H = -Jz I + (Jx + Jy) sx -> e^{+i Jz dt}(cos b I - i sin b sx), b=(Jx+Jy)dt */
    int n = 0;
    for (int t = 0; t < nb; t++) {
        const double* b = bonds + 5 * t;
        double Jx = b[2], Jy = b[3], Jz = b[4];
        so_trotter_gate* g = out + n++;
        memset(g, 0, sizeof(*g));
        g->nq = 2; g->q[0] = (int)b[0]; g->q[1] = (int)b[1];
        double a = (Jx - Jy) * dt, bb = (Jx + Jy) * dt;
        C pe = cexp(-I_ * Jz * dt), po = cexp(I_ * Jz * dt);
        put(g->U, 4, 0, 0, pe * cos(a)); put(g->U, 4, 3, 3, pe * cos(a));
        put(g->U, 4, 0, 3, pe * (-I_ * sin(a))); put(g->U, 4, 3, 0, pe * (-I_ * sin(a)));
        put(g->U, 4, 1, 1, po * cos(bb)); put(g->U, 4, 2, 2, po * cos(bb));
        put(g->U, 4, 1, 2, po * (-I_ * sin(bb))); put(g->U, 4, 2, 1, po * (-I_ * sin(bb)));
    }
    for (int t = 0; t < nf; t++) {
        const double* f = fields + 4 * t;
        double hx = f[1], hy = f[2], hz = f[3];
        if (!(fabs(hx) > 1e-14 || fabs(hy) > 1e-14 || fabs(hz) > 1e-14)) continue; /* :346 */
        /* exp(-i dt h.sigma) = cos(|h|dt) I - i sin(|h|dt) (h.sigma)/|h| */
        double h = sqrt(hx * hx + hy * hy + hz * hz), c = cos(h * dt), s = sin(h * dt) / h;
        so_trotter_gate* g = out + n++;
        memset(g, 0, sizeof(*g));
        g->nq = 1; g->q[0] = (int)f[0];
        put(g->U, 2, 0, 0, c - I_ * s * hz);
        put(g->U, 2, 1, 1, c + I_ * s * hz);
        put(g->U, 2, 0, 1, -I_ * s * (hx - I_ * hy));
        put(g->U, 2, 1, 0, -I_ * s * (hx + I_ * hy));
    }
    return n;
}
void so_trotter_step(C* psi, const so_trotter_gate* g, int n, int N) { /* :150-162 */
    for (int t = 0; t < n; t++) {
        if (g[t].nq == 1) so_apply_one_qubit_gate(psi, g[t].U, g[t].q[0], N);
        else so_apply_two_qubit_gate(psi, g[t].U, g[t].q[0], g[t].q[1], N);
    }
}

/* ========================================================================
 * Circuits -- cpuVariationalQuantumCircuitExecutor.jl:95-180
 * ======================================================================== */
void so_apply_circuit(C* psi, const so_op* ops, int n, const double* theta, int N) {
    for (int t = 0; t < n; t++) {
        const so_op* o = ops + t;
        double a = o->param > 0 ? theta[o->param - 1] : o->angle; /* :147 */
        const int* q = o->q;
        switch (o->type) {
        case SO_G_RX: so_apply_rx_psi(psi, q[0], a, N); break;
        case SO_G_RY: so_apply_ry_psi(psi, q[0], a, N); break;
        case SO_G_RZ: so_apply_rz_psi(psi, q[0], a, N); break;
        case SO_G_H: so_apply_hadamard_psi(psi, q[0], N); break;
        case SO_G_X: so_apply_pauli_x_psi(psi, q[0], N); break;
        case SO_G_Y: so_apply_pauli_y_psi(psi, q[0], N); break;
        case SO_G_Z: so_apply_pauli_z_psi(psi, q[0], N); break;
        case SO_G_S: so_apply_s_psi(psi, q[0], N); break;
        case SO_G_SDG: so_apply_sdagger_psi(psi, q[0], N); break;
        case SO_G_T: so_apply_t_psi(psi, q[0], N); break;
        case SO_G_TDG: so_apply_tdagger_psi(psi, q[0], N); break;
        case SO_G_CZ: so_apply_cz_psi(psi, q[0], q[1], N); break;
        case SO_G_CNOT: so_apply_cnot_psi(psi, q[0], q[1], N); break;
        case SO_G_RXX: so_apply_rxx_psi(psi, q[0], q[1], a, N); break;
        case SO_G_RYY: so_apply_ryy_psi(psi, q[0], q[1], a, N); break;
        case SO_G_RZZ: so_apply_rzz_psi(psi, q[0], q[1], a, N); break;
        case SO_G_CRY: so_apply_cry_psi(psi, q[0], q[1], a, N); break;
        case SO_G_CCZ: so_apply_ccz_psi(psi, q[0], q[1], q[2], N); break;
        case SO_G_TOFFOLI: so_apply_toffoli_psi(psi, q[0], q[1], q[2], N); break;
        default: break;
        }
    }
}

double so_pauli_sum_expect(const C* psi, int nterms, const double* coef, const char* paulis, int N) {
    double e = 0;
    char ops[64];
    int qs[64];
    for (int t = 0; t < nterms; t++) {
        int n = 0;
        for (int q = 0; q < N; q++) {
            char p = paulis[(size_t)t * N + q];
            if (p == 'X' || p == 'Y' || p == 'Z') { ops[n] = p; qs[n] = q + 1; n++; }
        }
        e += coef[t] * (n ? so_expect_pauli_string(psi, n, ops, qs, N) : so_norm2(psi, N));
    }
    return e;
}

double so_energy(const so_op* ops, int n, const double* theta, int N, int nterms,
                 const double* coef, const char* paulis) {
    int64_t dim = 1LL << N;
    C* psi = (C*)calloc(dim, sizeof(C));
    psi[0] = 1;
    so_apply_circuit(psi, ops, n, theta, N);
    double e = so_pauli_sum_expect(psi, nterms, coef, paulis, N);
    free(psi);
    return e;
}

void so_grad_parameter_shift(const so_op* ops, int n, const double* theta, int P, int N,
                             int nterms, const double* coef, const char* paulis, double shift,
                             const int* which, int nwhich, double* grad) {
    /* cpuVariationalQuantumCircuitGradients.jl:138-163 */
    double* tp = (double*)malloc(P * sizeof(double));
    memcpy(tp, theta, P * sizeof(double));
    for (int w = 0; w < nwhich; w++) {
        int k = which[w];
        tp[k] = theta[k] + shift;
        double cp = so_energy(ops, n, tp, N, nterms, coef, paulis);
        tp[k] = theta[k] - shift;
        double cm = so_energy(ops, n, tp, N, nterms, coef, paulis);
        grad[w] = (cp - cm) / (2 * sin(shift));
        tp[k] = theta[k];
    }
    free(tp);
}

void so_grad_finite_difference(const so_op* ops, int n, const double* theta, int P, int N,
                               int nterms, const double* coef, const char* paulis, double eps,
                               const int* which, int nwhich, double* grad) {
    /* cpuVariationalQuantumCircuitGradients.jl:250-269 */
    double* tw = (double*)malloc(P * sizeof(double));
    memcpy(tw, theta, P * sizeof(double));
    for (int w = 0; w < nwhich; w++) {
        int k = which[w];
        tw[k] = theta[k] + eps;
        double cp = so_energy(ops, n, tw, N, nterms, coef, paulis);
        tw[k] = theta[k] - eps;
        double cm = so_energy(ops, n, tw, N, nterms, coef, paulis);
        grad[w] = (cp - cm) / (2 * eps);
        tw[k] = theta[k];
    }
    free(tw);
}

/* ========================================================================
 * H|psi> -- the matrix-free Hamiltonian applications of the Chebyshev and
 * Lanczos integrators
 * ======================================================================== */
/* apply_hamiltonian_bitwise! (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55-148),
 * the pull loop: for every row k, the x bonds, then the y bonds (ZZ from k
 * itself, XX and YY from k with both bits flipped), then the fields (Z from k,
 * X and Y from k with the bit flipped).  Bond rows (i, j, Jxx, Jyy, Jzz) and
 * field rows (idx, hx, hy, hz) with 1-based sites, as CouplingTerm / FieldTerm
 * (cpuHamiltonianBuilder.jl:42,51).  The Y field follows the Y of
 * construct_sparse_hamiltonian (cpuHamiltonianBuilder.jl:297: -i on rows with
 * the bit clear) and of apply_Y! (cpuQuantumStateLanczos.jl:84-94); the pull
 * loop's `phase_y = (val == 0) ? 1im : -1im` (Chebyshev.jl:142) is the
 * transpose, i.e. -hy Y. */
static C bond_pull(const C* in, int64_t k, const double* b) {
    int bit_i = (int)b[0] - 1, bit_j = (int)b[1] - 1;
    int64_t mask_flip = (1LL << bit_i) | (1LL << bit_j);
    int val_i = (int)((k >> bit_i) & 1), val_j = (int)((k >> bit_j) & 1);
    C acc = 0;
    if (b[4] != 0.0) acc += b[4] * (val_i == val_j ? 1.0 : -1.0) * in[k];
    int64_t k_flip = k ^ mask_flip;
    if (b[2] != 0.0) acc += b[2] * in[k_flip];
    if (b[3] != 0.0) acc += b[3] * (val_i == val_j ? -1.0 : 1.0) * in[k_flip];
    return acc;
}
void so_apply_hamiltonian_bitwise(C* out, const C* in, const double* x_bonds, int nx, const double* y_bonds, int ny,
                                  const double* fields, int nf, int N) {
    int64_t dim = 1LL << N;
    for (int64_t k = 0; k < dim; k++) {
        C acc = 0;
        for (int t = 0; t < nx; t++) acc += bond_pull(in, k, x_bonds + 5 * t);
        for (int t = 0; t < ny; t++) acc += bond_pull(in, k, y_bonds + 5 * t);
        for (int t = 0; t < nf; t++) {
            const double* f = fields + 4 * t;
            int bit_idx = (int)f[0] - 1;
            int64_t mask = 1LL << bit_idx;
            int val = (int)((k >> bit_idx) & 1);
            if (f[3] != 0.0) acc += f[3] * (val == 0 ? 1.0 : -1.0) * in[k];
            int64_t k_flip = k ^ mask;
            if (f[1] != 0.0) acc += f[1] * in[k_flip];
            if (f[2] != 0.0) acc += f[2] * (val == 0 ? -I_ : I_) * in[k_flip];
        }
        out[k] = acc;
    }
}
/* apply_H_xxz! (cpuQuantumStateLanczos.jl:157-205): out = Jx sum X_i X_{i+1} +
 * Jy sum Y_i Y_{i+1} + Jz sum Z_i Z_{i+1} + h sum X_i, term by term through a
 * temporary as the reference accumulates (apply_XX! :98, apply_YY! :118,
 * apply_ZZ! :86, apply_X! :70) */
void so_apply_H_xxz(const C* psi, C* out, int N, double Jx, double Jy, double Jz, double h) {
    int64_t dim = 1LL << N;
    C* temp = (C*)calloc(dim, sizeof(C));
    for (int64_t s = 0; s < dim; s++) out[s] = 0;
    for (int pass = 0; pass < 4; pass++) {
        double J = pass == 0 ? Jx : pass == 1 ? Jy : pass == 2 ? Jz : h;
        if (J == 0.0) continue;
        for (int i = 1; i <= (pass == 3 ? N : N - 1); i++) {
            for (int64_t s = 0; s < dim; s++) temp[s] = 0;
            if (pass == 3) {
                int64_t step = 1LL << (i - 1);
                for (int64_t a = 0; a < dim; a++)
                    if (((a >> (i - 1)) & 1) == 0) { temp[a] += psi[a + step]; temp[a + step] += psi[a]; }
            } else if (pass == 2) {
                for (int64_t a = 0; a < dim; a++) {
                    int bi = (int)((a >> (i - 1)) & 1), bj = (int)((a >> i) & 1);
                    temp[a] += (double)(1 - 2 * (bi ^ bj)) * psi[a];
                }
            } else {
                int64_t si = 1LL << (i - 1), sj = 1LL << i;
                double sg = pass == 1 ? -1.0 : 1.0;
                for (int64_t a = 0; a < dim; a++) {
                    if (((a >> (i - 1)) & 1) == 0 && ((a >> i) & 1) == 0) {
                        int64_t s00 = a, s01 = a + sj, s10 = a + si, s11 = a + si + sj;
                        temp[s00] += sg * psi[s11];
                        temp[s01] += psi[s10];
                        temp[s10] += psi[s01];
                        temp[s11] += sg * psi[s00];
                    }
                }
            }
            for (int64_t s = 0; s < dim; s++) out[s] += J * temp[s];
        }
    }
    free(temp);
}

/* ========================================================================
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with multipliers
 * 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 / 0xBB67AE85,
 * all as published in the paper.
 * ======================================================================== */
void so_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
double so_u01_from_words(uint32_t hi, uint32_t lo) {
    /* 53-bit uniform in [0,1): 27 bits of hi, 26 bits of lo */
    uint64_t a = hi >> 5, b = lo >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

/* ========================================================================
 * MCWF step -- the rule shared with the CUDA library.
 *
 * 1. coherent step: the first-order Trotter gate list (lindblad_mcwf_step_trotter!,
 *    cpuQuantumChannelLindbladianEvolutionMonteCarloWaveFunction.jl:282);
 * 2. no-jump decay, amplitude-wise
 *      psi_i *= sqrt(1 - dt * sum_{sigma_z, sigma_x ops} gamma)          (:285, L^dag L = I)
 *             * prod_{sigma_minus on k, bit k set}   sqrt(1 - gamma dt)  (:353-358, decay^popcount)
 *             * prod_{sigma_plus  on k, bit k clear} sqrt(1 - gamma dt);
 * 3. norm_sq = ||psi~||^2 in FP64, dp = 1 - norm_sq (:289-290);
 * 4. u1, u2 = two 53-bit uniforms from Philox4x32-10 with counter
 *    (step_lo, step_hi, traj_lo, traj_hi) and key (seed_lo, seed_hi);
 * 5. jump iff u1 < dp && dp > 0 (:293).  The channel is chosen with the
 *    independent u2 (the reference reuses r, caveat at :364-377) by weights
 *    w_c = gamma_c dt <L_c^dag L_c>_{psi~} / norm_sq, walking the op list in
 *    order and taking the first c with cumulative > u2 * sum(w);
 * 6. renormalise (:303 / :381-384): the post-jump norm^2 is the excited (ground)
 *    population for sigma_minus (sigma_plus) and norm_sq for sigma_z/sigma_x.
 * ======================================================================== */
static double pop_bit(const C* psi, int64_t dim, int64_t mask, int set) {
    double r = 0;
    for (int64_t i = 0; i < dim; i++)
        if (((i & mask) != 0) == set) r += abs2(psi[i]);
    return r;
}
int so_mcwf_step(C* psi, int N, const so_trotter_gate* g, int ng, const so_jump_op* ops,
                 int nops, double dt, uint64_t seed, uint64_t traj, uint64_t step) {
    int64_t dim = 1LL << N;
    so_trotter_step(psi, g, ng, N);
    double gz = 0;
    for (int o = 0; o < nops; o++)
        if (ops[o].type == 2 || ops[o].type == 3) gz += ops[o].gamma;
    double fu = sqrt(1.0 - dt * gz);
    for (int64_t i = 0; i < dim; i++) {
        double f = fu;
        for (int o = 0; o < nops; o++) {
            int bit = (int)((i >> (ops[o].qubit - 1)) & 1);
            if ((ops[o].type == 0 && bit) || (ops[o].type == 1 && !bit))
                f *= sqrt(1.0 - ops[o].gamma * dt);
        }
        psi[i] *= f;
    }
    double norm_sq = so_norm2(psi, N), dp = 1.0 - norm_sq;
    uint32_t ctr[4] = {(uint32_t)step, (uint32_t)(step >> 32), (uint32_t)traj, (uint32_t)(traj >> 32)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    so_philox4x32_10(ctr, key, w);
    double u1 = so_u01_from_words(w[0], w[1]), u2 = so_u01_from_words(w[2], w[3]);
    int chosen = -1;
    double new_norm_sq = norm_sq;
    if (u1 < dp && dp > 0) {
        double wsum = 0;
        double* wt = (double*)malloc((nops > 0 ? nops : 1) * sizeof(double));
        double* pops = (double*)malloc((nops > 0 ? nops : 1) * sizeof(double));
        for (int o = 0; o < nops; o++) {
            int64_t mask = 1LL << (ops[o].qubit - 1);
            double ev;
            if (ops[o].type == 0) pops[o] = ev = pop_bit(psi, dim, mask, 1);
            else if (ops[o].type == 1) pops[o] = ev = pop_bit(psi, dim, mask, 0);
            else { pops[o] = norm_sq; ev = norm_sq; }
            wt[o] = ops[o].gamma * dt * ev / norm_sq;
            wsum += wt[o];
        }
        if (wsum > 0) {
            double target = u2 * wsum, cum = 0;
            chosen = nops - 1;
            for (int o = 0; o < nops; o++) {
                cum += wt[o];
                if (target < cum) { chosen = o; break; }
            }
            int k = ops[chosen].qubit;
            switch (ops[chosen].type) {
            case 0: so_apply_sigma_minus_psi(psi, k, N); break;
            case 1: so_apply_sigma_plus_psi(psi, k, N); break;
            case 2: so_apply_pauli_z_psi(psi, k, N); break;
            case 3: so_apply_pauli_x_psi(psi, k, N); break;
            }
            new_norm_sq = pops[chosen];
        }
        free(wt);
        free(pops);
    }
    double inv = 1.0 / sqrt(new_norm_sq);
    for (int64_t i = 0; i < dim; i++) psi[i] *= inv;
    return chosen;
}

typedef struct {
    int N, ng, nops, steps, record_every, ntraj, nthreads, tid;
    const so_trotter_gate* g;
    const so_jump_op* ops;
    double dt;
    uint64_t seed, t0, init_index;
    double *z_out, *zz_out;
    int* njumps;
} mcwf_job;

static void* mcwf_worker(void* arg) {
    mcwf_job* J = (mcwf_job*)arg;
    int N = J->N;
    int64_t dim = 1LL << N;
    C* psi = (C*)malloc(dim * sizeof(C));
    for (int t = J->tid; t < J->ntraj; t += J->nthreads) { /* static round-robin */
        memset(psi, 0, dim * sizeof(C));
        psi[J->init_index] = 1;
        int jumps = 0, r = 0;
        for (int s = 0; s <= J->steps; s++) {
            if (s > 0 && so_mcwf_step(psi, N, J->g, J->ng, J->ops, J->nops, J->dt, J->seed,
                                      J->t0 + t, (uint64_t)(s - 1)) >= 0)
                jumps++;
            if (s % J->record_every == 0) {
                for (int q = 1; q <= N; q++)
                    J->z_out[((size_t)r * J->ntraj + t) * N + q - 1] = so_expect_z(psi, q, N);
                for (int q = 1; q < N; q++)
                    J->zz_out[((size_t)r * J->ntraj + t) * (N - 1) + q - 1] = so_expect_zz(psi, q, q + 1, N);
                r++;
            }
        }
        if (J->njumps) J->njumps[t] = jumps;
    }
    free(psi);
    return NULL;
}

void so_mcwf_run(int N, const so_trotter_gate* g, int ng, const so_jump_op* ops, int nops,
                 double dt, uint64_t seed, uint64_t t0, int ntraj, int steps, int record_every,
                 uint64_t init_index, double* z_out, double* zz_out, int* njumps, int nthreads) {
    /* trajectories are independent: spread them over host threads, as the
     * reference's Threads.@threads over trajectories does */
    if (nthreads < 1) nthreads = 1;
    if (nthreads > ntraj) nthreads = ntraj > 0 ? ntraj : 1;
    mcwf_job* jobs = (mcwf_job*)calloc(nthreads, sizeof(mcwf_job));
    pthread_t* th = (pthread_t*)calloc(nthreads, sizeof(pthread_t));
    for (int i = 0; i < nthreads; i++) {
        mcwf_job J = {N, ng, nops, steps, record_every, ntraj, nthreads, i, g, ops, dt,
                      seed, t0, init_index, z_out, zz_out, njumps};
        jobs[i] = J;
    }
    for (int i = 1; i < nthreads; i++) pthread_create(&th[i], NULL, mcwf_worker, &jobs[i]);
    mcwf_worker(&jobs[0]);
    for (int i = 1; i < nthreads; i++) pthread_join(th[i], NULL);
    free(jobs);
    free(th);
}

/* ========================================================================
 * Density-matrix oracle (column-major rho[(j * dim) + i] = rho_ij)
 * ======================================================================== */
static void rows_apply(C* rho, int64_t dim, const so_trotter_gate* g, const C u[4][4], int nq) {
    /* right-multiply by U^dag on rows, as apply_fast_trotter_gates_to_matrix_rows_cpu!
     * (:178-230) does with the conjugated gates: M[i, c] = sum conj(U)[c, c'] M[i, c'] */
    if (nq == 1) {
        int64_t step = 1LL << (g->q[0] - 1);
        for (int64_t k = 0; k < dim; k++) {
            if (k & step) continue;
            for (int64_t i = 0; i < dim; i++) {
                C a0 = rho[k * dim + i], a1 = rho[(k + step) * dim + i];
                rho[k * dim + i] = conj(u[0][0]) * a0 + conj(u[0][1]) * a1;
                rho[(k + step) * dim + i] = conj(u[1][0]) * a0 + conj(u[1][1]) * a1;
            }
        }
    } else {
        int q1 = g->q[0], q2 = g->q[1];
        int64_t s1 = 1LL << (q1 - 1), s2 = 1LL << (q2 - 1);
        for (int64_t k = 0; k < dim; k++) {
            if ((k & s1) || (k & s2)) continue;
            int64_t c[4] = {k, k + s1, k + s2, k + s1 + s2};
            for (int64_t i = 0; i < dim; i++) {
                C v[4], o[4];
                for (int a = 0; a < 4; a++) v[a] = rho[c[a] * dim + i];
                for (int r = 0; r < 4; r++)
                    o[r] = conj(u[r][0]) * v[0] + conj(u[r][1]) * v[1] + conj(u[r][2]) * v[2] + conj(u[r][3]) * v[3];
                for (int a = 0; a < 4; a++) rho[c[a] * dim + i] = o[a];
            }
        }
    }
}
void so_trotter_step_rho(C* rho, const so_trotter_gate* g, int n, int N) {
    /* evolve_trotter_rho_cpu! (:266-285): U on every column, then U^dag on rows */
    int64_t dim = 1LL << N;
    for (int64_t j = 0; j < dim; j++) so_trotter_step(rho + j * dim, g, n, N);
    for (int t = 0; t < n; t++) {
        C u[4][4];
        int nn = g[t].nq == 1 ? 2 : 4;
        for (int r = 0; r < nn; r++)
            for (int c = 0; c < nn; c++) u[r][c] = mat(g[t].U, nn, r, c);
        /* 2-qubit row gates: the reference row kernel does not swap q1>q2;
         * gates built by the precompute have q1 < q2 */
        rows_apply(rho, dim, g + t, u, g[t].nq);
    }
}
void so_dissipator_dm(C* rho, const so_jump_op* op, double dt, int N) {
    /* _apply_dissipator_dm! (cpuQuantumChannelLindbladianEvolution.jl:377-460),
     * same in-place loop order (j outer, i inner) */
    int64_t dim = 1LL << N, mask = 1LL << (op->qubit - 1);
    double f = op->gamma * dt;
    int qb = op->qubit - 1;
    for (int64_t j = 0; j < dim; j++) {
        for (int64_t i = 0; i < dim; i++) {
            int bi = (int)((i >> qb) & 1), bj = (int)((j >> qb) & 1);
            C* rij = rho + j * dim + i;
            if (op->type == 0) {
                if (bi && bj) {
                    rho[(j ^ mask) * dim + (i ^ mask)] += f * (*rij);
                    *rij *= (1 - f);
                } else if (bi || bj) *rij *= (1 - 0.5 * f);
            } else if (op->type == 1) {
                if (!bi && !bj) {
                    rho[(j ^ mask) * dim + (i ^ mask)] += f * (*rij);
                    *rij *= (1 - f);
                } else if (!bi || !bj) *rij *= (1 - 0.5 * f);
            } else if (op->type == 2) {
                if (bi != bj) *rij *= (1 - 2 * f);
            } else {
                int64_t ifl = i ^ mask, jfl = j ^ mask;
                if (i < ifl || (i == ifl && j < jfl)) {
                    C vo = *rij, vf = rho[jfl * dim + ifl];
                    *rij += f * (vf - vo);
                    rho[jfl * dim + ifl] += f * (vo - vf);
                }
            }
        }
    }
}
double so_expect_z_rho(const C* rho, int k, int N) {
    int64_t dim = 1LL << N;
    double r = 0;
    for (int64_t i = 0; i < dim; i++) r += creal(rho[i * dim + i]) * (double)(1 - 2 * ((i >> (k - 1)) & 1));
    return r;
}
double so_expect_zz_rho(const C* rho, int a, int b, int N) {
    int64_t dim = 1LL << N;
    double r = 0;
    for (int64_t i = 0; i < dim; i++)
        r += creal(rho[i * dim + i]) * (double)(1 - 2 * (((i >> (a - 1)) ^ (i >> (b - 1))) & 1));
    return r;
}

/* ========================================================================
 * Born sampling and projective Z measurements
 * (utils/cpu/cpuQuantumStateMeasurements.jl), with the uniforms drawn from
 * Philox4x32-10 -- counter (shot_lo, shot_hi, stream_lo, stream_hi), key
 * (seed_lo, seed_hi), u from the first two words -- so that the CUDA library
 * can be checked draw for draw.
 * ======================================================================== */
static double shot_u(uint64_t seed, uint64_t shot, uint64_t stream) {
    uint32_t ctr[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    so_philox4x32_10(ctr, key, w);
    return so_u01_from_words(w[0], w[1]);
}
/* the benchmark's shot loop: cumprobs = cumsum(abs2.(psi)), idx =
 * searchsortedfirst(cumprobs, r) - 1 (run_benchmark_smoq_Float64.jl:424-435);
 * an r above the total takes the last index, as sample_from_probabilities (:203) */
void so_sample(const so_cplx* psi, int N, int64_t nshots, uint64_t seed, uint64_t stream, int64_t* out) {
    int64_t dim = 1LL << N;
    double* cum = (double*)malloc(dim * sizeof(double));
    double run = 0;
    for (int64_t i = 0; i < dim; i++) {
        run += abs2(psi[i]);
        cum[i] = run;
    }
    for (int64_t s = 0; s < nshots; s++) {
        double r = shot_u(seed, (uint64_t)s, stream);
        int64_t lo = 0, hi = dim - 1;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (cum[mid] >= r) hi = mid;
            else lo = mid + 1;
        }
        out[s] = lo;
    }
    free(cum);
}
/* projective_measurement_all! (:484): one sample, collapse onto it */
int64_t so_measure_all(so_cplx* psi, int N, uint64_t seed, uint64_t stream) {
    int64_t idx;
    so_sample(psi, N, 1, seed, stream, &idx);
    int64_t dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) psi[i] = 0;
    psi[idx] = 1.0;
    return idx;
}
/* _measure_z_single! (:224), k 1-based */
int so_measure_z_u(so_cplx* psi, int k, int N, double u) { /* _measure_z_single! :224-255, rand() = u */
    int64_t dim = 1LL << N, mask = 1LL << (k - 1);
    double prob_0 = 0;
    for (int64_t i = 0; i < dim; i++)
        if ((i & mask) == 0) prob_0 += abs2(psi[i]);
    int outcome = u < prob_0 ? 0 : 1;
    double norm_sq = 0;
    for (int64_t i = 0; i < dim; i++) {
        int bit = (int)((i >> (k - 1)) & 1);
        if (bit != outcome) psi[i] = 0;
        else norm_sq += abs2(psi[i]);
    }
    double f = 1.0 / sqrt(norm_sq);
    for (int64_t i = 0; i < dim; i++) psi[i] *= f;
    return outcome;
}
int so_measure_qubit(so_cplx* psi, int k, int N, uint64_t seed, uint64_t stream) {
    return so_measure_z_u(psi, k, N, shot_u(seed, 0, stream));
}

/* ========================================================================
 * Circuits with noise, measurements, resets and classical conditions: the
 * pure-state branch of apply_circuit! (cpuVariationalQuantumCircuitExecutor.jl:95-146).
 * Each restated routine takes the uniform u that the reference draws with rand().
 * ======================================================================== */
static void pauli_x_bit(C* psi, int k, int N) { /* the X loops of :287-296 / :322-331 */
    int64_t mask = 1LL << (k - 1), dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++) {
        if ((i & mask) == 0) {
            int64_t j = i | mask;
            C t = psi[i]; psi[i] = psi[j]; psi[j] = t;
        }
    }
}
static void pauli_z_bit(C* psi, int k, int N) { /* the Z loops of :271-279 / :307-315 / :338-345 */
    int64_t dim = 1LL << N;
    for (int64_t i = 0; i < dim; i++)
        if (((i >> (k - 1)) & 1) == 1) psi[i] = -psi[i];
}
/* utils/cpu/cpuQuantumChannelKrausOperators.jl:262-282 */
void so_noise_dephasing_u(C* psi, double p, int k, int N, double u) {
    if (p == 0.0) return;                                   /* p ≈ 0.0 */
    double q = (1.0 - sqrt(1.0 - p)) / 2.0;
    if (u < q) pauli_z_bit(psi, k, N);
}
/* :285-318 */
void so_noise_depolarizing_u(C* psi, double p, int k, int N, double u) {
    double r = u;
    if (r < p / 3) {
        pauli_x_bit(psi, k, N);
    } else if (r < 2 * p / 3) {
        int64_t mask = 1LL << (k - 1), dim = 1LL << N;
        for (int64_t i = 0; i < dim; i++) {
            if ((i & mask) == 0) {
                int64_t j = i | mask;
                C a = psi[i], b = psi[j];
                psi[i] = -I_ * b;
                psi[j] = I_ * a;
            }
        }
    } else if (r < p) {
        pauli_z_bit(psi, k, N);
    }
}
/* :321-334 */
void so_noise_bit_flip_u(C* psi, double p, int k, int N, double u) {
    if (u < p) pauli_x_bit(psi, k, N);
}
/* :337-347 */
void so_noise_phase_flip_u(C* psi, double p, int k, int N, double u) {
    if (u < p) pauli_z_bit(psi, k, N);
}
/* :350-386.  The jump follows the sigma- operator, psi[i_ground] = psi[i]
 * (apply_sigma_minus_psi!, cpuQuantumChannelGates.jl:746), not the line
 * `psi[i_ground+1] += psi[i+1]` of :367: only the replacing jump unravels the
 * same file's Kraus channel (:145-180) that the trajectory mean must match. */
void so_noise_amplitude_damping_u(C* psi, double gamma, int k, int N, double u) {
    int64_t mask = 1LL << (k - 1), dim = 1LL << N;
    double pop_1 = 0.0;
    for (int64_t i = 0; i < dim; i++)
        if ((i & mask) != 0) pop_1 += abs2(psi[i]);
    double p_jump = gamma * pop_1;
    if (u < p_jump && pop_1 > 1e-12) {
        for (int64_t i = 0; i < dim; i++) {
            if ((i & mask) != 0) {
                int64_t i_ground = i ^ mask;
                psi[i_ground] = psi[i];
                psi[i] = 0.0;
            }
        }
    } else {
        double s = sqrt(1 - gamma);
        for (int64_t i = 0; i < dim; i++)
            if ((i & mask) != 0) psi[i] *= s;
    }
    double nrm = 0;
    for (int64_t i = 0; i < dim; i++) nrm += abs2(psi[i]);
    nrm = sqrt(nrm);
    if (nrm > 1e-12)
        for (int64_t i = 0; i < dim; i++) psi[i] /= nrm;
}
/* _normalize! (cpuQuantumStateMeasurements.jl:629-635) */
static void normalize_1e15(C* psi, int N) {
    int64_t dim = 1LL << N;
    double ns = 0;
    for (int64_t i = 0; i < dim; i++) ns += abs2(psi[i]);
    if (ns > 1e-15) {
        double f = sqrt(ns);
        for (int64_t i = 0; i < dim; i++) psi[i] /= f;
    }
}
/* _force_qubit_state! (cpuQuantumStateMeasurements.jl:584-627): target 0 :zero, 1 :one, 2 :plus, 3 :minus */
static void force_qubit_state(C* psi, int k, int target, int N) {
    int64_t dim = 1LL << N, mask = 1LL << (k - 1);
    if (target == 0 || target == 2) {
        for (int64_t i = 0; i < dim; i++) {
            if ((i & mask) != 0) {
                int64_t j = i ^ mask;
                psi[j] += psi[i];
                psi[i] = 0;
            }
        }
    } else {
        for (int64_t i = 0; i < dim; i++) {
            if ((i & mask) == 0) {
                int64_t j = i ^ mask;
                psi[j] += psi[i];
                psi[i] = 0;
            }
        }
    }
    normalize_1e15(psi, N);
    if (target >= 2) so_apply_hadamard_psi(psi, k, N);
}
/* reset_state! (cpuQuantumStateMeasurements.jl:555-567): measure in Z, then force */
void so_reset_u(C* psi, int k, int target, int N, double u) {
    so_measure_z_u(psi, k, N, u);
    force_qubit_state(psi, k, target, N);
}
/* the draw of stochastic op `op_index` of trajectory `traj` (the CUDA library's rule) */
double so_circuit_draw(uint64_t seed, uint32_t op_index, uint64_t traj) {
    uint32_t ctr[4] = {op_index, 0x80000000u, (uint32_t)traj, (uint32_t)(traj >> 32)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    so_philox4x32_10(ctr, key, w);
    return so_u01_from_words(w[0], w[1]);
}
int so_apply_circuit_mcwf(C* psi, const so_op* ops, int n, const double* theta, int N, uint64_t seed,
                          uint64_t traj, int* outcomes) {
    int nout = 0;
    for (int t = 0; t < n; t++) {
        const so_op* o = ops + t;
        const int cond = o->pad;                   /* CircuitOperation.if_outcome */
        if (cond > 0 && (cond > nout || outcomes[cond - 1] != 1)) continue;   /* Executor.jl:103-105 */
        const int k = o->q[0];
        switch (o->type) {                         /* apply_operation! :124-140, apply_noise_mcwf! :187-201 */
        case SO_N_DEPOLARIZING: so_noise_depolarizing_u(psi, o->angle, k, N, so_circuit_draw(seed, t, traj)); break;
        case SO_N_AMPLITUDE_DAMPING:
            so_noise_amplitude_damping_u(psi, o->angle, k, N, so_circuit_draw(seed, t, traj));
            break;
        case SO_N_DEPHASING:
        case SO_N_PHASE_DAMPING: so_noise_dephasing_u(psi, o->angle, k, N, so_circuit_draw(seed, t, traj)); break;
        case SO_N_BIT_FLIP: so_noise_bit_flip_u(psi, o->angle, k, N, so_circuit_draw(seed, t, traj)); break;
        case SO_N_PHASE_FLIP: so_noise_phase_flip_u(psi, o->angle, k, N, so_circuit_draw(seed, t, traj)); break;
        case SO_N_THERMAL_RELAXATION: case SO_T_TRACE_OUT: case SO_L_LINDBLAD_STEP: break;
        case SO_M_MEASURE_Z:                       /* projective_measurement! :319-345 */
            outcomes[nout++] = so_measure_z_u(psi, k, N, so_circuit_draw(seed, t, traj));
            break;
        case SO_M_MEASURE_X:
            so_apply_hadamard_psi(psi, k, N);
            outcomes[nout++] = so_measure_z_u(psi, k, N, so_circuit_draw(seed, t, traj));
            so_apply_hadamard_psi(psi, k, N);
            break;
        case SO_M_MEASURE_Y:
            so_apply_sdagger_psi(psi, k, N);
            so_apply_hadamard_psi(psi, k, N);
            outcomes[nout++] = so_measure_z_u(psi, k, N, so_circuit_draw(seed, t, traj));
            so_apply_hadamard_psi(psi, k, N);
            so_apply_s_psi(psi, k, N);
            break;
        case SO_R_RESET: so_reset_u(psi, k, o->q[1], N, so_circuit_draw(seed, t, traj)); break;
        default: so_apply_circuit(psi, o, 1, theta, N); break;   /* gates: apply_gate_psi! :146 */
        }
    }
    return nout;
}

/* ========================================================================
 * Quantum reservoir computing, bitwise MCWF path
 * (utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:451-530, :531-590;
 * utils/cpu/cpuQRCstep.jl:96-113, :332-433, :457-475)
 * ======================================================================== */
int so_qrc_n_ops(int L, int n_rails) {
    int N = L * n_rails;
    return 3 * N + 3 * (L - 1) * n_rails + 3 * L * (n_rails - 1);
}
/* measure_all_observables_state_vector_cpu! (cpuQuantumStateObservables.jl:1483-1519) */
void so_measure_all_observables(const C* psi, int L, int n_rails, double* out) {
    int N = L * n_rails, idx = 0;
    for (int k = 1; k <= N; k++) {
        out[idx++] = so_expect_x(psi, k, N);
        out[idx++] = so_expect_y(psi, k, N);
        out[idx++] = so_expect_z(psi, k, N);
    }
    for (int rail = 1; rail <= n_rails; rail++)
        for (int site = 1; site <= L - 1; site++) {
            int i = (rail - 1) * L + site, j = i + 1;
            out[idx++] = so_expect_xx(psi, i, j, N);
            out[idx++] = so_expect_yy(psi, i, j, N);
            out[idx++] = so_expect_zz(psi, i, j, N);
        }
    for (int rail = 1; rail <= n_rails - 1; rail++)
        for (int site = 1; site <= L; site++) {
            int i = (rail - 1) * L + site, j = rail * L + site;
            out[idx++] = so_expect_xx(psi, i, j, N);
            out[idx++] = so_expect_yy(psi, i, j, N);
            out[idx++] = so_expect_zz(psi, i, j, N);
        }
}
/* the input window of step k (0-based), :481-489, from padded_u (T + L values,
 * [zeros(L); u] in run_mcwf_simulation): :batch -> win[q] = padded_u[k + q]
 * (1-based k, q), :broadcast -> padded_u[k + L] */
void so_qrc_window(const double* padded_u, int L, int k, int encoding, double* win) {
    for (int q = 0; q < L; q++) win[q] = padded_u[encoding == 1 ? (int64_t)k + L : (int64_t)k + q + 1];
}
/* encode_input_ry_psi! (cpuQRCstep.jl:96): |0..0>, then Ry(pi u_q) on qubit q */
void so_qrc_encode(const double* win, int L, C* psi_in) {
    int64_t dim = 1LL << L;
    for (int64_t i = 0; i < dim; i++) psi_in[i] = 0;
    psi_in[0] = 1;
    for (int k = 1; k <= L; k++) so_apply_ry_psi(psi_in, k, M_PI * win[k - 1], L);
}
/* qrc_reset_psi! (cpuQRCstep.jl:332-433) for L_in = L_res = L; returns the outcome */
int so_qrc_reset(C* out, const C* psi, const C* psi_in, int L, int protocol, double r) {
    int64_t d = 1LL << L;
    double total = 0, cum = 0;
    int64_t outcome = 0;
    /* M[i, j] = psi[i + d j]: i the input rail (low bits), j the reservoir */
    if (protocol == 1) {
        for (int64_t i = 0; i < d; i++)
            for (int64_t j = 0; j < d; j++) total += abs2(psi[i + d * j]);
        for (int64_t i = 0; i < d; i++) {
            double row = 0;
            for (int64_t j = 0; j < d; j++) row += abs2(psi[i + d * j]);
            cum += row / total;
            if (r <= cum) { outcome = i; break; }
        }
    } else {
        for (int64_t j = 0; j < d; j++)
            for (int64_t i = 0; i < d; i++) total += abs2(psi[i + d * j]);
        for (int64_t j = 0; j < d; j++) {
            double col = 0;
            for (int64_t i = 0; i < d; i++) col += abs2(psi[i + d * j]);
            cum += col / total;
            if (r <= cum) { outcome = j; break; }
        }
    }
    C* phi = (C*)malloc(d * sizeof(C));
    double nsq = 0;
    for (int64_t y = 0; y < d; y++) {
        phi[y] = protocol == 1 ? psi[outcome + d * y] : psi[y + d * outcome];
        nsq += abs2(phi[y]);
    }
    double nrm = sqrt(nsq);
    if (nrm > 1e-12) {
        for (int64_t y = 0; y < d; y++) phi[y] /= nrm;
    } else {
        for (int64_t y = 0; y < d; y++) phi[y] = 0;
        phi[0] = 1;
    }
    /* tensor_product_ket! (cpuQuantumStatePreparation.jl:1136): psi_in on the low bits */
    for (int64_t a = 0; a < d; a++)
        for (int64_t b = 0; b < d; b++) out[a + (b << L)] = psi_in[a] * phi[b];
    free(phi);
    return (int)outcome;
}
typedef struct {
    int L, ng, n_substeps, encoding, protocol, T, n_traj, nthreads, tid;
    const so_trotter_gate* g;
    const C* psi0;
    const double* u;
    uint64_t seed, traj_offset;
    double* X_traj; /* [n_traj][T][n_ops] */
} qrc_job;
static void* qrc_worker(void* arg) {
    qrc_job* J = (qrc_job*)arg;
    int L = J->L, N = 2 * L, nops = so_qrc_n_ops(L, 2);
    int64_t dim = 1LL << N, d = 1LL << L;
    C* psi = (C*)malloc(dim * sizeof(C));
    C* nxt = (C*)malloc(dim * sizeof(C));
    C* pin = (C*)malloc(d * sizeof(C));
    double* win = (double*)malloc(L * sizeof(double));
    for (int t = J->tid; t < J->n_traj; t += J->nthreads) {
        memcpy(psi, J->psi0, dim * sizeof(C));
        uint64_t traj = J->traj_offset + (uint64_t)t;
        for (int k = 0; k < J->T; k++) {
            so_qrc_window(J->u, L, k, J->encoding, win);
            so_qrc_encode(win, L, pin);
            so_qrc_reset(nxt, psi, pin, L, J->protocol, shot_u(J->seed, (uint64_t)k, traj));
            for (int s = 0; s < J->n_substeps; s++) so_trotter_step(nxt, J->g, J->ng, N);
            memcpy(psi, nxt, dim * sizeof(C));
            so_measure_all_observables(psi, L, 2, J->X_traj + ((int64_t)t * J->T + k) * nops);
        }
    }
    free(psi); free(nxt); free(pin); free(win);
    return NULL;
}
void so_qrc_run(int L, const so_trotter_gate* g, int ng, int n_substeps, int encoding, int protocol,
                const C* psi0, const double* u, int T, int n_traj, uint64_t seed, uint64_t traj_offset,
                double* X, double* X_traj, int nthreads) {
    int nops = so_qrc_n_ops(L, 2);
    double* per = X_traj ? X_traj : (double*)malloc((size_t)n_traj * T * nops * sizeof(double));
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n_traj) nthreads = n_traj > 0 ? n_traj : 1;
    qrc_job* jobs = (qrc_job*)calloc(nthreads, sizeof(qrc_job));
    pthread_t* th = (pthread_t*)calloc(nthreads, sizeof(pthread_t));
    for (int i = 0; i < nthreads; i++) {
        qrc_job J = {L, ng, n_substeps, encoding, protocol, T, n_traj, nthreads, i, g, psi0, u, seed, traj_offset, per};
        jobs[i] = J;
    }
    for (int i = 1; i < nthreads; i++) pthread_create(&th[i], NULL, qrc_worker, &jobs[i]);
    qrc_worker(&jobs[0]);
    for (int i = 1; i < nthreads; i++) pthread_join(th[i], NULL);
    /* X_sum ./ n_traj (:587-590), summed in trajectory order */
    for (int64_t x = 0; x < (int64_t)T * nops; x++) {
        double s = 0;
        for (int t = 0; t < n_traj; t++) s += per[(int64_t)t * T * nops + x];
        X[x] = s / n_traj;
    }
    if (!X_traj) free(per);
    free(jobs); free(th);
}
/* Tr(rho P) for the Pauli string with X on xmask and Z on zmask (Y where both):
 * P|j> = i^ny (-1)^popc(j & zmask) |j ^ xmask>; rho column-major */
double so_expect_pauli_rho(const C* rho, uint64_t xmask, uint64_t zmask, int N) {
    int64_t dim = 1LL << N;
    int ny = __builtin_popcountll(xmask & zmask) & 3;
    C ph = ny == 0 ? 1 : ny == 1 ? I_ : ny == 2 ? -1 : -I_;
    C s = 0;
    for (int64_t j = 0; j < dim; j++) {
        C v = rho[j + (int64_t)(j ^ xmask) * dim];
        s += (__builtin_popcountll((uint64_t)j & zmask) & 1) ? -v : v;
    }
    return creal(ph * s);
}
void so_qrc_dm_run(int L, const so_trotter_gate* g, int ng, int n_substeps, int encoding, int protocol,
                   const C* psi0, const double* u, int T, double* X) {
    int N = 2 * L, nops = so_qrc_n_ops(L, 2);
    int64_t dim = 1LL << N, d = 1LL << L;
    C* rho = (C*)malloc(dim * dim * sizeof(C));
    C* red = (C*)malloc(d * d * sizeof(C));
    C* pin = (C*)malloc(d * sizeof(C));
    double* win = (double*)malloc(L * sizeof(double));
    for (int64_t c = 0; c < dim; c++)
        for (int64_t r = 0; r < dim; r++) rho[r + c * dim] = psi0[r] * conj(psi0[c]);
    for (int k = 0; k < T; k++) {
        so_qrc_window(u, L, k, encoding, win);
        so_qrc_encode(win, L, pin);
        /* reduced state of the kept rail (rail 1: reservoir = high bits; rail 2: input = low bits) */
        for (int64_t a = 0; a < d; a++)
            for (int64_t b = 0; b < d; b++) {
                C s = 0;
                for (int64_t x = 0; x < d; x++)
                    s += protocol == 1 ? rho[(x + d * a) + (x + d * b) * dim] : rho[(a + d * x) + (b + d * x) * dim];
                red[a + b * d] = s;
            }
        /* rho_in (x) rho_res: rho_in on the low bits, the kept state on the high bits */
        for (int64_t i = 0; i < d; i++)
            for (int64_t j = 0; j < d; j++)
                for (int64_t i2 = 0; i2 < d; i2++)
                    for (int64_t j2 = 0; j2 < d; j2++)
                        rho[(i + d * j) + (i2 + d * j2) * dim] = pin[i] * conj(pin[i2]) * red[j + j2 * d];
        for (int s = 0; s < n_substeps; s++) so_trotter_step_rho(rho, g, ng, N);
        double* o = X + (int64_t)k * nops;
        int idx = 0;
        for (int q = 0; q < N; q++) {
            uint64_t m = 1ULL << q;
            o[idx++] = so_expect_pauli_rho(rho, m, 0, N);
            o[idx++] = so_expect_pauli_rho(rho, m, m, N);
            o[idx++] = so_expect_pauli_rho(rho, 0, m, N);
        }
        for (int pass = 0; pass < 2; pass++)
            for (int rail = 0; rail < 2; rail++)
                for (int site = 0; site < L; site++) {
                    int i, j;
                    if (pass == 0) { if (site == L - 1) continue; i = rail * L + site; j = i + 1; }
                    else { if (rail == 1) continue; i = site; j = L + site; }
                    uint64_t m = (1ULL << i) | (1ULL << j);
                    o[idx++] = so_expect_pauli_rho(rho, m, 0, N);
                    o[idx++] = so_expect_pauli_rho(rho, m, m, N);
                    o[idx++] = so_expect_pauli_rho(rho, 0, m, N);
                }
    }
    free(rho); free(red); free(pin); free(win);
}

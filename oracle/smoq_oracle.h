/*
 * smoq_oracle.h -- CPU restatement of SmoQ.jl's matrix-free state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * library (libsmoq_cuda.so): only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  It is never
 * the thing measured on the GPU path and never shipped behind the C-ABI.
 *
 * Conventions follow the reference exactly:
 *   - states are complex128 (C99 double complex == Julia ComplexF64 layout),
 *     length 2^N, little-endian: qubit k (1-based) <-> bit k-1;
 *   - every gate/observable entry point takes 1-based qubits like the Julia
 *     functions it restates (the utils/cpu Julia files), and the loops keep the
 *     reference's shape (scan all 2^N indices, branch on the bit) so that the
 *     CPU baseline times the same work the reference does;
 *   - 2x2 / 4x4 matrices are passed column-major (Julia Matrix memory order)
 *     as interleaved (re, im) doubles.
 *
 * Parity pins: tests/test_oracle_golden.py checks this restatement against
 * the known-answer tests the reference's own demo suites hold
 * (scripts_variational_quantum_circuits/demo_parametrized_gates.jl, the
 * docstring examples in utils/cpu/cpuQuantumStateObservables.jl, the
 * PS-vs-FD check of demo_VQC_base_test.jl) and against an independent dense
 * kron-product restatement written in numpy.
 */
#ifndef SMOQ_ORACLE_H
#define SMOQ_ORACLE_H
#include <complex.h>
#include <stdint.h>

typedef double _Complex so_cplx;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- single-qubit gates: utils/cpu/cpuQuantumChannelGates.jl ---- */
void so_apply_rx_psi(so_cplx* psi, int k, double theta, int N);   /* :142 */
void so_apply_ry_psi(so_cplx* psi, int k, double theta, int N);   /* :172 */
void so_apply_rz_psi(so_cplx* psi, int k, double theta, int N);   /* :201 */
void so_apply_hadamard_psi(so_cplx* psi, int k, int N);           /* :222 */
void so_apply_pauli_x_psi(so_cplx* psi, int k, int N);            /* :245 */
void so_apply_pauli_y_psi(so_cplx* psi, int k, int N);            /* :265 */
void so_apply_pauli_z_psi(so_cplx* psi, int k, int N);            /* :286 */
void so_apply_s_psi(so_cplx* psi, int k, int N);                  /* :307 */
void so_apply_sdagger_psi(so_cplx* psi, int k, int N);            /* :328 */
void so_apply_t_psi(so_cplx* psi, int k, int N);                  /* :360 */
void so_apply_tdagger_psi(so_cplx* psi, int k, int N);            /* :380 */
/* ---- multi-qubit gates ---- */
void so_apply_ccz_psi(so_cplx* psi, int q1, int q2, int q3, int N);     /* :448 */
void so_apply_toffoli_psi(so_cplx* psi, int c1, int c2, int t, int N);  /* :471 */
void so_apply_cnot_psi(so_cplx* psi, int control, int target, int N);   /* :870 */
void so_apply_cz_psi(so_cplx* psi, int qi, int qj, int N);              /* :889 */
void so_apply_cry_psi(so_cplx* psi, int control, int target, double theta, int N); /* :914 */
void so_apply_rxx_psi(so_cplx* psi, int qi, int qj, double theta, int N); /* :992 */
void so_apply_ryy_psi(so_cplx* psi, int qi, int qj, double theta, int N); /* :1039 */
void so_apply_rzz_psi(so_cplx* psi, int qi, int qj, double theta, int N); /* :1084 */
/* ---- jump operators ---- */
void so_apply_sigma_minus_psi(so_cplx* psi, int k, int N);   /* :739 */
void so_apply_sigma_plus_psi(so_cplx* psi, int k, int N);    /* :762 */
double so_population_excited_psi(const so_cplx* psi, int k, int N); /* :784 */

/* ---- generic bitwise gates ---- */
/* utils/cpu/cpuQuantumChannelUnitaryEvolutionTrotter.jl:77 */
void so_apply_one_qubit_gate(so_cplx* psi, const double* U, int qubit, int N);
/* utils/cpu/cpuQuantumChannelUnitaryEvolutionTrotter.jl:107 (q1/q2 swapped
 * without permuting U when q1 > q2) */
void so_apply_two_qubit_gate(so_cplx* psi, const double* U, int q1, int q2, int N);
/* utils/cpu/cpuQuantumChannelRandomUnitaries.jl:317 (U conjugated by SWAP
 * when q1 > q2) */
void so_apply_2qubit_gate_ru(so_cplx* psi, const double* U, int q1, int q2, int N);

/* ---- observables: utils/cpu/cpuQuantumStateObservables.jl ---- */
double so_expect_z(const so_cplx* psi, int k, int N);   /* :201 */
double so_expect_x(const so_cplx* psi, int k, int N);   /* :230 */
double so_expect_y(const so_cplx* psi, int k, int N);   /* :256 */
double so_expect_zz(const so_cplx* psi, int i, int j, int N); /* :341 */
double so_expect_xx(const so_cplx* psi, int i, int j, int N); /* :385 */
double so_expect_yy(const so_cplx* psi, int i, int j, int N); /* :427 */
/* Pauli string <P>, ops[i] in {'X','Y','Z'} on 1-based qubits[i].  Z-only
 * strings follow _expect_pauli_Z_string (:900).  Mixed strings sum the full
 * Hermitian pair (bra,ket)+(ket,bra); see the Q1 note in the .c file. */
double so_expect_pauli_string(const so_cplx* psi, int n, const char* ops,
                              const int* qubits, int N);
double so_norm2(const so_cplx* psi, int N);

/* ---- Trotter: utils/cpu/cpuQuantumChannelUnitaryEvolutionTrotter.jl ---- */
typedef struct {
    int32_t nq;       /* 1 or 2 */
    int32_t q[2];     /* 1-based qubits (FastTrotterGate.indices) */
    int32_t pad;
    double U[32];     /* column-major interleaved complex; 2x2 uses U[0..7] */
} so_trotter_gate;
/* closed-form restatement of precompute_trotter_gates_bitwise_cpu (:322):
 * bonds (i, j, Jxx, Jyy, Jzz) then fields (idx, hx, hy, hz); gates with
 * |h| <= 1e-14 are dropped as in :346.  Returns the number of gates. */
int so_precompute_trotter_gates(const double* bonds, int nb, const double* fields,
                                int nf, double dt, so_trotter_gate* out);
/* apply_fast_trotter_step_cpu! (:150) */
void so_trotter_step(so_cplx* psi, const so_trotter_gate* g, int n, int N);

/* ---- circuits: utils/cpu/cpuVariationalQuantumCircuitExecutor.jl ---- */
typedef struct {
    int32_t type;     /* SO_G_* */
    int32_t q[3];     /* 1-based */
    int32_t param;    /* 0 = fixed angle, >0 = theta[param-1] (CircuitOperation.param_idx) */
    int32_t pad;
    double angle;
} so_op;
enum { SO_G_RX = 0, SO_G_RY, SO_G_RZ, SO_G_H, SO_G_X, SO_G_Y, SO_G_Z, SO_G_S,
       SO_G_SDG, SO_G_T, SO_G_TDG, SO_G_CZ, SO_G_CNOT, SO_G_RXX, SO_G_RYY,
       SO_G_RZZ, SO_G_CRY, SO_G_CCZ, SO_G_TOFFOLI };
/* apply_circuit! (:95) -> apply_gate_psi! (:146) */
void so_apply_circuit(so_cplx* psi, const so_op* ops, int n, const double* theta, int N);

/* Pauli-sum observable: term t has coefficient coef[t] and, for each 1-based
 * qubit, a letter in paulis[t*N + q-1] ('I','X','Y','Z'). */
double so_pauli_sum_expect(const so_cplx* psi, int nterms, const double* coef,
                           const char* paulis, int N);
/* E(theta) = <0|U(theta)^dag H U(theta)|0> (the VQE cost closures of
 * scripts_variational_quantum_circuits/demo_vqe_dm_vs_mcwf.jl:189-202) */
double so_energy(const so_op* ops, int n, const double* theta, int N, int nterms,
                 const double* coef, const char* paulis);
/* calculate_gradients_parameter_shift (cpuVariationalQuantumCircuitGradients.jl:138) */
void so_grad_parameter_shift(const so_op* ops, int n, const double* theta, int P, int N,
                             int nterms, const double* coef, const char* paulis,
                             double shift, const int* which, int nwhich, double* grad);
/* calculate_gradients_finite_difference (:250) */
void so_grad_finite_difference(const so_op* ops, int n, const double* theta, int P, int N,
                               int nterms, const double* coef, const char* paulis,
                               double eps, const int* which, int nwhich, double* grad);

/* ---- H|psi> of the Chebyshev / Lanczos integrators ---- */
/* apply_hamiltonian_bitwise! (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55): bond rows
 * (i, j, Jxx, Jyy, Jzz), field rows (idx, hx, hy, hz), 1-based sites; the Y field as
 * construct_sparse_hamiltonian (cpuHamiltonianBuilder.jl:297), see the .c file */
void so_apply_hamiltonian_bitwise(so_cplx* out, const so_cplx* in, const double* x_bonds, int nx,
                                  const double* y_bonds, int ny, const double* fields, int nf, int N);
/* apply_H_xxz! (cpuQuantumStateLanczos.jl:157) */
void so_apply_H_xxz(const so_cplx* psi, so_cplx* out, int N, double Jx, double Jy, double Jz, double h);

/* ---- counter-based RNG (Philox4x32-10, Salmon et al., SC'11) ---- */
void so_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double so_u01_from_words(uint32_t hi, uint32_t lo);

/* ---- MCWF (batched trajectories) ----
 * jump op types: 0 = sigma_minus, 1 = sigma_plus, 2 = sigma_z, 3 = sigma_x
 * (JumpOperator, utils/cpu/cpuQuantumChannelLindbladianEvolution.jl:65). */
typedef struct { int32_t type; int32_t qubit; double gamma; } so_jump_op;
/* One first-order quantum-jump step on one trajectory (see the .c file for
 * the exact rule and the reference lines each part follows).  Returns the
 * index of the jump channel taken, or -1. */
int so_mcwf_step(so_cplx* psi, int N, const so_trotter_gate* g, int ng,
                 const so_jump_op* ops, int nops, double dt, uint64_t seed,
                 uint64_t traj, uint64_t step);
/* Runs trajectories [t0, t0+ntraj) of a batch from |init_index>, recording
 * per-trajectory <Z_i> and <Z_i Z_{i+1}> every record_every steps
 * (z_out[(r*ntraj + t)*N + i], zz_out[(r*ntraj + t)*(N-1) + i]).  OpenMP over
 * pthreads over trajectories when nthreads > 1 (mirrors Threads.@threads). */
void so_mcwf_run(int N, const so_trotter_gate* g, int ng, const so_jump_op* ops, int nops,
                 double dt, uint64_t seed, uint64_t t0, int ntraj, int steps,
                 int record_every, uint64_t init_index, double* z_out, double* zz_out,
                 int* njumps, int nthreads);

/* ---- density-matrix oracle (N <= 10) ----
 * rho is column-major dim x dim complex128. */
void so_trotter_step_rho(so_cplx* rho, const so_trotter_gate* g, int n, int N); /* evolve_trotter_rho_cpu! :266 */
void so_dissipator_dm(so_cplx* rho, const so_jump_op* op, double dt, int N);    /* _apply_dissipator_dm! :377 */
double so_expect_z_rho(const so_cplx* rho, int k, int N);
double so_expect_zz_rho(const so_cplx* rho, int i, int j, int N);

/* timing helper for the CPU baseline */
double so_wtime(void);
/* threads over the amplitudes of one state in the generic 2x2/4x4, Rx/Ry/Rz,
 * CZ/Rzz and Z-string/Pauli-string loops (default 1 = the reference's
 * single-threaded loops; the parity tests at the measured sizes raise it).
 * States are unchanged by the split; FP64 observable sums change only their
 * summation order. */
void so_set_threads(int n);
int so_get_threads(void);
/* threads over the amplitudes of one state in the gate and observable loops
 * (default 1 = the reference's single-threaded loops; the parity tests at the
 * measured sizes raise it); results are unchanged up to the summation order of
 * the FP64 observable sums */
void so_set_threads(int n);
int so_get_threads(void);

/* ---- Born sampling / projective Z measurement: utils/cpu/cpuQuantumStateMeasurements.jl ---- */
/* u from Philox4x32-10, counter (shot, stream), key seed (the CUDA library's draws) */
void so_sample(const so_cplx* psi, int N, int64_t nshots, uint64_t seed, uint64_t stream, int64_t* out); /* :203 */
int64_t so_measure_all(so_cplx* psi, int N, uint64_t seed, uint64_t stream);                             /* :484 */
int so_measure_qubit(so_cplx* psi, int k, int N, uint64_t seed, uint64_t stream);                         /* :224 */
int so_measure_z_u(so_cplx* psi, int k, int N, double u);       /* :224 with rand() = u */

/* ---- noise unravelings (utils/cpu/cpuQuantumChannelKrausOperators.jl), reset and the
 * pure-state circuit executor with them (cpuVariationalQuantumCircuitExecutor.jl:95-201).
 * u is the uniform the reference draws with rand(). */
enum { SO_N_DEPOLARIZING = 32, SO_N_AMPLITUDE_DAMPING, SO_N_DEPHASING, SO_N_BIT_FLIP, SO_N_PHASE_FLIP,
       SO_N_PHASE_DAMPING, SO_N_THERMAL_RELAXATION,
       SO_M_MEASURE_Z = 48, SO_M_MEASURE_X, SO_M_MEASURE_Y, SO_R_RESET, SO_T_TRACE_OUT, SO_L_LINDBLAD_STEP };
void so_noise_dephasing_u(so_cplx* psi, double p, int k, int N, double u);        /* :262 */
void so_noise_depolarizing_u(so_cplx* psi, double p, int k, int N, double u);     /* :285 */
void so_noise_bit_flip_u(so_cplx* psi, double p, int k, int N, double u);         /* :321 */
void so_noise_phase_flip_u(so_cplx* psi, double p, int k, int N, double u);       /* :337 */
/* :350, with the sigma- jump (psi_0 = psi_1), not the `+=` of :367 */
void so_noise_amplitude_damping_u(so_cplx* psi, double gamma, int k, int N, double u);
/* reset_state! (cpuQuantumStateMeasurements.jl:555): target 0 :zero, 1 :one, 2 :plus, 3 :minus */
void so_reset_u(so_cplx* psi, int k, int target, int N, double u);
/* the uniform of stochastic op `op_index` of trajectory `traj`: Philox4x32-10,
 * key seed, counter (op_index, 0x80000000, traj) */
double so_circuit_draw(uint64_t seed, uint32_t op_index, uint64_t traj);
/* apply_circuit! for one trajectory: ops with 1-based qubits, gates as in
 * so_apply_circuit and the SO_N_/SO_M_/SO_R_/... types above; per op: pad =
 * if_outcome, angle = p (gamma), q[1] = the reset target.  outcomes receives the
 * measurement results in order; returns their number. */
int so_apply_circuit_mcwf(so_cplx* psi, const so_op* ops, int n, const double* theta, int N, uint64_t seed,
                          uint64_t traj, int* outcomes);

/* ---- quantum reservoir computing, bitwise MCWF path ----
 * utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:451 (_run_traj_loop_bitwise!),
 * :531 (run_mcwf_simulation, bitwise), utils/cpu/cpuQRCstep.jl:96
 * (encode_input_ry_psi!), :332 (qrc_reset_psi!).  Two rails of L qubits (N = 2L,
 * the reset reshapes the state as 2^L x 2^L).  encoding: 0 :batch, 1 :broadcast;
 * protocol: 1 :traceout_rail_1, 2 :traceout_rail_2.  The reset's rand() is the
 * Philox draw u(seed, counter (step, trajectory)).  u is padded_u (T + L values,
 * [zeros(L); inputs] as run_mcwf_simulation builds it).  X[k * n_ops + o] =
 * trajectory mean of feature o after input k; X_traj (or NULL) per trajectory. */
int so_qrc_n_ops(int L, int n_rails);
void so_measure_all_observables(const so_cplx* psi, int L, int n_rails, double* out); /* :1483 */
void so_qrc_window(const double* padded_u, int L, int k, int encoding, double* win);
void so_qrc_encode(const double* win, int L, so_cplx* psi_in);
int so_qrc_reset(so_cplx* out, const so_cplx* psi, const so_cplx* psi_in, int L, int protocol, double r);
void so_qrc_run(int L, const so_trotter_gate* g, int ng, int n_substeps, int encoding, int protocol,
                const so_cplx* psi0, const double* u, int T, int n_traj, uint64_t seed, uint64_t traj_offset,
                double* X, double* X_traj, int nthreads);
/* the density-matrix pipeline the trajectory mean converges to: run_dm_simulation
 * (utils/cpu/cpuQRCSimulationDensityMatrix.jl:114, loop :186-244): the same window
 * and encoding, qrc_reset_rho (cpuQRCstep.jl:457: partial trace, then
 * rho_in (x) rho_res), U on columns and conj(U) on rows per Trotter step */
void so_qrc_dm_run(int L, const so_trotter_gate* g, int ng, int n_substeps, int encoding, int protocol,
                   const so_cplx* psi0, const double* u, int T, double* X);
double so_expect_pauli_rho(const so_cplx* rho, uint64_t xmask, uint64_t zmask, int N);

#ifdef __cplusplus
}
#endif
#endif

/*
 * smoq_cuda.h -- C ABI of libsmoq_cuda.so, the B200 (sm_100a) state-vector
 * engine behind SmoQ.jl's matrix-free gate / observable / evolution API.
 *
 * Every entry point below replaces one reference function (cited as
 * file:line inside the SmoQ.jl tree).  Conventions:
 *   - qubits are 0-based bit positions (the Julia wrapper passes k-1 for the
 *     reference's 1-based k; bit k-1 of the index is qubit k, little-endian,
 *     utils/cpu/cpuQuantumChannelGates.jl:48-51);
 *   - a state holds `batch` independent states of 2^N amplitudes, state-major,
 *     interleaved complex (ComplexF32 for SMOQ_C64, ComplexF64 for
 *     SMOQ_C128); every gate acts on all states of the batch;
 *   - matrices are column-major interleaved complex doubles (Julia Matrix
 *     memory order); gate coefficients are always computed in FP64 on the
 *     host, expectation values and norms are accumulated in FP64;
 *   - every call returns smoq_status and never aborts, exits or traps;
 *     smoq_last_error() gives the message.  Calls are asynchronous on the
 *     context's stream; calls that return host values synchronise it.  A
 *     context is not re-entrant: use one per host thread.
 */
#ifndef SMOQ_CUDA_H
#define SMOQ_CUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SMOQ_OK = 0,
    SMOQ_ERR_BADINPUT = 1,    /* replaces error()/@assert in the reference, e.g.
                                 utils/cpu/cpuQuantumStateObservables.jl:183 */
    SMOQ_ERR_OOM = 2,
    SMOQ_ERR_CUDA = 3,
    SMOQ_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
    SMOQ_ERR_UNSUPPORTED = 5,
    SMOQ_ERR_NOGPU = 6
} smoq_status;

typedef enum { SMOQ_C64 = 0, SMOQ_C128 = 1 } smoq_dtype;

typedef struct smoq_ctx smoq_ctx;
typedef struct smoq_state smoq_state;
typedef struct smoq_plan smoq_plan;

/* ---------------------------------------------------------------- context */
smoq_status smoq_ctx_create(int device, smoq_ctx** out);
/* States and plans refer to their context: destroy them before the context. */
smoq_status smoq_ctx_destroy(smoq_ctx* ctx);
const char* smoq_last_error(smoq_ctx* ctx);
smoq_status smoq_ctx_synchronize(smoq_ctx* ctx);
/* the cudaStream_t every call of this context is ordered on */
void* smoq_ctx_stream(smoq_ctx* ctx);
enum {
    SMOQ_OPT_TILE_BITS_C64 = 1,   /* tile width (qubits) of fused passes, complex64 */
    SMOQ_OPT_TILE_BITS_C128 = 2,
    SMOQ_OPT_LOW_BITS_C64 = 3,    /* minimum contiguous low qubits per tile segment */
    SMOQ_OPT_LOW_BITS_C128 = 4,
    SMOQ_OPT_USE_GRAPHS = 5,      /* capture Trotter blocks as CUDA graphs (default 1) */
    SMOQ_OPT_KERNEL_TIMING = 6,   /* bracket fused passes with CUDA events (default 0) */
    SMOQ_OPT_ENGINE = 7           /* fused-pass engine: -1 auto (default), 0 shared-memory sweeps,
                                     2 stage sweeps (4-bit register stages, tile widths 12-13),
                                     3 compiled pass kernels (engine 2's schedule, each complex64 pass
                                     compiled with NVRTC at upload; needs libnvrtc).  Auto: reusable
                                     complex64 programs (Trotter plans, MCWF) run engine 3 when NVRTC
                                     loads, everything else engine 0.  The complex64 backward passes of
                                     smoq_energy_grad run compiled adjoint kernels under auto and 3,
                                     the shared-memory adjoint kernel under 0 and 2 */,
    SMOQ_OPT_JIT_BUFFERS = 8,     /* compiled pass kernels: tile buffers per CTA, 1 (default) or 2 (the next
                                     tile's bulk load runs under the current tile's stages) */
    SMOQ_OPT_JIT_GROUPS = 10,     /* compiled pass kernels: 16-amplitude register groups per thread, 2
                                     (default; 2^(T-5) threads) or 1 (2^(T-4) threads) */
    SMOQ_OPT_VQE_RESIDENT = 12,   /* smoq_energy_grad_jobs: 1 (default) = circuits of N <= 13 (complex64)
                                     or N <= 12 (complex128) run together in one launch, each in one
                                     CTA's shared memory; 0 = every circuit through the tiled passes */
    SMOQ_OPT_AUTOTUNE = 13,       /* No counterpart in the reference.  1 (default) = when a reusable
                                     complex64 program (a Trotter plan) of N >= 20 is first run on the
                                     compiled pass kernels, (a) time its block with each candidate
                                     geometry -- tile width, low bits, fusion depth -- on a scratch
                                     state and keep the fastest for the plan, then (b) time each
                                     compiled pass kernel's variants (register groups per thread, CTAs
                                     per SM, one or two tile buffers; bit-identical results) and keep
                                     the fastest; choices are cached per (GPU, program), across
                                     processes in the file SMOQ_TUNE_CACHE names if set; 2 = (b) only,
                                     with the geometry the options set; 0 = the options' settings */
    SMOQ_OPT_FUSION_DEPTH = 14    /* No counterpart in the reference.  Max fused ops per pass: a longer
                                     pass is split into consecutive passes of the same tile (0 =
                                     default, as many as fit); applies to gate sequences, plans and
                                     the forward and backward passes of smoq_energy_grad */
};
smoq_status smoq_ctx_set_option(smoq_ctx* ctx, int option, long long value);
/* launches: kernels launched by this context; tile_passes/tile_ms/tile_bytes:
 * fused passes, their summed event time and algorithmic bytes (timing on) */
smoq_status smoq_ctx_counters(smoq_ctx* ctx, long long* launches, long long* tile_passes,
                              double* tile_ms, double* tile_bytes);
smoq_status smoq_ctx_reset_counters(smoq_ctx* ctx);
/* No counterpart in the reference: the autotuner's per-pass timings (ms per
 * launch of each variant) and choices so far, as text */
smoq_status smoq_ctx_tune_report(smoq_ctx* ctx, char* buf, int len);
/* the library's build identification, e.g. "smoq_cuda sm_100a" */
const char* smoq_version(void);
/* 1 when the plan compiler (engine 3) can run: NVRTC could be loaded */
int smoq_jit_available(void);

/* ----------------------------------------------------------------- states */
/* Vector{ComplexF64}(undef, 2^N) per state; zero-initialised */
smoq_status smoq_state_create(smoq_ctx* ctx, int N, smoq_dtype dtype, int batch, smoq_state** out);
/* borrow a device buffer (e.g. a CuArray's pointer, 16-byte aligned); never freed here */
smoq_status smoq_state_wrap(smoq_ctx* ctx, void* devptr, int N, smoq_dtype dtype, int batch,
                            smoq_state** out);
smoq_status smoq_state_destroy(smoq_state* st);
void* smoq_state_device_ptr(smoq_state* st);
/* host <-> device copies of the whole batch in the state's own dtype */
smoq_status smoq_state_upload(smoq_state* st, const void* host, size_t bytes);
smoq_status smoq_state_download(smoq_state* st, void* host, size_t bytes);
/* amplitudes [first, first + count) of the batch (state-major: state b starts at
 * b * 2^N) into host memory: a window of a state too large to copy whole,
 * like reading ψ[first+1 : first+count] of the reference's Vector{ComplexF64} */
smoq_status smoq_state_download_range(smoq_state* st, uint64_t first, uint64_t count, void* host);
/* make_initial_psi (utils/cpu/cpuQuantumStatePreparation.jl:1211): every
 * state of the batch becomes the basis state |index> */
smoq_status smoq_state_set_basis(smoq_state* st, uint64_t index);
/* dst <- src with dtype conversion (c128 <-> c64), same N and batch */
smoq_status smoq_state_copy(smoq_state* dst, smoq_state* src);

/* ---------------------------------------------- gates: utils/cpu/cpuQuantumChannelGates.jl */
smoq_status smoq_apply_rx(smoq_state* st, int q, double theta);   /* apply_rx_psi! :142 */
smoq_status smoq_apply_ry(smoq_state* st, int q, double theta);   /* apply_ry_psi! :172 */
smoq_status smoq_apply_rz(smoq_state* st, int q, double theta);   /* apply_rz_psi! :201 */
smoq_status smoq_apply_h(smoq_state* st, int q);                  /* apply_hadamard_psi! :222 */
smoq_status smoq_apply_x(smoq_state* st, int q);                  /* apply_pauli_x_psi! :245 */
smoq_status smoq_apply_y(smoq_state* st, int q);                  /* apply_pauli_y_psi! :265 */
smoq_status smoq_apply_z(smoq_state* st, int q);                  /* apply_pauli_z_psi! :286;
                                                                     apply_sigma_z! MCWF.jl:170 */
smoq_status smoq_apply_s(smoq_state* st, int q);                  /* apply_s_psi! :307 */
smoq_status smoq_apply_sdg(smoq_state* st, int q);                /* apply_sdagger_psi! :328 */
smoq_status smoq_apply_t(smoq_state* st, int q);                  /* apply_t_psi! :360 */
smoq_status smoq_apply_tdg(smoq_state* st, int q);                /* apply_tdagger_psi! :380 */
smoq_status smoq_apply_ccz(smoq_state* st, int q1, int q2, int q3);      /* apply_ccz_psi! :448 */
smoq_status smoq_apply_toffoli(smoq_state* st, int c1, int c2, int t);   /* apply_toffoli_psi! :471 */
smoq_status smoq_apply_cnot(smoq_state* st, int control, int target);    /* apply_cnot_psi! :870 */
smoq_status smoq_apply_cz(smoq_state* st, int q1, int q2);               /* apply_cz_psi! :889 */
smoq_status smoq_apply_cry(smoq_state* st, int control, int target, double theta); /* apply_cry_psi! :914 */
smoq_status smoq_apply_rxx(smoq_state* st, int q1, int q2, double theta);  /* apply_rxx_psi! :992 */
smoq_status smoq_apply_ryy(smoq_state* st, int q1, int q2, double theta);  /* apply_ryy_psi! :1039 */
smoq_status smoq_apply_rzz(smoq_state* st, int q1, int q2, double theta);  /* apply_rzz_psi! :1084 */
smoq_status smoq_apply_sigma_minus(smoq_state* st, int q);       /* apply_sigma_minus_psi! :739 */
smoq_status smoq_apply_sigma_plus(smoq_state* st, int q);        /* apply_sigma_plus_psi! :762 */
/* generic 2x2: apply_one_qubit_gate_bitwise_cpu! (cpuQuantumChannelUnitaryEvolutionTrotter.jl:77),
 * apply_gate! (cpuQuantumChannelRandomUnitaries.jl:230) */
smoq_status smoq_apply_u1(smoq_state* st, int q, const double* U);
/* generic 4x4 on (q1, q2), basis |00>,|q_lo=1>,|q_hi=1>,|11>.
 * convention 0: apply_two_qubit_gate_bitwise_cpu! (Trotter.jl:107) -- when
 *   q1 > q2 the qubits are swapped and U is used as given;
 * convention 1: apply_2qubit_gate! (RandomUnitaries.jl:317) -- when q1 > q2
 *   U is conjugated by SWAP first. */
smoq_status smoq_apply_u2(smoq_state* st, int q1, int q2, const double* U, int convention);

/* ----------------------------------------------------- fused gate sequences */
/* gate types of smoq_op (the CircuitOperation symbols of
 * utils/cpu/cpuVariationalQuantumCircuitBuilder.jl:82 GATE_TYPES, plus the
 * generic matrices) */
enum {
    SMOQ_G_RX = 0, SMOQ_G_RY, SMOQ_G_RZ, SMOQ_G_H, SMOQ_G_X, SMOQ_G_Y, SMOQ_G_Z, SMOQ_G_S,
    SMOQ_G_SDG, SMOQ_G_T, SMOQ_G_TDG, SMOQ_G_CZ, SMOQ_G_CNOT, SMOQ_G_RXX, SMOQ_G_RYY,
    SMOQ_G_RZZ, SMOQ_G_CRY, SMOQ_G_CCZ, SMOQ_G_TOFFOLI, SMOQ_G_U1, SMOQ_G_U2
};
/* operations beyond the gates, for smoq_apply_circuit_mcwf (the NOISE, MEASURE,
 * RESET, TRACE and analog types of GATE_TYPES' neighbours,
 * cpuVariationalQuantumCircuitBuilder.jl:82-94).  Each acts on q[0] alone: the
 * reference's noise/measure/reset ops on several qubits loop over them in order
 * (apply_channel_*!, cpuQuantumChannelKrausOperators.jl:426-556;
 * projective_measurement!, cpuQuantumStateMeasurements.jl:319; reset_state!,
 * :555), so a caller lists one op per qubit in that order. */
enum {
    SMOQ_N_DEPOLARIZING = 32,     /* angle = p: X, Y, Z with p/3 each (_apply_depolarizing_single! :285) */
    SMOQ_N_AMPLITUDE_DAMPING,     /* angle = gamma (_apply_amplitude_damping_single! :350) */
    SMOQ_N_DEPHASING,             /* angle = p: Z with (1 - sqrt(1 - p)) / 2 (_apply_dephasing_single! :262) */
    SMOQ_N_BIT_FLIP,              /* angle = p: X with p (_apply_bit_flip_single! :321) */
    SMOQ_N_PHASE_FLIP,            /* angle = p: Z with p (_apply_phase_flip_single! :337) */
    SMOQ_N_PHASE_DAMPING,         /* as SMOQ_N_DEPHASING (apply_noise_mcwf!, Executor.jl:199) */
    SMOQ_N_THERMAL_RELAXATION,    /* no effect on a pure state (apply_noise_mcwf! has no branch for it) */
    SMOQ_M_MEASURE_Z = 48,        /* projective measurement, outcome recorded (_measure_z_single! :224) */
    SMOQ_M_MEASURE_X,             /* H, measure Z, H (projective_measurement! :319) */
    SMOQ_M_MEASURE_Y,             /* S^dag, H, measure Z, H, S */
    SMOQ_R_RESET,                 /* measure Z, then force q[0] to q[1] = 0 :zero, 1 :one, 2 :plus,
                                     3 :minus (reset_state! :555, _force_qubit_state! :584) */
    SMOQ_T_TRACE_OUT,             /* no effect on a pure state (apply_trace_out_psi!, Executor.jl:231) */
    SMOQ_L_LINDBLAD_STEP          /* no effect (apply_lindblad_mcwf!, Executor.jl:242, a stub) */
};
typedef struct {
    int32_t type;     /* SMOQ_G_*, or (smoq_apply_circuit_mcwf only) SMOQ_N_* / SMOQ_M_* / SMOQ_R_* / ... */
    int32_t q[3];     /* 0-based qubits */
    int32_t param;    /* -1: fixed `angle`; >= 0: theta[param] (CircuitOperation.param_idx - 1) */
    int32_t if_outcome; /* CircuitOperation.if_outcome: 0 always; k > 0 only where the trajectory's
                         measurement k (1-based, in execution order) gave 1 (smoq_apply_circuit_mcwf
                         only; the gate-only calls require 0) */
    double angle;
    double U[32];     /* SMOQ_G_U1 / SMOQ_G_U2 (convention 0), column-major interleaved */
} smoq_op;
/* apply_circuit! (cpuVariationalQuantumCircuitExecutor.jl:95) for gate-only
 * circuits: the sequence is planned into fused tile passes (gates on a
 * tile's qubits are applied in shared memory between one HBM read and one
 * HBM write of the tile).  theta may be NULL when no op has param >= 0. */
smoq_status smoq_apply_sequence(smoq_state* st, const smoq_op* ops, int n, const double* theta);
/* the same, one launch per gate (the plain, unfused path) */
smoq_status smoq_apply_sequence_unfused(smoq_state* st, const smoq_op* ops, int n,
                                        const double* theta);
/* apply_circuit! (cpuVariationalQuantumCircuitExecutor.jl:95) on pure states for
 * any circuit: gates, noise channels unravelled stochastically (apply_noise_mcwf!,
 * :187), projective measurements (apply_measure_psi!, :210), resets
 * (apply_reset_psi!, :220) and classical conditions (if_outcome, :103-105).
 * Every state of st is one trajectory.  Stochastic op i of trajectory b draws
 * u = the 53-bit uniform of Philox4x32-10 with key = seed and counter
 * (i, 0x80000000, traj_offset + b) (i = the op's index in `ops`), and uses it
 * where the reference calls rand().  Runs of gates between stochastic ops are
 * fused into tile passes as in smoq_apply_sequence; a Pauli noise op costs one
 * pass over the trajectories that drew a Pauli; amplitude damping, measurement
 * and reset cost one FP64 reduction and one pass.  Amplitude damping jumps with
 * sigma- (the |1> amplitude REPLACES the |0> one): the reference's
 * `psi[i_ground] += psi[i]` (cpuQuantumChannelKrausOperators.jl:367) is not
 * followed, since only the replacing jump unravels the reference's own Kraus
 * channel (:145-180).  A measurement with if_outcome != 0 is UNSUPPORTED (the
 * reference's measure() cannot build one).  outcomes (host, may be NULL):
 * batch * n_meas values, outcomes[b * n_meas + m] = result of measurement m of
 * trajectory b, n_meas = the number of SMOQ_M_* ops in `ops`. */
smoq_status smoq_apply_circuit_mcwf(smoq_state* st, const smoq_op* ops, int n, const double* theta,
                                    uint64_t seed, uint64_t traj_offset, int32_t* outcomes);

/* ----------------------------------- observables: utils/cpu/cpuQuantumStateObservables.jl */
/* each writes `batch` doubles to the host array out (one per state) */
smoq_status smoq_expect_x(smoq_state* st, int q, double* out);   /* expect_local :175 -> _expect_X :230 */
smoq_status smoq_expect_y(smoq_state* st, int q, double* out);   /* _expect_Y :256 */
smoq_status smoq_expect_z(smoq_state* st, int q, double* out);   /* _expect_Z :201 */
smoq_status smoq_expect_xx(smoq_state* st, int q1, int q2, double* out); /* expect_corr :306 -> :385 */
smoq_status smoq_expect_yy(smoq_state* st, int q1, int q2, double* out); /* _expect_YY :427 */
smoq_status smoq_expect_zz(smoq_state* st, int q1, int q2, double* out); /* _expect_ZZ :341 */
/* get_expectation_pauli_string :840 (ops letters 'X','Y','Z' on 0-based qubits) */
smoq_status smoq_expect_pauli_string(smoq_state* st, int n, const char* ops, const int* qubits,
                                     double* out);
/* measure_all_observables_state_vector_cpu! (cpuQuantumStateObservables.jl:1483) for
 * the multi-rail ladder of N = L * n_rails qubits: out[b * n_ops + k] in the
 * reference's order -- (<X_q>, <Y_q>, <Z_q>) for every qubit, then (<XX>, <YY>, <ZZ>)
 * for every bond along each rail, then for every rung between rails;
 * n_ops = 3N + 3 (L-1) n_rails + 3 L (n_rails-1).  Z and ZZ share Z-string passes. */
smoq_status smoq_measure_all_observables(smoq_state* st, int L, int n_rails, double* out);
/* diagonal batch in ONE pass: out[b * nobs + o] = <Z-string zmasks[o]> of state b
 * (zmask 0 gives the squared norm); the Z/ZZ part of
 * measure_all_observables_one_pass :1532 */
smoq_status smoq_expect_zstrings(smoq_state* st, const uint64_t* zmasks, int nobs, double* out);
/* No counterpart in the reference.  The same diagonal batch as
 * smoq_expect_zstrings for callers that cannot allocate device memory at
 * call time (fixed-footprint hosts, callers that already hold most of HBM,
 * code that must not wait on the allocator, callers without a smoq_ctx):
 * it allocates nothing.  psi points to batch * 2^N caller-owned device
 * amplitudes (16-byte aligned), out to batch * nobs caller-owned device
 * doubles (out[b * nobs + o]); kernels run on `stream` (a cudaStream_t,
 * NULL = default stream) and the call returns without synchronising.  Limits:
 * nobs <= 32, batch <= 65535 and batch * nobs <= 65536 (the fixed scratch of
 * 512 KiB per GPU); larger requests return SMOQ_ERR_BADINPUT with a message
 * in errbuf (may be NULL).  The first call on each device looks up the
 * scratch array's device address (make it before any stream capture), and
 * the first call after the device's CUDA context changed (cudaDeviceReset)
 * looks it up again; calls that can overlap on one device race on the shared
 * scratch. */
smoq_status smoq_expect_zstrings_noalloc(const void* psi, int N, smoq_dtype dtype, int batch,
                                         const uint64_t* zmasks, int nobs, double* out, void* stream,
                                         char* errbuf, size_t errlen);
/* population_excited_psi (Gates.jl:784) */
smoq_status smoq_population_excited(smoq_state* st, int q, double* out);
/* squared norm per state; get_norm (cpuQuantumStatePreparation.jl:377) is its sqrt */
smoq_status smoq_norm2(smoq_state* st, double* out);
/* normalize_state! (cpuQuantumStatePreparation.jl:307) */
smoq_status smoq_normalize(smoq_state* st);

/* ------------------------ Hamiltonian IR and Trotter (cpuHamiltonianBuilder.jl,
 *                          cpuQuantumChannelUnitaryEvolutionTrotter.jl) */
typedef struct {           /* FastTrotterGate (Trotter.jl:62) with 0-based indices */
    int32_t nq;            /* 1 or 2 */
    int32_t q[2];
    int32_t pad;
    double U[32];          /* column-major interleaved; 2x2 gates use U[0..7] */
} smoq_trotter_gate;
/* precompute_trotter_gates_bitwise_cpu (Trotter.jl:322): bonds are
 * CouplingTerm (cpuHamiltonianBuilder.jl:42) rows (i, j, Jxx, Jyy, Jzz) and
 * fields FieldTerm (:51) rows (idx, hx, hy, hz), 0-based sites; gates are
 * exp(-i H_local dt) in closed form.  *n_out receives the gate count. */
smoq_status smoq_precompute_trotter_gates(const double* bonds, int nb, const double* fields,
                                          int nf, double dt, smoq_trotter_gate* out, int* n_out);
/* A Trotter plan: order 1 applies the gates once per step (apply_fast_trotter_step_cpu!,
 * Trotter.jl:150); order 2 applies them, then the same list reversed (Strang
 * splitting; the caller passes gates computed for dt/2). */
smoq_status smoq_trotter_plan_create(smoq_ctx* ctx, int N, smoq_dtype dtype,
                                     const smoq_trotter_gate* gates, int n, int order,
                                     smoq_plan** out);
smoq_status smoq_plan_destroy(smoq_plan* plan);
/* evolve_trotter_psi_cpu! (Trotter.jl:250): n_steps steps in place */
smoq_status smoq_trotter_step(smoq_plan* plan, smoq_state* st, int n_steps);
/* solve_trotter_bitwise_cpu (Trotter.jl:293) with <Z_i> records: runs `steps`
 * steps and records <Z_i> of every state at t = 0, record_every, ... into
 * z_out[r][b][i] (host, (steps/record_every + 1) * batch * N doubles). */
smoq_status smoq_trotter_run(smoq_plan* plan, smoq_state* st, int steps, int record_every,
                             double* z_out);

/* ------------------ MCWF (cpuQuantumChannelLindbladianEvolutionMonteCarloWaveFunction.jl) */
typedef struct {           /* JumpOperator (cpuQuantumChannelLindbladianEvolution.jl:65) */
    int32_t type;          /* 0 sigma_minus, 1 sigma_plus, 2 sigma_z, 3 sigma_x */
    int32_t qubit;         /* 0-based */
    double gamma;
} smoq_jump_op;
/* Batched quantum-jump evolution (lindblad_mcwf_batched_step! :340,
 * evolve_mcwf_batched_trotter! :412, generalised to any mix of the four jump
 * types): every state of `st` is one trajectory, starting from whatever st
 * holds (normalised).  The plan must be order 1 (the coherent step).
 * Trajectory b uses Philox4x32-10 stream (key = seed, counter = (step, traj_offset + b)).
 * Records at t = 0, record_every, ...: the trajectory means of <Z_i>
 * (z_mean[r][i]) and <Z_i Z_{i+1}> (zz_mean[r][i]); optional per-trajectory
 * values z_traj[r][b][i], zz_traj[r][b][i] (NULL to skip); jumps[b] counts the
 * jumps per trajectory (NULL to skip). */
smoq_status smoq_mcwf_run(smoq_plan* plan, smoq_state* st, const smoq_jump_op* ops, int nops,
                          double dt, uint64_t seed, uint64_t traj_offset, int steps,
                          int record_every, double* z_mean, double* zz_mean, double* z_traj,
                          double* zz_traj, int* jumps);

/* ------------------------------------------- quantum reservoir computing (QRC) */
/* The bitwise QRC trajectory loop: _run_traj_loop_bitwise! and the bitwise
 * run_mcwf_simulation (utils/cpu/cpuQRCSimulationMonteCarloWaveFunction.jl:451,
 * :531) with encode_input_ry_psi! and qrc_reset_psi! (utils/cpu/cpuQRCstep.jl:96,
 * :332).  Two rails of L qubits (N = 2L; the reset reshapes the state as
 * 2^L x 2^L).  Per input k: encode the window of inputs as Ry(pi u) rotations of
 * the input rail (low L qubits), measure one rail by inverse-CDF sampling, keep
 * the normalised state of the other rail as the new reservoir (high L qubits),
 * run n_substeps steps of the plan's Trotter step, and measure the ladder's
 * observable set (smoq_measure_all_observables order).  The draw r of
 * trajectory traj_offset + t at input k is the 53-bit Philox4x32-10 uniform of
 * smoq_sample with shot = k, stream = traj_offset + t, key = seed. */
typedef struct {
    int32_t L;             /* qubits per rail (N = 2L); <= 7 complex64, <= 6 complex128 */
    int32_t n_substeps;    /* Trotter steps per input */
    int32_t encoding;      /* 0 :batch (window u_{k-L+1..k}, zeros before the series), 1 :broadcast (u_k on every qubit) */
    int32_t reset;         /* 1 :traceout_rail_1 (measure the input rail), 2 :traceout_rail_2 (measure the reservoir) */
    uint64_t seed;
    uint64_t traj_offset;
} smoq_qrc_params;
/* plan: a Trotter plan on N = 2L qubits (one step = the FastTrotterGate list);
 * psi0: host 2^N complex128 (re, im interleaved), NULL = |0...0>; padded_u:
 * T + L values, the input series after L leading zeros ([zeros(L); u], as
 * run_mcwf_simulation builds it; values in [0, 1]); X (host, T * n_ops) receives the trajectory mean of every
 * feature after every input, n_ops = 3N + 3 (L-1) 2 + 3 L; X_traj (host,
 * n_traj * T * n_ops, or NULL) the per-trajectory features. */
smoq_status smoq_qrc_run(smoq_plan* plan, const smoq_qrc_params* p, const double* psi0, const double* padded_u,
                         int T, int64_t n_traj, double* X, double* X_traj);

/* ------------------------------------------- VQE energy and adjoint gradient */
typedef struct {           /* one Pauli-sum term: coef * prod of letters */
    double coef;
    uint64_t xmask;        /* qubits carrying X or Y */
    uint64_t zmask;        /* qubits carrying Z or Y */
} smoq_pauli_term;
/* E(theta) = <0|U^dag H U|0> and dE/dtheta for `batch` parameter sets at once
 * (theta[b * n_params + p]).  Gradient by the adjoint method (one forward
 * sweep, then an uncompute sweep in reverse); replaces the gradient backends
 * of calculate_gradients (cpuVariationalQuantumCircuitGradients.jl:88) for
 * gate-only circuits whose parameterised gates are RX/RY/RZ/RXX/RYY/RZZ.
 * energies[b], grads[b * n_params + p] are host arrays.  The energy is
 * <phi|H|phi> / <phi|phi> with both sums in FP64 over the computed state phi
 * (exactly <phi|H|phi> for a unitary circuit; for complex64 the division
 * removes the norm drift of a deep circuit), and the gradient is divided by
 * the same <phi|phi>.  complex64 backward passes of tile width 12 run as
 * compiled kernels (NVRTC; SMOQ_OPT_ENGINE auto or 3): 4-qubit register stages
 * on both states with the generator measurements in between, the gate
 * coefficients passed per launch, so the compile of a circuit's first parameter
 * set serves every later one. */
smoq_status smoq_energy_grad(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n,
                             int n_params, const smoq_pauli_term* H, int nterms, int batch,
                             const double* theta, double* energies, double* grads);
/* Energy and adjoint gradient of a NOISY circuit along fixed trajectories: the
 * ops of smoq_apply_circuit_mcwf (noise, measurements, resets, if_outcome) with
 * its draws (trajectory t = traj_offset + 0 .. n_traj-1, from |0...0>).  With
 * the draws fixed, each trajectory is a product of unitaries, drawn Paulis and
 * normalised branch maps K (amplitude damping, collapse, reset); the gradient
 * is the path-wise dE/dtheta of E = <psi_T|H|psi_T> (branches held fixed):
 * lambda runs backwards through U^dag, and through a branch map as
 * K^T (lambda - Re<psi'|lambda> psi').  A branch map cannot be uncomputed, so
 * the forward pass stores the state in front of every checkpoint_every-th
 * branch op and the backward pass restores the nearest one, replaying the
 * recorded steps; memory: ceil(branch ops / checkpoint_every) + 2 states.  The
 * reference's gradients treat noise as identity (cpuVQCEnzymeWrapper.jl:160-170,
 * behind calculate_gradients, cpuVariationalQuantumCircuitGradients.jl:88);
 * this differentiates the trajectories the noise produced, whose mean is the
 * gradient of the mean energy.  energies[t] (host) and grads[t * n_params + p]
 * (host, may be NULL); parameterised gates RX/RY/RZ/RXX/RYY/RZZ/CRY. */
smoq_status smoq_energy_grad_mcwf(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n, int n_params,
                                  const smoq_pauli_term* H, int nterms, const double* theta, uint64_t seed,
                                  uint64_t traj_offset, int n_traj, int checkpoint_every, double* energies,
                                  double* grads);
/* energy only (forward + reduction), same arguments */
smoq_status smoq_energy(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_op* ops, int n,
                        int n_params, const smoq_pauli_term* H, int nterms, int batch,
                        const double* theta, double* energies);

/* Many independent VQE circuits at once (a batch of different circuits, sizes and
 * Hamiltonians: the reference evaluates such batches one circuit at a time with
 * calculate_gradients, cpuVariationalQuantumCircuitGradients.jl:88, inside a
 * Threads.@threads loop).  Each job is one circuit with one parameter vector;
 * grad may be NULL (energy only).  Circuits whose two states fit one CTA's
 * shared memory (N <= 13 complex64, N <= 12 complex128) run together in one
 * launch, one CTA per circuit, off a device work queue (SMOQ_OPT_VQE_RESIDENT);
 * the others are taken off a host queue by up to 8 worker threads, each planning
 * a circuit and running it on a worker context of its own (own stream and error
 * word, the context's options; created on first use and kept until the context
 * is destroyed), so the small grids of several circuits share the GPU.  The
 * call returns when all jobs are done.  The first failing job's status is
 * returned, with its index in the message. */
typedef struct {
    int N;                        /* qubits of this circuit */
    const smoq_op* ops;           /* its gate list */
    int n;
    int n_params;
    const smoq_pauli_term* H;     /* its Hamiltonian */
    int nterms;
    const double* theta;          /* n_params values */
    double* energy;               /* host, 1 value */
    double* grad;                 /* host, n_params values, or NULL */
} smoq_vqe_job;
smoq_status smoq_energy_grad_jobs(smoq_ctx* ctx, smoq_dtype dtype, const smoq_vqe_job* jobs, int njobs);

/* out = H in for every state of the batch (H = sum of Pauli strings, smoq_pauli_term);
 * expect[b] = Re <in_b|H|in_b> (host, may be NULL).  The Hamiltonian apply of
 * apply_hamiltonian_bitwise! (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55) and
 * apply_H_xxz! / apply_H_ising! (cpuQuantumStateLanczos.jl:157,220), for any Pauli sum:
 * the building block of Chebyshev and Lanczos.  in and out: same shape, not aliased. */
smoq_status smoq_apply_pauli_sum(smoq_state* in, smoq_state* out, const smoq_pauli_term* H, int nterms,
                                 double* expect);
/* apply_hamiltonian_bitwise!(psi_out, psi_in, params::HamiltonianParams)
 * (cpuQuantumChannelUnitaryEvolutionChebyshev.jl:55): out = H in for the
 * HamiltonianParams (cpuHamiltonianBuilder.jl:69) given as its x_bonds and
 * y_bonds, rows (i, j, Jxx, Jyy, Jzz) of CouplingTerm (:42), and fields, rows
 * (idx, hx, hy, hz) of FieldTerm (:51), with 0-based sites; terms with a zero
 * coefficient are skipped as the reference skips them.  The Y field is the
 * Pauli Y of construct_sparse_hamiltonian (cpuHamiltonianBuilder.jl:297) and
 * apply_Y! (cpuQuantumStateLanczos.jl:84); the reference's pull loop
 * (Chebyshev.jl:142) applies its transpose, -hy Y.  in, out: same shape, not aliased. */
smoq_status smoq_apply_hamiltonian_bitwise(smoq_state* out, smoq_state* in, const double* x_bonds, int nx,
                                           const double* y_bonds, int ny, const double* fields, int nf);
/* apply_H_xxz!(psi, out, N, Jx, Jy, Jz, h) (cpuQuantumStateLanczos.jl:157): out = Jx sum X_i X_{i+1}
 * + Jy sum Y_i Y_{i+1} + Jz sum Z_i Z_{i+1} + h sum X_i on the open chain; apply_H_ising!
 * (:220) is Jx = Jy = 0 */
smoq_status smoq_apply_h_xxz(smoq_state* psi, smoq_state* out, double Jx, double Jy, double Jz, double h);

/* ------------------------------------------------------- density matrices */
/* A density matrix of N qubits (N <= 16) is a smoq_state of 2N qubits holding
 * rho column-major (rho[i, j] at i + j 2^N, the memory of Julia's
 * Matrix{ComplexF64}): bits 0..N-1 index the row, bits N..2N-1 the column;
 * |k><k| is smoq_state_set_basis(st, k + k * 2^N).
 * smoq_dm_plan_create builds a plan whose one step is the reference's DM step:
 * rho -> U rho U^dag for the gate list (evolve_trotter_rho_cpu!,
 * cpuQuantumChannelUnitaryEvolutionTrotter.jl:266-285), then, for each jump in
 * order, one Euler step rho += gamma dt (L rho L^dag - {L^dag L, rho}/2)
 * (_apply_dissipator_dm!, cpuQuantumChannelLindbladianEvolution.jl:377-460).
 * Run it with smoq_trotter_step / smoq_plan_destroy like any plan; the state
 * passed must have 2N qubits.  2-qubit gates follow the smoq_trotter_gate
 * convention on both sides (rows: U, columns: conj(U)). */
smoq_status smoq_dm_plan_create(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_trotter_gate* gates, int ngates,
                                const smoq_jump_op* jumps, int njumps, double dt, smoq_plan** out);
/* out[b * nobs + o] = sum_i Re rho_ii (-1)^popc(i & zmasks[o]) for every matrix of
 * the batch: <Z...> strings of a density matrix (cpuQuantumStateObservables.jl:1246-1420
 * restricted to Z strings; mask 0 gives the trace).  1 <= nobs <= 32; out is host. */
smoq_status smoq_dm_expect_zstrings(smoq_state* rho, int N, const uint64_t* zmasks, int nobs, double* out);

/* ------------------------------------------------- sampling and measurement */
/* Born-rule sampling from |psi|^2: out[b * nshots + s] = basis index of shot s of
 * state b.  Replaces sample_from_probabilities (cpuQuantumStateMeasurements.jl:203)
 * and the benchmark's cumsum + searchsortedfirst shot loop
 * (run_benchmark_smoq_Float64.jl:424-435).  Uniforms from Philox4x32-10 with key =
 * seed and counter = (shot, stream + b): the same seed and stream give the same
 * shots.  N >= 8.  out is a host array. */
smoq_status smoq_sample(smoq_state* st, long long nshots, unsigned long long seed, unsigned long long stream,
                        long long* out);
/* projective_measurement_all! (cpuQuantumStateMeasurements.jl:484): one shot per
 * state (shot 0 of the stream above), each state collapsed onto its outcome;
 * outcome[b] = basis index (bit k-1 = qubit k).  N >= 8. */
smoq_status smoq_measure_all(smoq_state* st, unsigned long long seed, unsigned long long stream,
                             long long* outcome);
/* _measure_z_single! (cpuQuantumStateMeasurements.jl:224): Z measurement of qubit q
 * (0-based) of every state, collapse and renormalise; outcome[b] in {0, 1}.  The
 * uniform is shot 0 of (seed, stream + b). */
smoq_status smoq_measure_qubit(smoq_state* st, int q, unsigned long long seed, unsigned long long stream,
                               int* outcome);

/* No counterpart in the reference: the failure path of the bounded device
 * waits, for tests.  Launches one block whose mbarrier wait (the wait every
 * tile kernel uses for its bulk copies) can never complete -- the barrier
 * expects bytes no copy delivers -- so the wait gives up after limit_ns
 * (1 us .. 100 ms), records the timeout and returns; nothing is left in
 * flight.  Returns SMOQ_ERR_TIMEOUT, as a tile kernel's timed-out wait would,
 * and leaves the context usable. */
smoq_status smoq_debug_wait_timeout(smoq_ctx* ctx, uint64_t limit_ns);

/* ------------------------------------------------- host-only introspection */
/* No counterpart in the reference.  Runs the fused-pass planner (host code,
 * no GPU or context needed) on a gate sequence exactly as
 * smoq_apply_sequence would with `engine` (0, 2 or 3) and reports, per pass,
 * the tile geometry and the fused ops (kind = 0 dense 2x2, 1 dense 4x4,
 * 2 parity 4x4, 3 monomial, 4 diagonal, 10 stage header of engines 2-3;
 * coefficients as the kernels read them).  Counts are written even when the
 * output arrays are too small (NULL arrays allowed). */
typedef struct {
    int32_t T, L, H, nops;
    int32_t hb[24];
} smoq_pass_info;
typedef struct {
    int32_t kind, nq;
    int32_t lb[4], gb[4];
    int32_t perm[8];       /* monomial permutation; stage header (kind 10): the stage's 4 tile bits,
                              then the lane bit rotating each */
    int32_t slot[4];       /* engines 2-3: the stage position of each qubit */
    int32_t mode;          /* unused */
    double c[32];          /* 16 interleaved complex coefficients */
} smoq_fused_op_info;
/* Host-only check of the plan compiler (engine 3): plans `ops` as smoq_apply_sequence
 * would with engine 3 and compiles every complex64 pass kernel with NVRTC, without a GPU
 * and without loading them.  flags: 1 = return the compiler's register/spill report in msg,
 * 2 = two tile buffers per CTA (SMOQ_OPT_JIT_BUFFERS 2), 4 = run-time coefficients (the form
 * the complex64 forward of smoq_energy_grad compiles: gate coefficients passed per launch),
 * 8 = one register group per thread (SMOQ_OPT_JIT_GROUPS 1), 16 = the generated source of the
 * first pass in msg (nothing compiled; with 32, the sources of every pass one after another,
 * *n_compiled = their count, and with 4 as well each source is followed by a line "//@coefs"
 * and its run-time coefficient block as hex floats, re im per entry).  *n_compiled = kernels compiled; msg gets "ok" (or the
 * report) or the first error.  SMOQ_ERR_UNSUPPORTED when NVRTC is not available. */
smoq_status smoq_debug_compile_plan(int N, smoq_dtype dtype, int tile_bits, int low_bits, const smoq_op* ops, int n,
                                    const double* theta, int flags, int* n_compiled, char* msg, int msg_len);
/* Host-only check of the compiled adjoint kernels of smoq_energy_grad (complex64):
 * builds the backward program of `ops` (measurements of the parameterised gates'
 * generators interleaved with the inverse gates), plans it into tile passes of width
 * tile_bits - 1, stage-schedules every pass the compiled adjoint kernel takes and
 * compiles those kernels with NVRTC, without a GPU and without loading them.
 * *n_passes = backward passes, *n_compiled = passes compiled for the compiled kernel
 * (the rest run on the shared-memory adjoint kernel).  flags: 1 = the compiler's
 * register/spill report in msg, 2 = the generated source of the first such pass in
 * msg (nothing compiled).  SMOQ_ERR_UNSUPPORTED when NVRTC is not available. */
smoq_status smoq_debug_compile_adjoint(int N, const smoq_op* ops, int n, int n_params, const double* theta,
                                       int tile_bits, int low_bits, int flags, int* n_passes, int* n_compiled,
                                       char* msg, int msg_len);
/* Host-only view of the autotuner's geometry rule: ms[c] = the timed run of
 * candidate c (< 0: not plannable), candidate 0 the default geometry.  Returns the
 * candidate kept: the fastest, unless the default is within 2% of it (one timed
 * run each: smaller differences are noise); -1 when none was plannable. */
int smoq_debug_pick_geometry(const float* ms, int n);
smoq_status smoq_debug_plan_sequence(int N, smoq_dtype dtype, int tile_bits, int low_bits, int engine,
                                     const smoq_op* ops, int n, const double* theta, smoq_pass_info* passes, int max_passes,
                                     smoq_fused_op_info* fused, int max_fused, int* n_passes, int* n_fused);

#ifdef __cplusplus
}
#endif
#endif

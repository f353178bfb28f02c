// circuit_common.cuh -- the per-trajectory rules of noisy circuits, shared by
// the trajectory executor (circuit.cu) and the noisy adjoint gradient
// (noisy_grad.cu), on the device and on the host:
//  * the draw of stochastic op i of trajectory t: the 53-bit uniform of
//    Philox4x32-10 with key = seed and counter (i, 0x80000000, t);
//  * the Pauli a Pauli-noise op applies for a draw u
//    (utils/cpu/cpuQuantumChannelKrausOperators.jl:262-347);
//  * the real 2x2 map of an amplitude-damping, measurement or reset op on its
//    qubit's pairs, normalisation included, from the trajectory's halves
//    s0 = sum_{bit=0} |psi|^2, s1 = sum_{bit=1} |psi|^2 and its draw u
//    (Kraus :350-386; cpuQuantumStateMeasurements.jl:224-255, :555, :584-635).
#pragma once
#include <math.h>
#include <stdint.h>
#include "../../include/smoq_cuda.h"

namespace smoq {

constexpr uint32_t kCircuitTag = 0x80000000u;  // counter word 1 of every circuit draw

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): the published rounds and
// constants.  c is the counter (in place: it becomes the four output words),
// (k0, k1) the key.
__host__ __device__ __forceinline__ void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = mulhi32(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = mulhi32(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
// 53-bit uniform in [0, 1): 27 bits of hi, 26 bits of lo
__host__ __device__ __forceinline__ double u01_53(uint32_t hi, uint32_t lo) {
    const uint64_t a = hi >> 5, b = lo >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

__host__ __device__ __forceinline__ double circuit_draw(uint64_t seed, uint32_t op_index, uint64_t traj) {
    uint32_t c[4] = {op_index, kCircuitTag, (uint32_t)traj, (uint32_t)(traj >> 32)};
    philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return u01_53(c[0], c[1]);
}

// code of the Pauli a noise op applies for the draw u: 0 I, 1 X, 2 Y, 3 Z
__host__ __device__ __forceinline__ int pauli_code(int type, double p, double u) {
    switch (type) {
        case SMOQ_N_DEPOLARIZING:  // cpuQuantumChannelKrausOperators.jl:285-318
            return u < p / 3 ? 1 : (u < 2 * p / 3 ? 2 : (u < p ? 3 : 0));
        case SMOQ_N_BIT_FLIP:      // :321-334
            return u < p ? 1 : 0;
        case SMOQ_N_PHASE_FLIP:    // :337-347
            return u < p ? 3 : 0;
        default:                   // dephasing / phase damping, :262-282: Z with q = (1 - sqrt(1 - p)) / 2
            return u < (1.0 - sqrt(1.0 - p)) / 2.0 ? 3 : 0;
    }
}

enum BranchKind : int32_t { BR_AMPDAMP = 0, BR_MEASURE = 1, BR_RESET = 2 };

// The branch of one trajectory as the real 2x2 map K on the qubit's pairs,
// (a0, a1) -> (K[0] a0 + K[1] a1, K[2] a0 + K[3] a1), the reference's
// renormalisation included; *outcome = the recorded bit (measurements) or -1.
// kind: BranchKind; target: the reset target (0 :zero, 1 :one, 2 :plus, 3 :minus).
__host__ __device__ __forceinline__ void branch_map(int kind, int target, double gamma, double s0, double s1,
                                                    double u, double K[4], int* outcome) {
    K[0] = 1, K[1] = 0, K[2] = 0, K[3] = 1;
    *outcome = -1;
    if (kind == BR_AMPDAMP) {
        // _apply_amplitude_damping_single! (cpuQuantumChannelKrausOperators.jl:350-386):
        // jump with probability gamma * pop_1 (and pop_1 > 1e-12), else damp |1> by
        // sqrt(1 - gamma); then divide by the norm when it exceeds 1e-12.  The jump is
        // sigma- (the |1> amplitude replaces the |0> one), which unravels the same
        // file's Kraus channel (:145-180); the line psi[i_ground] += psi[i] (:367) does not.
        if (u < gamma * s1 && s1 > 1e-12) {
            const double n = sqrt(s1);
            K[0] = 0, K[1] = n > 1e-12 ? 1.0 / n : 1.0, K[3] = 0;
        } else {
            const double d = sqrt(1.0 - gamma), n = sqrt(s0 + (1.0 - gamma) * s1);
            const double f = n > 1e-12 ? 1.0 / n : 1.0;
            K[0] = f, K[3] = d * f;
        }
        return;
    }
    // _measure_z_single! (cpuQuantumStateMeasurements.jl:224-255): outcome 0 iff
    // u < P(0) = s0; keep that half, divide by its norm
    const int m = u < s0 ? 0 : 1;
    const double f = 1.0 / sqrt(m ? s1 : s0);
    if (kind == BR_MEASURE) {
        *outcome = m;
        K[0] = m ? 0.0 : f;
        K[3] = m ? f : 0.0;
        return;
    }
    // reset_state! (:555): the measurement, then _force_qubit_state! (:584-627):
    // the kept amplitude moves to the target's half; :plus / :minus add a Hadamard
    K[0] = K[1] = K[2] = K[3] = 0;
    const double h = f * 0.70710678118654752440;
    switch (target) {
        case 0: K[m] = f; break;                  // row 0 takes column m
        case 1: K[2 + m] = f; break;              // row 1 takes column m
        case 2: K[m] = h, K[2 + m] = h; break;    // (|0> + |1>) / sqrt 2
        default: K[m] = h, K[2 + m] = -h; break;  // (|0> - |1>) / sqrt 2
    }
}

}  // namespace smoq

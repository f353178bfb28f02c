// smoq_internal.h -- shared definitions of libsmoq_cuda.so (host + device).
//
// Layout in HBM: a state object holds B states ("batch", e.g. MCWF
// trajectories or VQE parameter sets) of 2^N amplitudes each, state-major
// (state b at offset b * 2^N), amplitudes interleaved (re, im) exactly like
// Julia's Vector{ComplexF32/ComplexF64}.  Little-endian qubits: qubit k
// (0-based at this ABI) is bit k of the amplitude index.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <complex>
#include <string>
#include <vector>
#include "../../include/smoq_cuda.h"

namespace smoq {

using cd = std::complex<double>;

// ----------------------------------------------------------------------------
// Device op program.  One DevOp is one fused operation applied to every
// amplitude group of a tile (tile kernel) or of the whole state (direct
// kernel).  Matrix element (r, c) of a k-qubit op lives in c[r * 2^k + c];
// bit t of a local matrix index is the value of the op's qubit t.
// ----------------------------------------------------------------------------
enum OpKind : int32_t {
    OPK_DENSE1 = 0,   // 2x2 dense on qubit 0
    OPK_DENSE2 = 1,   // 4x4 dense on qubits (0, 1)
    OPK_PARITY2 = 2,  // 4x4 that keeps parity: even block {00,11}, odd block {01,10}
    OPK_MONO = 3,     // monomial (permutation x phase) on 1..3 qubits
    OPK_DIAG = 4,     // diagonal on 0..3 qubits; qubits need not be tile bits
    OPK_STATESCALE = 5,  // amp *= scale[b] (per state, real, from aux pointer)
    OPK_REALTAB = 6,  // amp *= prod_j tab[j][byte j of global index] (real factors)
    OPK_JUMP = 7,     // per-state jump (sigma-/sigma+/sigma_z/sigma_x) from aux list
    OPK_STAGE = 10,   // stage-sweep engine: header of a stage; perm[0..3] = the stage's 4
                      // tile bits (ascending), perm[4..7] = lane bit feeding the rotation of
                      // each stage bit (-1 none), aux2 = number of member ops that follow;
                      // nq = 0 marks a single op applied by a plain shared-memory sweep
    OPK_INNER = 9,    // adjoint sweep: Im<lambda|G|phi> on 1-2 tile bits, accumulated into
                      // partials column perm[0]; G is a signed monomial: row r holds i^slot[r]
                      // at column perm[1 + r] (slot[r] = INNER_ZERO: an all-zero row);
                      // flags: INNER_DIAGG (G real diagonal), INNER_PRE (cd/cf hold a dense
                      // 2^nq x 2^nq matrix applied to both states first), INNER_PREDIAG
                      // (that matrix is diagonal)
};


// OPK_INNER encoding details
enum InnerBits : int32_t { INNER_ZERO = 4, INNER_DIAGG = 1, INNER_PRE = 2, INNER_PREDIAG = 8 };
// OPK_DENSE1 / OPK_DENSE2 flag: every coefficient is real (Ry, CZ products): a
// kernel may multiply with real scalars, half the FMAs of complex coefficients
enum DenseBits : int32_t { OPF_REAL = 4 };
// OPK_DIAG flag: a diagonal split off a rotation (split_rotations): the stage schedule
// keeps its qubits on stage bits, so a compiled kernel folds it into literal phases
enum DiagFlagBits : int32_t { DIAG_STAGED = 16 };

struct alignas(16) DevOp {
    int32_t kind;
    int32_t nq;         // 1..3 qubits (OPK_DIAG: 0..4)
    int32_t lb[4];      // tile-local bit of qubit t, -1 when the qubit is not a tile bit
    int32_t gb[4];      // global bit of qubit t
    int32_t slot[4];    // stage engines: stage position of qubit t; OPK_INNER: the i^k codes
    int32_t mode;       // unused (kept: the compiled kernels mirror this layout)
    int32_t flags;      // OPK_PARITY2: bit 0 even block diagonal, bit 1 odd block diagonal
    int32_t pad0[2];
    int32_t perm[8];    // OPK_MONO: out[r] = ph[r] * in[perm[r]]
    const void* aux;    // OPK_STATESCALE: const double* scale[B]; OPK_REALTAB: const double* tabs
    int64_t aux2;       // OPK_REALTAB: number of byte tables
    double2 cd[16];     // coefficients, double precision
    float2 cf[16];      // the same, rounded to float (complex64 kernels)
};

// Tile geometry of one pass: the tile is the set of amplitudes whose index
// varies over the low L bits and over the high bits hb[0..H-1]; every other
// index bit is fixed by the tile number.
struct TileGeom {
    int32_t N, T, L, H;
    int32_t hb[24];
};

// Per-pass epilogue: per-tile partial sums of |psi|^2 and of |psi|^2 over
// amplitudes with bit q set (q in pop_mask order), written to
// partials[(tile_global) * (1 + npop) + j].
struct Epilogue {
    double* partials;   // nullptr: no epilogue
    int32_t npop;
    int32_t popq[40];
};

struct TileArgs {
    void* psi;
    int64_t state_len;       // 2^N
    int64_t tiles_per_state; // 2^(N-T)
    int64_t ntiles;          // B * tiles_per_state
    const DevOp* ops;
    int32_t nops;
    int32_t* err;
    TileGeom g;
    Epilogue ep;
};

// One Pauli-sum term on the device: coef * i^ny * X^x Z^z (ny = popcount(x & z),
// the Y letters: Y = i X Z)
struct HamTerm {
    double coef;
    uint64_t x, z;
    int32_t ny;
    int32_t pad;
};

// Arguments of the adjoint backward pass over the tile pair (phi, lambda); the
// compiled adjoint kernels (jit.cpp) mirror this layout
struct AdjArgs {
    TileArgs a;        // a.psi = phi
    void* lam;
    double* partials;  // [n_rows][n_cols]: row = CTA x warps + warp, column = measurement
    int64_t n_rows;
    int32_t n_cols;
};

// ----------------------------------------------------------------------------
// Host-side gate IR consumed by the planner.
// ----------------------------------------------------------------------------
// Storage of a gate matrix (up to 16 x 16): complex entries that are NOT
// initialised on construction -- a gate list holds thousands of these, and every
// producer writes the 2^nq x 2^nq block it uses before anything reads it.
struct GateMatrix {
    alignas(16) double v[512];
    cd& operator[](int i) { return reinterpret_cast<cd*>(v)[i]; }
    const cd& operator[](int i) const { return reinterpret_cast<const cd*>(v)[i]; }
    operator cd*() { return reinterpret_cast<cd*>(v); }
    operator const cd*() const { return reinterpret_cast<const cd*>(v); }
};

struct GateIR {
    int nq = 0;             // 0..3 qubits (diagonals merged by the fuser: up to 4)
    int q[4] = {0, 0, 0, 0};  // 0-based global qubits
    bool diag = false;      // diagonal in the computational basis (commutes with diagonals)
    int special = 0;        // 0: matrix gate; OPK_STATESCALE / OPK_REALTAB / OPK_JUMP
    const void* aux = nullptr;
    int64_t aux2 = 0;
    GateMatrix m;           // row-major 2^nq x 2^nq; bit t of an index = qubit q[t]
    int tag = -1;           // caller tag (e.g. parameter index) carried through
};

// a pass program compiled to its own kernel (engine 3, jit.cpp)
struct JitKernel {
    const void* fn[2] = {nullptr, nullptr};  // without / with the norm+population epilogue
    int threads = 0;
    int per_sm[2] = {1, 1};
    size_t smem = 0;
    bool rtc = false;  // takes the run-time coefficient block as its second parameter
};

struct Pass {
    TileGeom g;
    std::vector<DevOp> ops;
    bool epilogue = false;
    bool staged = false;    // scheduled for the stage-sweep engine (OPK_STAGE headers)
    bool want_jit = false;  // engine 3: compile this staged pass to its own kernel at upload
    bool rtc = false;       // compiled kernel reads the op coefficients at run time: its
                            // source depends on the circuit's structure, not its angles
    std::vector<float2> coefs;  // with rtc: the coefficient block of this pass's launches
    const JitKernel* jit = nullptr;
};

// planner.cpp
std::vector<Pass> plan_passes(const std::vector<GateIR>& gates, int N, int T, int Lmin,
                              int epilogue_after_special = -1, int Lreq = 0);
// turn a planned pass into stage sweeps of 4 tile bits (engines 2, 3); amp_bytes
// selects the bank geometry
void schedule_stages(Pass& p, int amp_bytes, bool allow_inner = false, bool split = false);
void build_devop(const GateIR& gt, const TileGeom* g, DevOp& op);
// jit.cpp: compile (or fetch from the process cache) the kernel of a staged complex64 pass
// (minb_add: that many more CTAs per SM than the default register budget allows)
const JitKernel* jit_pass_kernel(const Pass& p, int nbuf, int groups, std::string& err, int minb_add = 0);
// one kernel variant of a staged pass, for jit_precompile
struct JitRequest {
    const Pass* p;
    int nbuf, groups, minb_add;
};
// jit.cpp: compile the requested kernels with NVRTC on host threads (no CUDA
// calls there); a later jit_pass_kernel of the same variant only loads it
void jit_precompile(const std::vector<JitRequest>& reqs);
// jit.cpp: the compiled kernel of a staged ADJOINT pass (complex64): U^dag ops on the
// tile pair (phi, lambda) and the OPK_INNER measurements in 4-bit register stages
std::string jit_adjoint_source(const Pass& p, std::string& err);
// compile generated sources with NVRTC on host threads (no CUDA calls) for a later load
void jit_precompile_sources(const std::vector<const std::string*>& srcs);
// the structural signature of a staged pass (equal signatures: equal kernel sources)
std::vector<int32_t> jit_pass_signature(const Pass& p);
// the loaded kernel of a signature, or nullptr
const JitKernel* jit_sig_find(const std::vector<int32_t>& sig);
// load the adjoint kernel of `p` from its source (compiled ahead, or compiled here)
// and file it under its signature
const JitKernel* jit_adjoint_load(const Pass& p, const std::string& src, const std::vector<int32_t>& sig,
                                  std::string& err);
// jit.cpp: the run-time coefficient block of a pass compiled with rtc (the kernel's
// second parameter, in the order the generated code indexes it)
void jit_rtc_block(const Pass& p, std::vector<float2>& out);
// the kernel parameter space of a launch (CUDA 12.1+ on Volta and later)
constexpr size_t kMaxKernelParamBytes = 32764;
// jit.cpp: generate and compile the adjoint kernel of a staged backward pass without
// loading it (host only); `info` (optional) receives the compiler's resource report;
// with `source` the generated source is returned there instead of being compiled
bool jit_check_adjoint(const Pass& p, std::string& err, std::string* info, std::string* source = nullptr);
// the tuning-cache key of a staged pass program (hash of its default kernel source)
uint64_t jit_pass_key(const Pass& p, int nbuf);
// jit.cpp: generate and compile a staged complex64 pass without a GPU (plan checks)
bool jit_check_pass(const Pass& p, int nbuf, int groups, std::string& err, size_t* cubin_bytes, std::string* info);
// jit.cpp: the loaded kernel of a run-time-coefficient pass with this signature and
// variant, or nullptr (no source generated)
const JitKernel* jit_pass_find(const Pass& p, int nbuf, int groups, int minb_add);
// jit.cpp: the generated source of a staged complex64 pass (host only)
bool jit_pass_source(const Pass& p, int nbuf, int groups, std::string& src, std::string& err);
// jit.cpp: NVRTC could be loaded
bool jit_available();

// gate library (planner.cpp)
GateIR gate_1q(int q, const cd m[4]);
GateIR gate_2q(int q0, int q1, const cd m[16]);
GateIR gate_named(int type, const int* q, double angle);

}  // namespace smoq

// ----------------------------------------------------------------------------
// Objects behind the opaque C handles.
// ----------------------------------------------------------------------------
struct smoq_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int32_t* d_err = nullptr;          // device error word (timeouts, bad input)
    double* d_scratch = nullptr;       // reduction partials
    size_t scratch_bytes = 0;
    double* h_pinned = nullptr;        // pinned host staging for small results
    size_t pinned_bytes = 0;
    int tile_bits_c64 = 13;
    int tile_bits_c128 = 12;
    int low_bits_c64 = 5;
    int low_bits_c128 = 4;
    int use_graphs = 1;
    int engine = -1;                   // fused passes: -1 = auto, 0 = shared-memory sweeps,
                                       // 2 = stage sweeps, 3 = compiled pass kernels
    int st_occ[2][2][2] = {};          // CTAs per SM of the stage kernel [dtype][epilogue][GP-1]
    int kernel_timing = 0;             // bracket tile passes with events
    int jit_buffers = 1;               // compiled pass kernels: tile buffers per CTA (1 or 2)
    int jit_groups = 2;                // compiled pass kernels: 16-amplitude register groups per thread
    bool vqe_resident = true;          // many-circuit VQE: small circuits in one shared-memory launch
    bool autotune = true;              // tune plan geometry and compiled-kernel variants at plan upload
    bool tune_geometry = true;         // ... the geometry too (else the options' tile width, low bits, depth)
    int fusion_depth = 0;              // max fused ops per pass (0 = as many as fit)
    std::string tune_report;           // the tuner's per-pass timings and choices
    long long launches = 0;            // kernels launched by this ctx
    long long tile_passes = 0;
    double tile_ms = 0;                // summed tile-pass time when kernel_timing
    double tile_bytes = 0;             // algorithmic bytes of the timed tile passes
    int num_sms = 148;
    int tile_occ[2][2][16] = {};       // CTAs per SM of tile_pass_kernel [dtype][epilogue][T]
    std::vector<smoq_ctx*> workers;    // worker contexts of the many-circuit VQE call
};

struct smoq_state {
    smoq_ctx* ctx = nullptr;
    int N = 0;
    int dtype = SMOQ_C64;
    int batch = 1;
    void* ptr = nullptr;
    bool owned = true;
    size_t amp_bytes() const { return dtype == SMOQ_C64 ? 8 : 16; }
    size_t bytes() const { return ((size_t)1 << N) * (size_t)batch * amp_bytes(); }
};

// kernels (k_*.cu)
namespace smoq {
cudaError_t launch_direct_op(smoq_state* st, const DevOp& op);
cudaError_t launch_tile_pass(smoq_ctx* ctx, smoq_state* st, const Pass& p, const DevOp* d_ops,
                             const Epilogue* ep);
cudaError_t launch_diag_reduce(smoq_ctx* ctx, smoq_state* st, const uint64_t* zmasks, int nobs,
                               double* d_out);
cudaError_t launch_pauli_reduce(smoq_ctx* ctx, smoq_state* st, uint64_t xmask, uint64_t zmask,
                                int ny, double* d_out);
cudaError_t launch_set_basis(smoq_state* st, uint64_t index);
// a bounded mbarrier wait that nothing completes (the failure path's test)
cudaError_t launch_wait_timeout_probe(smoq_ctx* ctx, uint64_t limit_ns);
cudaError_t launch_scale(smoq_state* st, const double* d_scale_per_state, double scalar);
cudaError_t launch_convert(smoq_state* dst, smoq_state* src);
size_t diag_reduce_scratch_doubles(smoq_state* st, int nobs);
size_t tile_max_smem(int amp_bytes, int T);
cudaError_t tile_kernels_init(smoq_ctx* ctx);
cudaError_t stage_kernels_init(smoq_ctx* ctx);
cudaError_t launch_stage(smoq_ctx* ctx, const TileArgs& a, int dtype, bool epi);
cudaError_t launch_jit(smoq_ctx* ctx, const TileArgs& a, const JitKernel* k, bool epi,
                       const float2* coefs = nullptr);
cudaError_t vqe_kernels_init(smoq_ctx* ctx);
// lam = H psi for one state (vqe.cu); per block the FP64 partials of Re<psi|lam>
// (d_part[blk]) and <psi|psi> (d_part[eblocks + blk])
cudaError_t launch_ham_apply(smoq_ctx* ctx, const smoq_state* st, void* lam, const HamTerm* d_terms, int nterms,
                             double* d_part, int eblocks);
cudaError_t qrc_kernels_init(smoq_ctx* ctx);
}  // namespace smoq

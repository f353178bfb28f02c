// capi.cu -- the extern "C" entry points of libsmoq_cuda.so (include/smoq_cuda.h).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include "smoq_internal.h"
#include "k_common.cuh"

using namespace smoq;

// ------------------------------------------------------------------ helpers
static smoq_status fail(smoq_ctx* ctx, smoq_status s, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return s;
}
static smoq_status cuda_fail(smoq_ctx* ctx, cudaError_t e, const char* where) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return fail(ctx, SMOQ_ERR_OOM, buf);
    return fail(ctx, SMOQ_ERR_CUDA, buf);
}
#define CK(ctx, call)                                              \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
    } while (0)

static smoq_status check_state(smoq_state* st) {
    if (!st || !st->ctx) return SMOQ_ERR_BADINPUT;
    return SMOQ_OK;
}
static smoq_status check_q(smoq_state* st, int q, const char* what) {
    if (q < 0 || q >= st->N) {
        char b[160];
        snprintf(b, sizeof(b), "%s: qubit %d out of range for N=%d", what, q, st->N);
        return fail(st->ctx, SMOQ_ERR_BADINPUT, b);
    }
    return SMOQ_OK;
}
static smoq_status ensure_scratch(smoq_ctx* ctx, size_t doubles) {
    const size_t bytes = doubles * sizeof(double);
    if (bytes <= ctx->scratch_bytes) return SMOQ_OK;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    ctx->d_scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t nb = std::max(bytes, (size_t)1 << 20);
    CK(ctx, cudaMalloc(&ctx->d_scratch, nb));
    ctx->scratch_bytes = nb;
    return SMOQ_OK;
}
static smoq_status ensure_pinned(smoq_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->pinned_bytes) return SMOQ_OK;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    ctx->h_pinned = nullptr;
    ctx->pinned_bytes = 0;
    size_t nb = std::max(bytes, (size_t)1 << 20);
    CK(ctx, cudaMallocHost((void**)&ctx->h_pinned, nb));
    ctx->pinned_bytes = nb;
    return SMOQ_OK;
}
// sync the ctx stream and turn a device error word into a status
static smoq_status sync_check(smoq_ctx* ctx) {
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    int32_t h = 0;
    CK(ctx, cudaMemcpy(&h, ctx->d_err, sizeof(h), cudaMemcpyDeviceToHost));
    if (h != 0) {
        CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream));
        if (h == DEVERR_TIMEOUT) return fail(ctx, SMOQ_ERR_TIMEOUT, "a bounded device wait ran out");
        if ((h & 255) == DEVERR_BOUNDS)
            return fail(ctx, SMOQ_ERR_CUDA, "device bounds check failed at site " + std::to_string(h >> 8));
        return fail(ctx, SMOQ_ERR_BADINPUT, "device-side input check failed");
    }
    return SMOQ_OK;
}

static int tile_bits(smoq_ctx* ctx, int dtype) {
    return dtype == SMOQ_C64 ? ctx->tile_bits_c64 : ctx->tile_bits_c128;
}
static int low_bits(smoq_ctx* ctx, int dtype) {
    return dtype == SMOQ_C64 ? ctx->low_bits_c64 : ctx->low_bits_c128;
}

// fused-pass engine of a program: the ctx option, or in auto mode (-1) the
// compiled pass kernels for reusable complex64 programs (Trotter plans, MCWF)
// when NVRTC is available and the shared-memory sweeps otherwise
static int engine_for(smoq_ctx* ctx, bool reusable, int dtype) {
    if (ctx->engine >= 0) return ctx->engine;
    return (reusable && dtype == SMOQ_C64 && jit_available()) ? 3 : 0;
}

// the fusion depth: a pass with more than `cap` fused ops becomes consecutive
// passes of the same tile geometry (the ops keep their order, and every op of a
// pass acts on that pass's tile, so the split changes nothing but the count)
static void cap_fusion_depth(std::vector<Pass>& pl, int cap) {
    if (cap <= 0) return;
    std::vector<Pass> out;
    for (Pass& p : pl) {
        if ((int)p.ops.size() <= cap) {
            out.push_back(std::move(p));
            continue;
        }
        for (size_t i = 0; i < p.ops.size(); i += (size_t)cap) {
            Pass q;
            q.g = p.g;
            q.ops.assign(p.ops.begin() + i, p.ops.begin() + std::min(p.ops.size(), i + (size_t)cap));
            q.epilogue = p.epilogue && i + (size_t)cap >= p.ops.size();
            out.push_back(std::move(q));
        }
    }
    pl.swap(out);
}

// plan a gate list into fused passes; with the stage engines every pass of
// tile width 12 (13 for complex64) gets a stage schedule
// rtc: the compiled kernels read their coefficients at run time (a variational
// circuit: one compile per circuit structure serves every parameter set)
static std::vector<Pass> plan_for(int engine, const std::vector<GateIR>& ir, int N, int dtype, int tbits, int lbits,
                                  int epilogue_special = -1, int max_ops = 0, bool rtc = false) {
    std::vector<Pass> pl = plan_passes(ir, N, tbits, lbits, epilogue_special, dtype == SMOQ_C64 ? 1 : 0);
    cap_fusion_depth(pl, max_ops);
    if (engine == 2 || engine == 3)
        for (Pass& p : pl)
            if (p.g.T == 12 || (p.g.T == 13 && dtype == SMOQ_C64)) {
                // literal compiled kernels: rotations split into diagonals the kernel folds
                const bool jit = engine == 3 && dtype == SMOQ_C64;
                schedule_stages(p, dtype == SMOQ_C64 ? 8 : 16, false, jit && !rtc);
                p.want_jit = jit && p.staged;
                if (p.want_jit && rtc) {
                    p.rtc = true;
                    jit_rtc_block(p, p.coefs);
                    // (a block beyond the parameter space: the stage-sweep engine runs the pass)
                    if (sizeof(TileArgs) + sizeof(float2) * p.coefs.size() > kMaxKernelParamBytes) {
                        p.rtc = p.want_jit = false;
                        p.coefs.clear();
                    }
                }
            }
    return pl;
}

// ------------------------------------------------------------ pass runner
namespace {
struct DevProgram {
    std::vector<Pass> passes;
    std::vector<size_t> offs;  // first op of each pass in d_ops
    DevOp* d_ops = nullptr;
    cudaStream_t s = nullptr;  // the stream d_ops was allocated on (stream-ordered free:
                               // cudaFree would wait for every stream of the device)
    size_t nops = 0;
    int epi_pass = -1;
    ~DevProgram() {
        if (d_ops) cudaFreeAsync(d_ops, s);
    }
};
}  // namespace

static smoq_status upload_program(smoq_ctx* ctx, DevProgram& P) {
    std::vector<JitRequest> reqs;
    for (Pass& p : P.passes) {
        if (p.want_jit && !p.jit && p.rtc)  // a known structure: no source generated
            p.jit = jit_pass_find(p, ctx->jit_buffers, ctx->jit_groups, 0);
        if (p.want_jit && !p.jit) reqs.push_back(JitRequest{&p, ctx->jit_buffers, ctx->jit_groups, 0});
    }
    if (reqs.size() > 1) jit_precompile(reqs);
    for (Pass& p : P.passes) {
        if (!p.want_jit || p.jit) continue;
        std::string why;
        p.jit = jit_pass_kernel(p, ctx->jit_buffers, ctx->jit_groups, why);
        if (!p.jit) return fail(ctx, SMOQ_ERR_UNSUPPORTED, "compiled pass kernel: " + why);
    }
    std::vector<DevOp> all;
    P.offs.clear();
    for (size_t i = 0; i < P.passes.size(); ++i) {
        P.offs.push_back(all.size());
        all.insert(all.end(), P.passes[i].ops.begin(), P.passes[i].ops.end());
        if (P.passes[i].epilogue) P.epi_pass = (int)i;
    }
    P.nops = all.size();
    if (all.empty()) return SMOQ_OK;
    if (P.d_ops) CK(ctx, cudaFreeAsync(P.d_ops, P.s));  // (a program uploaded again)
    P.d_ops = nullptr;
    P.s = ctx->stream;
    CK(ctx, cudaMallocAsync((void**)&P.d_ops, all.size() * sizeof(DevOp), ctx->stream));
    // on the context's (non-blocking) stream: a cudaMemcpy from pageable memory may
    // return before its DMA lands, and nothing would order it before the passes
    CK(ctx, cudaMemcpyAsync(P.d_ops, all.data(), all.size() * sizeof(DevOp), cudaMemcpyHostToDevice, ctx->stream));
    return SMOQ_OK;
}

struct EventPair {
    cudaEvent_t a, b;
    double bytes;
};

// ================================================================ autotuner
// For every compiled pass of a reusable program (engine 3) the tuner times the
// kernel variants -- 16-amplitude register groups per thread (2 or 1), CTAs per
// SM (the register budget's default, or one more), and one tile buffer per CTA
// or two (the next tile's bulk load in flight under the current tile's stages)
// -- on a zeroed scratch state of the program's size with CUDA events on the
// context's stream, and keeps the fastest.  The variants apply the same literal
// FMA sequence to every amplitude, so the choice changes the timing, never the
// result.  States below 2^20 amplitudes are not tuned (their passes take
// microseconds).  Choices are
// cached per (GPU, pass program) for the life of the process and, when the
// environment variable SMOQ_TUNE_CACHE names a file, across processes (one
// line per pass program: key, variant).  Passes whose ops read per-state
// runtime data (MCWF scales, decay tables, jumps) or carry an epilogue keep
// the default variant.
namespace {
struct TuneVariant {
    int groups, minb_add, nbuf;
};
const TuneVariant kTuneVariants[] = {{2, 0, 1}, {2, 1, 1}, {1, 0, 1}, {1, 1, 1}, {2, 0, 2}, {1, 0, 2}};
constexpr int kTuneVariantCount = 6;
constexpr int kTuneMinN = 20;
std::mutex g_tune_mu;
std::map<uint64_t, int> g_tune;
bool g_tune_loaded = false;

uint64_t device_hash(int device) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    uint64_t h = 1469598103934665603ull;
    for (const char* c = prop.name; *c; ++c) h = (h ^ (unsigned char)*c) * 1099511628211ull;
    return (h ^ (uint64_t)prop.multiProcessorCount) * 1099511628211ull;
}

void tune_cache_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("SMOQ_TUNE_CACHE");
    if (!path || !*path) return;
    std::ifstream f(path);
    std::string key;
    int v;
    while (f >> key >> v)
        if (v >= 0 && v < kTuneVariantCount) g_tune[std::strtoull(key.c_str(), nullptr, 16)] = v;
}

void tune_cache_store_locked(uint64_t key, int v) {
    g_tune[key] = v;
    const char* path = std::getenv("SMOQ_TUNE_CACHE");
    if (!path || !*path) return;
    std::ofstream f(path, std::ios::app);
    char k[32];
    std::snprintf(k, sizeof k, "%016llx", (unsigned long long)key);
    f << k << " " << v << "\n";
}

bool tunable(const Pass& p) {
    if (!p.jit || p.epilogue) return false;
    for (const DevOp& op : p.ops)
        if (op.kind == OPK_STATESCALE || op.kind == OPK_REALTAB || op.kind == OPK_JUMP) return false;
    return true;
}
}  // namespace

static smoq_status autotune_program(smoq_ctx* ctx, DevProgram& P, int N) {
    if (N < kTuneMinN) return SMOQ_OK;
    std::vector<size_t> todo;
    for (size_t i = 0; i < P.passes.size(); ++i)
        if (tunable(P.passes[i]) && !P.passes[i].ops.empty()) todo.push_back(i);
    if (todo.empty()) return SMOQ_OK;
    const uint64_t dh = device_hash(ctx->device);
    // the cached choices first
    std::vector<uint64_t> keys(P.passes.size(), 0);
    std::vector<size_t> fresh;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_cache_load_locked();
        for (size_t i : todo) {
            keys[i] = jit_pass_key(P.passes[i], 1) ^ dh;
            auto it = g_tune.find(keys[i]);
            if (it == g_tune.end()) {
                fresh.push_back(i);
                continue;
            }
            const TuneVariant& v = kTuneVariants[it->second];
            std::string why;
            if (const JitKernel* k = jit_pass_kernel(P.passes[i], v.nbuf, v.groups, why, v.minb_add))
                P.passes[i].jit = k;
        }
    }
    if (fresh.empty()) return SMOQ_OK;
    // scratch state: only when it fits twice over with a GiB to spare
    const size_t bytes = (size_t)8 << N;
    size_t free_b = 0, total_b = 0;
    CK(ctx, cudaMemGetInfo(&free_b, &total_b));
    if (free_b < 2 * bytes + ((size_t)1 << 30)) {
        ctx->tune_report += "autotune skipped: no room for a scratch state\n";
        return SMOQ_OK;
    }
    // compile every variant of every fresh pass with NVRTC on host threads, then load them here
    std::vector<const JitKernel*> ks(fresh.size() * kTuneVariantCount, nullptr);
    {
        std::vector<JitRequest> reqs;
        for (size_t j = 0; j < ks.size(); ++j) {
            const TuneVariant& v = kTuneVariants[j % kTuneVariantCount];
            reqs.push_back(JitRequest{&P.passes[fresh[j / kTuneVariantCount]], v.nbuf, v.groups, v.minb_add});
        }
        jit_precompile(reqs);
        for (size_t j = 0; j < ks.size(); ++j) {
            const TuneVariant& v = kTuneVariants[j % kTuneVariantCount];
            std::string why;
            ks[j] = jit_pass_kernel(P.passes[fresh[j / kTuneVariantCount]], v.nbuf, v.groups, why, v.minb_add);
        }
    }
    void* scratch = nullptr;
    CK(ctx, cudaMallocAsync(&scratch, bytes, ctx->stream));
    std::unique_ptr<void, std::function<void(void*)>> hold(scratch, [ctx](void* q) { cudaFreeAsync(q, ctx->stream); });
    CK(ctx, cudaMemsetAsync(scratch, 0, bytes, ctx->stream));
    cudaEvent_t e0, e1;
    CK(ctx, cudaEventCreate(&e0));
    CK(ctx, cudaEventCreate(&e1));
    std::ostringstream rep;
    const long long launches0 = ctx->launches;
    for (size_t f = 0; f < fresh.size(); ++f) {
        Pass& p = P.passes[fresh[f]];
        TileArgs a;
        a.psi = scratch;
        a.state_len = (int64_t)1 << N;
        a.tiles_per_state = (int64_t)1 << (N - p.g.T);
        a.ntiles = a.tiles_per_state;
        a.ops = P.d_ops + P.offs[fresh[f]];
        a.nops = (int32_t)p.ops.size();
        a.err = ctx->d_err;
        a.g = p.g;
        a.ep.partials = nullptr;
        a.ep.npop = 0;
        int best = -1;
        float best_ms = 0;
        rep << "pass " << fresh[f] << " (T " << p.g.T << ", L " << p.g.L << ", " << p.ops.size() << " ops):";
        for (int v = 0; v < kTuneVariantCount; ++v) {
            const JitKernel* k = ks[f * kTuneVariantCount + v];
            if (!k) continue;
            const float2* kc = p.rtc ? p.coefs.data() : nullptr;
            cudaError_t e = launch_jit(ctx, a, k, false, kc);  // warm-up
            cudaEventRecord(e0, ctx->stream);
            for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch_jit(ctx, a, k, false, kc);
            cudaEventRecord(e1, ctx->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return cuda_fail(ctx, e, "autotune launch");
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= 3;
            rep << " v" << v << " " << ms;
            if (best < 0 || ms < best_ms) best = v, best_ms = ms;
        }
        rep << " -> v" << best << "\n";
        if (best >= 0) {
            p.jit = ks[f * kTuneVariantCount + best];
            std::lock_guard<std::mutex> lk(g_tune_mu);
            tune_cache_store_locked(keys[fresh[f]], best);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches = launches0;  // the timing launches are not the caller's work
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    int32_t herr = 0;
    CK(ctx, cudaMemcpy(&herr, ctx->d_err, sizeof(herr), cudaMemcpyDeviceToHost));
    if (herr) {
        CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream));
        return fail(ctx, SMOQ_ERR_TIMEOUT, "autotune: a bounded device wait ran out");
    }
    ctx->tune_report += rep.str();
    return SMOQ_OK;
}

static smoq_status run_program(smoq_ctx* ctx, smoq_state* st, const DevProgram& P, const Epilogue* ep,
                               std::vector<EventPair>* timing) {
    for (size_t i = 0; i < P.passes.size(); ++i) {
        const Pass& p = P.passes[i];
        if (p.ops.empty()) continue;
        EventPair ev{};
        if (timing) {
            cudaEventCreate(&ev.a);
            cudaEventCreate(&ev.b);
            cudaEventRecord(ev.a, ctx->stream);
        }
        cudaError_t e = launch_tile_pass(ctx, st, p, P.d_ops + P.offs[i], p.epilogue ? ep : nullptr);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "tile pass launch");
        ctx->tile_passes++;
        if (timing) {
            cudaEventRecord(ev.b, ctx->stream);
            ev.bytes = 2.0 * (double)st->bytes();
            timing->push_back(ev);
        }
    }
    return SMOQ_OK;
}

static void harvest_timing(smoq_ctx* ctx, std::vector<EventPair>& timing) {
    for (auto& ev : timing) {
        float ms = 0;
        cudaEventSynchronize(ev.b);
        cudaEventElapsedTime(&ms, ev.a, ev.b);
        ctx->tile_ms += ms;
        ctx->tile_bytes += ev.bytes;
        cudaEventDestroy(ev.a);
        cudaEventDestroy(ev.b);
    }
    timing.clear();
}

// ================================================================= context
extern "C" {

const char* smoq_version(void) { return "smoq_cuda 0.1 sm_100a"; }

int smoq_jit_available(void) { return jit_available() ? 1 : 0; }

smoq_status smoq_ctx_create(int device, smoq_ctx** out) {
    if (!out) return SMOQ_ERR_BADINPUT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return SMOQ_ERR_NOGPU;
    if (device < 0 || device >= n) return SMOQ_ERR_BADINPUT;
    std::unique_ptr<smoq_ctx> ctx(new smoq_ctx());
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return SMOQ_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return SMOQ_ERR_CUDA;
    ctx->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return SMOQ_ERR_CUDA;
    if (cudaMalloc(&ctx->d_err, sizeof(int32_t)) != cudaSuccess) return SMOQ_ERR_OOM;
    if (cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return SMOQ_ERR_CUDA;
    if (tile_kernels_init(ctx.get()) != cudaSuccess) return SMOQ_ERR_CUDA;
    if (stage_kernels_init(ctx.get()) != cudaSuccess) return SMOQ_ERR_CUDA;
    if (vqe_kernels_init(ctx.get()) != cudaSuccess) return SMOQ_ERR_CUDA;
    if (qrc_kernels_init(ctx.get()) != cudaSuccess) return SMOQ_ERR_CUDA;
    if (ensure_scratch(ctx.get(), 1 << 17) != SMOQ_OK) return SMOQ_ERR_OOM;
    if (ensure_pinned(ctx.get(), 1 << 20) != SMOQ_OK) return SMOQ_ERR_OOM;
    *out = ctx.release();
    return SMOQ_OK;
}

smoq_status smoq_ctx_destroy(smoq_ctx* ctx) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    for (smoq_ctx* w : ctx->workers) smoq_ctx_destroy(w);
    ctx->workers.clear();
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SMOQ_OK;
}

const char* smoq_last_error(smoq_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

smoq_status smoq_ctx_synchronize(smoq_ctx* ctx) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    return sync_check(ctx);
}

void* smoq_ctx_stream(smoq_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

smoq_status smoq_debug_wait_timeout(smoq_ctx* ctx, uint64_t limit_ns) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    if (limit_ns < 1000 || limit_ns > 100000000ull)
        return fail(ctx, SMOQ_ERR_BADINPUT, "wait limit must be in 1 us .. 100 ms");
    CK(ctx, launch_wait_timeout_probe(ctx, limit_ns));
    return sync_check(ctx);
}

smoq_status smoq_ctx_set_option(smoq_ctx* ctx, int option, long long v) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    switch (option) {
        case SMOQ_OPT_TILE_BITS_C64:
            if (v < 4 || v > 14) return fail(ctx, SMOQ_ERR_BADINPUT, "tile bits (c64) must be 4..14");
            ctx->tile_bits_c64 = (int)v;
            break;
        case SMOQ_OPT_TILE_BITS_C128:
            if (v < 3 || v > 13) return fail(ctx, SMOQ_ERR_BADINPUT, "tile bits (c128) must be 3..13");
            ctx->tile_bits_c128 = (int)v;
            break;
        case SMOQ_OPT_LOW_BITS_C64:
            if (v < 1 || v > 14) return fail(ctx, SMOQ_ERR_BADINPUT, "low bits (c64) must be 1..14");
            ctx->low_bits_c64 = (int)v;
            break;
        case SMOQ_OPT_LOW_BITS_C128:
            if (v < 0 || v > 13) return fail(ctx, SMOQ_ERR_BADINPUT, "low bits (c128) must be 0..13");
            ctx->low_bits_c128 = (int)v;
            break;
        case SMOQ_OPT_USE_GRAPHS: ctx->use_graphs = v != 0; break;
        case SMOQ_OPT_KERNEL_TIMING: ctx->kernel_timing = v != 0; break;
        case SMOQ_OPT_ENGINE:
            if (v < -1 || v > 3 || v == 1) return fail(ctx, SMOQ_ERR_BADINPUT, "engine must be -1 (auto), 0, 2 or 3");
            ctx->engine = (int)v;
            break;
        case SMOQ_OPT_JIT_GROUPS:
            if (v != 1 && v != 2) return fail(ctx, SMOQ_ERR_BADINPUT, "compiled-kernel register groups must be 1 or 2");
            ctx->jit_groups = (int)v;
            break;
        case SMOQ_OPT_JIT_BUFFERS:
            if (v != 1 && v != 2) return fail(ctx, SMOQ_ERR_BADINPUT, "compiled-kernel tile buffers must be 1 or 2");
            ctx->jit_buffers = (int)v;
            break;
        case SMOQ_OPT_VQE_RESIDENT: ctx->vqe_resident = v != 0; break;
        case SMOQ_OPT_AUTOTUNE:
            if (v < 0 || v > 2) return fail(ctx, SMOQ_ERR_BADINPUT, "autotune must be 0, 1 or 2");
            ctx->autotune = v != 0;
            ctx->tune_geometry = v == 1;
            break;
        case SMOQ_OPT_FUSION_DEPTH:
            if (v < 0 || v > 1000000) return fail(ctx, SMOQ_ERR_BADINPUT, "fusion depth must be >= 0");
            ctx->fusion_depth = (int)v;
            break;
        default: return fail(ctx, SMOQ_ERR_BADINPUT, "unknown option");
    }
    return SMOQ_OK;
}

smoq_status smoq_ctx_tune_report(smoq_ctx* ctx, char* buf, int len) {
    if (!ctx || !buf || len < 1) return SMOQ_ERR_BADINPUT;
    std::strncpy(buf, ctx->tune_report.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
    return SMOQ_OK;
}

smoq_status smoq_ctx_counters(smoq_ctx* ctx, long long* launches, long long* tile_passes, double* tile_ms,
                              double* tile_bytes) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    if (launches) *launches = ctx->launches;
    if (tile_passes) *tile_passes = ctx->tile_passes;
    if (tile_ms) *tile_ms = ctx->tile_ms;
    if (tile_bytes) *tile_bytes = ctx->tile_bytes;
    return SMOQ_OK;
}

smoq_status smoq_ctx_reset_counters(smoq_ctx* ctx) {
    if (!ctx) return SMOQ_ERR_BADINPUT;
    ctx->launches = 0;
    ctx->tile_passes = 0;
    ctx->tile_ms = 0;
    ctx->tile_bytes = 0;
    return SMOQ_OK;
}

// ================================================================== states
smoq_status smoq_state_create(smoq_ctx* ctx, int N, smoq_dtype dtype, int batch, smoq_state** out) {
    if (!ctx || !out) return SMOQ_ERR_BADINPUT;
    *out = nullptr;
    if (N < 1 || N > 40) return fail(ctx, SMOQ_ERR_BADINPUT, "N must be in 1..40");
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return fail(ctx, SMOQ_ERR_BADINPUT, "bad dtype");
    if (batch < 1) return fail(ctx, SMOQ_ERR_BADINPUT, "batch must be >= 1");
    std::unique_ptr<smoq_state> st(new smoq_state());
    st->ctx = ctx;
    st->N = N;
    st->dtype = dtype;
    st->batch = batch;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaMalloc(&st->ptr, st->bytes());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "smoq_state_create");
    e = cudaMemsetAsync(st->ptr, 0, st->bytes(), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "smoq_state_create memset");
    *out = st.release();
    return SMOQ_OK;
}

smoq_status smoq_state_wrap(smoq_ctx* ctx, void* devptr, int N, smoq_dtype dtype, int batch,
                            smoq_state** out) {
    if (!ctx || !out || !devptr) return SMOQ_ERR_BADINPUT;
    if (((uintptr_t)devptr & 15) != 0) return fail(ctx, SMOQ_ERR_BADINPUT, "device pointer must be 16-byte aligned");
    if (N < 1 || N > 40 || batch < 1 || (dtype != SMOQ_C64 && dtype != SMOQ_C128))
        return fail(ctx, SMOQ_ERR_BADINPUT, "bad state shape");
    smoq_state* st = new smoq_state();
    st->ctx = ctx;
    st->N = N;
    st->dtype = dtype;
    st->batch = batch;
    st->ptr = devptr;
    st->owned = false;
    *out = st;
    return SMOQ_OK;
}

smoq_status smoq_state_destroy(smoq_state* st) {
    if (!st) return SMOQ_ERR_BADINPUT;
    if (st->owned && st->ptr) {
        cudaStreamSynchronize(st->ctx->stream);
        cudaFree(st->ptr);
    }
    delete st;
    return SMOQ_OK;
}

void* smoq_state_device_ptr(smoq_state* st) { return st ? st->ptr : nullptr; }

smoq_status smoq_state_upload(smoq_state* st, const void* host, size_t bytes) {
    if (check_state(st) || !host) return SMOQ_ERR_BADINPUT;
    if (bytes != st->bytes()) return fail(st->ctx, SMOQ_ERR_BADINPUT, "upload size mismatch");
    CK(st->ctx, cudaMemcpyAsync(st->ptr, host, bytes, cudaMemcpyHostToDevice, st->ctx->stream));
    return SMOQ_OK;
}

smoq_status smoq_state_download(smoq_state* st, void* host, size_t bytes) {
    if (check_state(st) || !host) return SMOQ_ERR_BADINPUT;
    if (bytes != st->bytes()) return fail(st->ctx, SMOQ_ERR_BADINPUT, "download size mismatch");
    CK(st->ctx, cudaMemcpyAsync(host, st->ptr, bytes, cudaMemcpyDeviceToHost, st->ctx->stream));
    return sync_check(st->ctx);
}

smoq_status smoq_state_download_range(smoq_state* st, uint64_t first, uint64_t count, void* host) {
    if (check_state(st) || (!host && count)) return SMOQ_ERR_BADINPUT;
    const uint64_t total = (uint64_t)st->batch << st->N;
    if (first > total || count > total - first) return fail(st->ctx, SMOQ_ERR_BADINPUT, "download range out of bounds");
    if (!count) return SMOQ_OK;
    const size_t amp = st->amp_bytes();
    CK(st->ctx, cudaMemcpyAsync(host, (const char*)st->ptr + first * amp, count * amp, cudaMemcpyDeviceToHost,
                                st->ctx->stream));
    return sync_check(st->ctx);
}

smoq_status smoq_state_set_basis(smoq_state* st, uint64_t index) {
    if (check_state(st)) return SMOQ_ERR_BADINPUT;
    if (st->N < 64 && index >= (1ull << st->N)) return fail(st->ctx, SMOQ_ERR_BADINPUT, "basis index out of range");
    CK(st->ctx, launch_set_basis(st, index));
    return SMOQ_OK;
}

smoq_status smoq_state_copy(smoq_state* dst, smoq_state* src) {
    if (check_state(dst) || check_state(src)) return SMOQ_ERR_BADINPUT;
    if (dst->N != src->N || dst->batch != src->batch) return fail(src->ctx, SMOQ_ERR_BADINPUT, "shape mismatch");
    CK(src->ctx, launch_convert(dst, src));
    return SMOQ_OK;
}

// =================================================================== gates
static smoq_status apply_gate_ir(smoq_state* st, const GateIR& g) {
    DevOp op;
    try {
        build_devop(g, nullptr, op);
    } catch (const std::exception& ex) {
        return fail(st->ctx, SMOQ_ERR_BADINPUT, ex.what());
    }
    CK(st->ctx, launch_direct_op(st, op));
    return SMOQ_OK;
}

static smoq_status gate_common(smoq_state* st, int type, int nq, const int* q, double theta) {
    if (check_state(st)) return SMOQ_ERR_BADINPUT;
    for (int t = 0; t < nq; ++t) {
        if (smoq_status s = check_q(st, q[t], "gate")) return s;
        for (int u = 0; u < t; ++u)
            if (q[u] == q[t]) return fail(st->ctx, SMOQ_ERR_BADINPUT, "gate qubits must be distinct");
    }
    if (!std::isfinite(theta)) return fail(st->ctx, SMOQ_ERR_BADINPUT, "gate angle is not finite");
    return apply_gate_ir(st, gate_named(type, q, theta));
}

#define G1(name, TYPE)                                        \
    smoq_status name(smoq_state* st, int q) {                 \
        return gate_common(st, TYPE, 1, &q, 0.0);             \
    }
#define G1T(name, TYPE)                                       \
    smoq_status name(smoq_state* st, int q, double theta) {   \
        return gate_common(st, TYPE, 1, &q, theta);           \
    }
G1T(smoq_apply_rx, SMOQ_G_RX)
G1T(smoq_apply_ry, SMOQ_G_RY)
G1T(smoq_apply_rz, SMOQ_G_RZ)
G1(smoq_apply_h, SMOQ_G_H)
G1(smoq_apply_x, SMOQ_G_X)
G1(smoq_apply_y, SMOQ_G_Y)
G1(smoq_apply_z, SMOQ_G_Z)
G1(smoq_apply_s, SMOQ_G_S)
G1(smoq_apply_sdg, SMOQ_G_SDG)
G1(smoq_apply_t, SMOQ_G_T)
G1(smoq_apply_tdg, SMOQ_G_TDG)

smoq_status smoq_apply_cnot(smoq_state* st, int c, int t) {
    int q[2] = {c, t};
    return gate_common(st, SMOQ_G_CNOT, 2, q, 0.0);
}
smoq_status smoq_apply_cz(smoq_state* st, int a, int b) {
    int q[2] = {a, b};
    return gate_common(st, SMOQ_G_CZ, 2, q, 0.0);
}
smoq_status smoq_apply_cry(smoq_state* st, int c, int t, double theta) {
    int q[2] = {c, t};
    return gate_common(st, SMOQ_G_CRY, 2, q, theta);
}
smoq_status smoq_apply_rxx(smoq_state* st, int a, int b, double theta) {
    int q[2] = {a, b};
    return gate_common(st, SMOQ_G_RXX, 2, q, theta);
}
smoq_status smoq_apply_ryy(smoq_state* st, int a, int b, double theta) {
    int q[2] = {a, b};
    return gate_common(st, SMOQ_G_RYY, 2, q, theta);
}
smoq_status smoq_apply_rzz(smoq_state* st, int a, int b, double theta) {
    int q[2] = {a, b};
    return gate_common(st, SMOQ_G_RZZ, 2, q, theta);
}
smoq_status smoq_apply_ccz(smoq_state* st, int a, int b, int c) {
    int q[3] = {a, b, c};
    return gate_common(st, SMOQ_G_CCZ, 3, q, 0.0);
}
smoq_status smoq_apply_toffoli(smoq_state* st, int c1, int c2, int t) {
    int q[3] = {c1, c2, t};
    return gate_common(st, SMOQ_G_TOFFOLI, 3, q, 0.0);
}

// sigma- = |0><1| (moves the |1> amplitude to |0>, zeroes the source);
// sigma+ = |1><0|; both are monomial 2x2 with a zero row.
smoq_status smoq_apply_sigma_minus(smoq_state* st, int q) {
    if (check_state(st)) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "sigma_minus")) return s;
    cd m[4] = {0, 1, 0, 0};
    return apply_gate_ir(st, gate_1q(q, m));
}
smoq_status smoq_apply_sigma_plus(smoq_state* st, int q) {
    if (check_state(st)) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "sigma_plus")) return s;
    cd m[4] = {0, 0, 1, 0};
    return apply_gate_ir(st, gate_1q(q, m));
}

static void load_colmajor(const double* U, int n, cd* row_major) {
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) row_major[r * n + c] = cd(U[2 * (c * n + r)], U[2 * (c * n + r) + 1]);
}

smoq_status smoq_apply_u1(smoq_state* st, int q, const double* U) {
    if (check_state(st) || !U) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "u1")) return s;
    cd m[4];
    load_colmajor(U, 2, m);
    return apply_gate_ir(st, gate_1q(q, m));
}

static GateIR u2_gate(int q1, int q2, const double* U, int convention) {
    cd m[16];
    load_colmajor(U, 4, m);
    if (convention == 0) {
        // Trotter.jl:110-112: the smaller qubit is bit 0 of U's index whatever the order
        return gate_2q(std::min(q1, q2), std::max(q1, q2), m);
    }
    // RandomUnitaries.jl:327-333: U's bit 0 is q1 (SWAP-conjugated when q1 > q2)
    return gate_2q(q1, q2, m);
}

smoq_status smoq_apply_u2(smoq_state* st, int q1, int q2, const double* U, int convention) {
    if (check_state(st) || !U) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q1, "u2")) return s;
    if (smoq_status s = check_q(st, q2, "u2")) return s;
    if (q1 == q2) return fail(st->ctx, SMOQ_ERR_BADINPUT, "u2 qubits must differ");
    if (convention != 0 && convention != 1) return fail(st->ctx, SMOQ_ERR_BADINPUT, "bad u2 convention");
    return apply_gate_ir(st, u2_gate(q1, q2, U, convention));
}

// ================================================================ sequences
static smoq_status ops_to_ir(smoq_state* st, int N, const smoq_op* ops, int n, const double* theta,
                             std::vector<GateIR>& out) {
    smoq_ctx* ctx = st ? st->ctx : nullptr;
    out.clear();
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        const smoq_op& o = ops[i];
        int nq = 1;
        switch (o.type) {
            case SMOQ_G_CZ: case SMOQ_G_CNOT: case SMOQ_G_RXX: case SMOQ_G_RYY: case SMOQ_G_RZZ:
            case SMOQ_G_CRY: case SMOQ_G_U2: nq = 2; break;
            case SMOQ_G_CCZ: case SMOQ_G_TOFFOLI: nq = 3; break;
            default: nq = 1;
        }
        if (o.type < 0 || o.type > SMOQ_G_U2)
            return fail(ctx, SMOQ_ERR_BADINPUT,
                        o.type >= SMOQ_N_DEPOLARIZING ? "noise, measurement and reset ops need smoq_apply_circuit_mcwf"
                                                      : "unknown op type");
        if (o.if_outcome != 0)
            return fail(ctx, SMOQ_ERR_BADINPUT, "a conditional op (if_outcome) needs smoq_apply_circuit_mcwf");
        for (int t = 0; t < nq; ++t) {
            if (o.q[t] < 0 || o.q[t] >= N) return fail(ctx, SMOQ_ERR_BADINPUT, "op qubit out of range");
            for (int u = 0; u < t; ++u)
                if (o.q[u] == o.q[t]) return fail(ctx, SMOQ_ERR_BADINPUT, "op qubits must be distinct");
        }
        double a = o.angle;
        if (o.param >= 0) {
            if (!theta) return fail(ctx, SMOQ_ERR_BADINPUT, "op needs theta but theta is NULL");
            a = theta[o.param];
        }
        if (!std::isfinite(a)) return fail(ctx, SMOQ_ERR_BADINPUT, "op angle is not finite");
        if (o.type == SMOQ_G_U1) {
            cd m[4];
            load_colmajor(o.U, 2, m);
            out.push_back(gate_1q(o.q[0], m));
        } else if (o.type == SMOQ_G_U2) {
            out.push_back(u2_gate(o.q[0], o.q[1], o.U, 0));
        } else {
            out.push_back(gate_named(o.type, o.q, a));
        }
        out.back().tag = o.param;
    }
    return SMOQ_OK;
}

smoq_status smoq_apply_sequence(smoq_state* st, const smoq_op* ops, int n, const double* theta) {
    if (check_state(st) || (!ops && n > 0) || n < 0) return SMOQ_ERR_BADINPUT;
    if (n == 0) return SMOQ_OK;
    smoq_ctx* ctx = st->ctx;
    std::vector<GateIR> ir;
    if (smoq_status s = ops_to_ir(st, st->N, ops, n, theta, ir)) return s;
    DevProgram P;
    try {
        P.passes = plan_for(engine_for(ctx, false, st->dtype), ir, st->N, st->dtype, tile_bits(ctx, st->dtype),
                            low_bits(ctx, st->dtype), -1, ctx->fusion_depth);
    } catch (const std::exception& ex) {
        return fail(ctx, SMOQ_ERR_BADINPUT, ex.what());
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));  // P.d_ops is freed when P goes out of scope
    if (smoq_status s = upload_program(ctx, P)) return s;
    std::vector<EventPair> timing;
    smoq_status s = run_program(ctx, st, P, nullptr, ctx->kernel_timing ? &timing : nullptr);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    harvest_timing(ctx, timing);
    if (s) return s;
    return sync_check(ctx);
}


smoq_status smoq_debug_compile_plan(int N, smoq_dtype dtype, int tbits, int lbits, const smoq_op* ops, int n,
                                   const double* theta, int flags, int* n_compiled, char* msg, int msg_len) {
    const bool verbose = (flags & 1) != 0;
    if (N < 1 || N > 40 || n < 0 || (n > 0 && !ops) || !n_compiled) return SMOQ_ERR_BADINPUT;
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return SMOQ_ERR_BADINPUT;
    *n_compiled = 0;
    auto say = [&](const std::string& m) {
        if (msg && msg_len > 0) {
            std::strncpy(msg, m.c_str(), (size_t)msg_len - 1);
            msg[msg_len - 1] = 0;
        }
    };
    std::vector<GateIR> ir;
    if (smoq_status s = ops_to_ir(nullptr, N, ops, n, theta, ir)) return s;
    std::vector<Pass> pl;
    try {
        if (flags & ~(1 | 2 | 4 | 8 | 16 | 32)) {
            say("unknown flag");
            return SMOQ_ERR_BADINPUT;
        }
        pl = plan_for(3, ir, N, dtype, tbits, lbits, -1, 0, (flags & 4) != 0);
    } catch (const std::exception& e) {
        say(e.what());
        return SMOQ_ERR_BADINPUT;
    }
    std::string report;
    for (const Pass& p : pl) {
        if (!p.want_jit) continue;
        std::string why, info;
        if (flags & 16) {  // the generated source of the first compiled pass (32: of every pass)
            if (!jit_pass_source(p, (flags & 2) ? 2 : 1, (flags & 8) ? 1 : 2, info, why)) {
                say(why);
                return SMOQ_ERR_BADINPUT;
            }
            ++*n_compiled;
            report += info;
            if (p.rtc && (flags & 32)) {  // the pass's run-time coefficient block, after its source
                report += "\n//@coefs";
                char num[80];
                for (const float2& c : p.coefs) {
                    std::snprintf(num, sizeof num, " %a %a", (double)c.x, (double)c.y);
                    report += num;
                }
                report += "\n";
            }
            if (flags & 32) continue;
            say(report);
            return SMOQ_OK;
        }
        if (!jit_check_pass(p, (flags & 2) ? 2 : 1, (flags & 8) ? 1 : 2, why, nullptr, verbose ? &info : nullptr)) {
            say(why);
            return why.rfind("NVRTC (", 0) == 0 ? SMOQ_ERR_UNSUPPORTED : SMOQ_ERR_BADINPUT;
        }
        report += info;
        ++*n_compiled;
    }
    say(verbose || (flags & 16) ? report : std::string("ok"));
    return SMOQ_OK;
}

smoq_status smoq_debug_plan_sequence(int N, smoq_dtype dtype, int tbits, int lbits, int engine, const smoq_op* ops, int n,
                                     const double* theta, smoq_pass_info* passes, int max_passes,
                                     smoq_fused_op_info* fused, int max_fused, int* n_passes, int* n_fused) {
    if (N < 1 || N > 40 || n < 0 || (n > 0 && !ops) || !n_passes || !n_fused) return SMOQ_ERR_BADINPUT;
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return SMOQ_ERR_BADINPUT;
    if (engine < 0 || engine > 3 || engine == 1) return SMOQ_ERR_BADINPUT;
    std::vector<GateIR> ir;
    if (smoq_status s = ops_to_ir(nullptr, N, ops, n, theta, ir)) return s;
    std::vector<Pass> pl;
    try {
        pl = plan_for(engine, ir, N, dtype, tbits, lbits);
    } catch (const std::exception&) {
        return SMOQ_ERR_BADINPUT;
    }
    int np = 0, no = 0;
    for (const Pass& p : pl) {
        if (passes && np < max_passes) {
            smoq_pass_info& pi = passes[np];
            std::memset(&pi, 0, sizeof(pi));
            pi.T = p.g.T;
            pi.L = p.g.L;
            pi.H = p.g.H;
            pi.nops = (int32_t)p.ops.size();
            for (int m = 0; m < p.g.H; ++m) pi.hb[m] = p.g.hb[m];
        }
        ++np;
        for (const DevOp& op : p.ops) {
            if (fused && no < max_fused) {
                smoq_fused_op_info& fi = fused[no];
                std::memset(&fi, 0, sizeof(fi));
                fi.kind = op.kind;
                fi.nq = op.nq;
                for (int t = 0; t < 4; ++t) {
                    fi.lb[t] = op.lb[t];
                    fi.gb[t] = op.gb[t];
                }
                for (int r = 0; r < 8; ++r) fi.perm[r] = op.perm[r];
                for (int t = 0; t < 4; ++t) fi.slot[t] = op.slot[t];
                for (int k = 0; k < 16; ++k) {
                    fi.c[2 * k] = op.cd[k].x;
                    fi.c[2 * k + 1] = op.cd[k].y;
                }
            }
            ++no;
        }
    }
    *n_passes = np;
    *n_fused = no;
    return SMOQ_OK;
}

smoq_status smoq_apply_sequence_unfused(smoq_state* st, const smoq_op* ops, int n, const double* theta) {
    if (check_state(st) || (!ops && n > 0) || n < 0) return SMOQ_ERR_BADINPUT;
    std::vector<GateIR> ir;
    if (smoq_status s = ops_to_ir(st, st->N, ops, n, theta, ir)) return s;
    for (const GateIR& g : ir)
        if (smoq_status s = apply_gate_ir(st, g)) return s;
    return SMOQ_OK;
}

// ============================================================= observables
static smoq_status fetch(smoq_ctx* ctx, const double* d, size_t n, double* host) {
    if (smoq_status s = ensure_pinned(ctx, n * sizeof(double))) return s;
    CK(ctx, cudaMemcpyAsync(ctx->h_pinned, d, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (smoq_status s = sync_check(ctx)) return s;
    std::memcpy(host, ctx->h_pinned, n * sizeof(double));
    return SMOQ_OK;
}

// out region for reductions lives after the partials in the scratch buffer
static smoq_status diag_reduce_host(smoq_state* st, const uint64_t* zmasks, int nobs, double* out) {
    smoq_ctx* ctx = st->ctx;
    const int per = 32;
    std::vector<double> all((size_t)st->batch * nobs);
    for (int o0 = 0; o0 < nobs; o0 += per) {
        const int k = std::min(per, nobs - o0);
        const size_t part = diag_reduce_scratch_doubles(st, k);
        const size_t outn = (size_t)st->batch * k;
        if (smoq_status s = ensure_scratch(ctx, part + outn)) return s;
        double* d_out = ctx->d_scratch + part;
        CK(ctx, launch_diag_reduce(ctx, st, zmasks + o0, k, d_out));
        std::vector<double> tmp(outn);
        if (smoq_status s = fetch(ctx, d_out, outn, tmp.data())) return s;
        for (int b = 0; b < st->batch; ++b)
            for (int j = 0; j < k; ++j) all[(size_t)b * nobs + o0 + j] = tmp[(size_t)b * k + j];
    }
    std::memcpy(out, all.data(), all.size() * sizeof(double));
    return SMOQ_OK;
}

static smoq_status pauli_reduce_host(smoq_state* st, uint64_t xmask, uint64_t zmask, int ny, double* out) {
    smoq_ctx* ctx = st->ctx;
    if (xmask == 0) return diag_reduce_host(st, &zmask, 1, out);
    const size_t part = diag_reduce_scratch_doubles(st, 1);
    const size_t outn = (size_t)st->batch;
    if (smoq_status s = ensure_scratch(ctx, part + outn)) return s;
    double* d_out = ctx->d_scratch + part;
    CK(ctx, launch_pauli_reduce(ctx, st, xmask, zmask, ny, d_out));
    return fetch(ctx, d_out, outn, out);
}

smoq_status smoq_expect_z(smoq_state* st, int q, double* out) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "expect_z")) return s;
    uint64_t m = 1ull << q;
    return diag_reduce_host(st, &m, 1, out);
}
smoq_status smoq_expect_x(smoq_state* st, int q, double* out) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "expect_x")) return s;
    return pauli_reduce_host(st, 1ull << q, 0, 0, out);
}
smoq_status smoq_expect_y(smoq_state* st, int q, double* out) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "expect_y")) return s;
    return pauli_reduce_host(st, 1ull << q, 1ull << q, 1, out);
}
static smoq_status corr(smoq_state* st, int a, int b, double* out, char p) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, a, "expect_corr")) return s;
    if (smoq_status s = check_q(st, b, "expect_corr")) return s;
    if (a == b) return fail(st->ctx, SMOQ_ERR_BADINPUT, "correlator qubits must differ");
    const uint64_t m = (1ull << a) | (1ull << b);
    if (p == 'z') return diag_reduce_host(st, &m, 1, out);
    if (p == 'x') return pauli_reduce_host(st, m, 0, 0, out);
    return pauli_reduce_host(st, m, m, 2, out);
}
smoq_status smoq_expect_xx(smoq_state* st, int a, int b, double* out) { return corr(st, a, b, out, 'x'); }
smoq_status smoq_expect_yy(smoq_state* st, int a, int b, double* out) { return corr(st, a, b, out, 'y'); }
smoq_status smoq_expect_zz(smoq_state* st, int a, int b, double* out) { return corr(st, a, b, out, 'z'); }

smoq_status smoq_expect_pauli_string(smoq_state* st, int n, const char* ops, const int* qubits, double* out) {
    if (check_state(st) || !out || n < 0 || (n > 0 && (!ops || !qubits))) return SMOQ_ERR_BADINPUT;
    uint64_t x = 0, z = 0, seen = 0;
    int ny = 0;
    for (int t = 0; t < n; ++t) {
        if (smoq_status s = check_q(st, qubits[t], "pauli_string")) return s;
        const uint64_t b = 1ull << qubits[t];
        if (seen & b) return fail(st->ctx, SMOQ_ERR_BADINPUT, "qubits must be unique");
        seen |= b;
        switch (ops[t]) {
            case 'X': case 'x': x |= b; break;
            case 'Y': case 'y': x |= b; z |= b; ny++; break;
            case 'Z': case 'z': z |= b; break;
            default: return fail(st->ctx, SMOQ_ERR_BADINPUT, "pauli letters must be X, Y or Z");
        }
    }
    return pauli_reduce_host(st, x, z, ny, out);
}

smoq_status smoq_expect_zstrings(smoq_state* st, const uint64_t* zmasks, int nobs, double* out) {
    if (check_state(st) || !out || !zmasks || nobs < 1) return SMOQ_ERR_BADINPUT;
    const uint64_t lim = st->N >= 64 ? ~0ull : ((1ull << st->N) - 1);
    for (int o = 0; o < nobs; ++o)
        if (zmasks[o] & ~lim) return fail(st->ctx, SMOQ_ERR_BADINPUT, "zmask has bits beyond N");
    return diag_reduce_host(st, zmasks, nobs, out);
}

smoq_status smoq_measure_all_observables(smoq_state* st, int L, int n_rails, double* out) {
    if (check_state(st) || !out || L < 1 || n_rails < 1) return SMOQ_ERR_BADINPUT;
    const int N = L * n_rails;
    if (N != st->N) return fail(st->ctx, SMOQ_ERR_BADINPUT, "L * n_rails must equal the state's N");
    // the reference's order: (X, Y, Z) per qubit, then (XX, YY, ZZ) per rail bond, then per rung
    struct Obs { uint64_t x, z; int ny; };
    std::vector<Obs> obs;
    for (int k = 0; k < N; ++k) {
        const uint64_t b = 1ull << k;
        obs.push_back({b, 0, 0});
        obs.push_back({b, b, 1});
        obs.push_back({0, b, 0});
    }
    auto pair = [&](int i, int j) {
        const uint64_t m = (1ull << i) | (1ull << j);
        obs.push_back({m, 0, 0});
        obs.push_back({m, m, 2});
        obs.push_back({0, m, 0});
    };
    for (int r = 0; r < n_rails; ++r)
        for (int s = 0; s < L - 1; ++s) pair(r * L + s, r * L + s + 1);
    for (int r = 0; r < n_rails - 1; ++r)
        for (int s = 0; s < L; ++s) pair(r * L + s, (r + 1) * L + s);
    const int nops = (int)obs.size();
    const int B = st->batch;
    // diagonal ones (Z, ZZ) in Z-string reductions of up to 32 masks, the others one by one
    std::vector<int> zi;
    for (int o = 0; o < nops; ++o)
        if (!obs[o].x) zi.push_back(o);
    std::vector<double> v;
    for (size_t a = 0; a < zi.size(); a += 32) {
        const int k = (int)std::min<size_t>(32, zi.size() - a);
        std::vector<uint64_t> m(k);
        for (int t = 0; t < k; ++t) m[t] = obs[zi[a + t]].z;
        v.assign((size_t)B * k, 0.0);
        if (smoq_status s = diag_reduce_host(st, m.data(), k, v.data())) return s;
        for (int b = 0; b < B; ++b)
            for (int t = 0; t < k; ++t) out[(size_t)b * nops + zi[a + t]] = v[(size_t)b * k + t];
    }
    v.assign(B, 0.0);
    for (int o = 0; o < nops; ++o) {
        if (!obs[o].x) continue;
        if (smoq_status s = pauli_reduce_host(st, obs[o].x, obs[o].z, obs[o].ny, v.data())) return s;
        for (int b = 0; b < B; ++b) out[(size_t)b * nops + o] = v[b];
    }
    return SMOQ_OK;
}

smoq_status smoq_population_excited(smoq_state* st, int q, double* out) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    if (smoq_status s = check_q(st, q, "population_excited")) return s;
    uint64_t m[2] = {0, 1ull << q};
    std::vector<double> v((size_t)st->batch * 2);
    if (smoq_status s = diag_reduce_host(st, m, 2, v.data())) return s;
    for (int b = 0; b < st->batch; ++b) out[b] = 0.5 * (v[2 * b] - v[2 * b + 1]);
    return SMOQ_OK;
}

smoq_status smoq_norm2(smoq_state* st, double* out) {
    if (check_state(st) || !out) return SMOQ_ERR_BADINPUT;
    uint64_t m = 0;
    return diag_reduce_host(st, &m, 1, out);
}

smoq_status smoq_normalize(smoq_state* st) {
    if (check_state(st)) return SMOQ_ERR_BADINPUT;
    smoq_ctx* ctx = st->ctx;
    std::vector<double> n2(st->batch);
    if (smoq_status s = smoq_norm2(st, n2.data())) return s;
    for (int b = 0; b < st->batch; ++b) {
        if (!(n2[b] > 0)) return fail(ctx, SMOQ_ERR_BADINPUT, "Cannot normalize zero vector");
        n2[b] = 1.0 / std::sqrt(n2[b]);
    }
    double* d = nullptr;
    CK(ctx, cudaMallocAsync((void**)&d, n2.size() * sizeof(double), ctx->stream));
    CK(ctx, cudaMemcpyAsync(d, n2.data(), n2.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, launch_scale(st, d, 1.0));
    CK(ctx, cudaFreeAsync(d, ctx->stream));
    return sync_check(ctx);
}

}  // extern "C"

// ================================================================== plans
struct smoq_plan {
    smoq_ctx* ctx = nullptr;
    int N = 0;
    int dtype = SMOQ_C64;
    int order = 1;
    std::vector<GateIR> step;  // gates of one step (order 2: list + reversed list)
    // the fused-pass geometry of the plan's blocks: tile width, low bits and the
    // fusion depth (max fused ops per pass, 0 = as many as fit); the context's
    // defaults, or the autotuner's choice made when the first block is built
    int tbits = 0, lbits = 0, max_ops = 0;
    bool geometry_chosen = false;
    struct Block {
        DevProgram prog;
        cudaGraphExec_t gexec = nullptr;
        void* gptr = nullptr;
        int gbatch = 0;
        long long kernels = 0;
        ~Block() {
            if (gexec) cudaGraphExecDestroy(gexec);
        }
    };
    std::map<int, std::unique_ptr<Block>> blocks;  // keyed by steps per block
};

static smoq_status choose_geometry(smoq_plan* P, const std::vector<GateIR>& all);

static smoq_status get_block(smoq_plan* P, int nsteps, smoq_plan::Block** out) {
    auto it = P->blocks.find(nsteps);
    if (it != P->blocks.end()) {
        *out = it->second.get();
        return SMOQ_OK;
    }
    std::unique_ptr<smoq_plan::Block> B(new smoq_plan::Block());
    std::vector<GateIR> all;
    all.reserve(P->step.size() * nsteps);
    for (int s = 0; s < nsteps; ++s) all.insert(all.end(), P->step.begin(), P->step.end());
    if (!P->geometry_chosen) {
        P->tbits = tile_bits(P->ctx, P->dtype);
        P->lbits = low_bits(P->ctx, P->dtype);
        P->max_ops = P->ctx->fusion_depth;
        if (smoq_status s = choose_geometry(P, all)) return s;
        P->geometry_chosen = true;
    }
    try {
        B->prog.passes = plan_for(engine_for(P->ctx, true, P->dtype), all, P->N, P->dtype, P->tbits, P->lbits, -1,
                                  P->max_ops);
    } catch (const std::exception& ex) {
        return fail(P->ctx, SMOQ_ERR_BADINPUT, ex.what());
    }
    if (smoq_status s = upload_program(P->ctx, B->prog)) return s;
    if (P->ctx->autotune && P->dtype == SMOQ_C64)
        if (smoq_status s = autotune_program(P->ctx, B->prog, P->N)) return s;
    for (auto& p : B->prog.passes)
        if (!p.ops.empty()) B->kernels++;
    *out = B.get();
    P->blocks[nsteps] = std::move(B);
    return SMOQ_OK;
}

// Plan-level autotuning (reusable complex64 programs of N >= 20 on the compiled
// pass kernels, when SMOQ_OPT_AUTOTUNE is on): the block is planned with each
// candidate geometry -- tile width, low bits, fusion depth -- compiled, and run
// once on a zeroed scratch state; the fastest geometry is kept for every block of
// the plan and cached per (GPU, N, gate pattern).  The first candidate is the
// default: another one replaces it only when it is faster by more than
// kGeometryMargin (one timed run per candidate: smaller differences are noise).
// Every candidate computes the same evolution (fusion regroups the same gates).
namespace {
struct PlanGeometry {
    int tbits, lbits, max_ops;
};
const PlanGeometry kGeometries[] = {{13, 5, 0}, {13, 4, 0}, {12, 5, 0}, {12, 4, 0}, {13, 5, 12}};
constexpr float kGeometryMargin = 0.02f;

// the candidate kept: the fastest, unless the default (candidate 0) is within the
// margin of it; ms[c] < 0: candidate c could not be planned (-1: none could)
int pick_geometry(const float* ms, int n) {
    int best = -1;
    for (int c = 0; c < n; ++c)
        if (ms[c] >= 0 && (best < 0 || ms[c] < ms[best])) best = c;
    if (best > 0 && ms[0] >= 0 && ms[best] > (1.0f - kGeometryMargin) * ms[0]) best = 0;
    return best;
}
std::map<uint64_t, int> g_geometry;  // guarded by g_tune_mu
}  // namespace

static smoq_status choose_geometry(smoq_plan* P, const std::vector<GateIR>& all) {
    smoq_ctx* ctx = P->ctx;
    if (!ctx->autotune || !ctx->tune_geometry || P->dtype != SMOQ_C64 || P->N < kTuneMinN ||
        engine_for(ctx, true, P->dtype) != 3)
        return SMOQ_OK;
    // key: device, N and the gate pattern (qubits, diagonal or not) of the block
    uint64_t key = device_hash(ctx->device) ^ 0x9E3779B97F4A7C15ull;
    auto mix = [&key](uint64_t v) { key = (key ^ v) * 1099511628211ull; };
    mix((uint64_t)P->N);
    for (const GateIR& g : all) {
        mix((uint64_t)g.nq | ((uint64_t)g.diag << 8));
        for (int t = 0; t < g.nq; ++t) mix((uint64_t)g.q[t]);
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_cache_load_locked();
        auto it = g_geometry.find(key);
        if (it == g_geometry.end()) {
            auto jt = g_tune.find(key);  // geometry choices share the cache file (key, candidate index)
            if (jt != g_tune.end()) it = g_geometry.emplace(key, jt->second).first;
        }
        if (it != g_geometry.end() && it->second >= 0 && it->second < (int)(sizeof(kGeometries) / sizeof(kGeometries[0]))) {
            const PlanGeometry& G = kGeometries[it->second];
            P->tbits = G.tbits, P->lbits = G.lbits, P->max_ops = G.max_ops;
            return SMOQ_OK;
        }
    }
    const size_t bytes = (size_t)8 << P->N;
    size_t free_b = 0, total_b = 0;
    CK(ctx, cudaMemGetInfo(&free_b, &total_b));
    if (free_b < 2 * bytes + ((size_t)1 << 30)) {
        ctx->tune_report += "geometry tuning skipped: no room for a scratch state\n";
        return SMOQ_OK;
    }
    void* scratch = nullptr;
    CK(ctx, cudaMallocAsync(&scratch, bytes, ctx->stream));
    std::unique_ptr<void, std::function<void(void*)>> hold(scratch, [ctx](void* q) { cudaFreeAsync(q, ctx->stream); });
    CK(ctx, cudaMemsetAsync(scratch, 0, bytes, ctx->stream));
    smoq_state st;
    st.ctx = ctx;
    st.N = P->N;
    st.dtype = SMOQ_C64;
    st.batch = 1;
    st.ptr = scratch;
    st.owned = false;
    cudaEvent_t e0, e1;
    CK(ctx, cudaEventCreate(&e0));
    CK(ctx, cudaEventCreate(&e1));
    std::ostringstream rep;
    constexpr int ng = (int)(sizeof(kGeometries) / sizeof(kGeometries[0]));
    float times[ng];
    for (int c = 0; c < ng; ++c) times[c] = -1.0f;
    const long long launches0 = ctx->launches, passes0 = ctx->tile_passes;
    for (int c = 0; c < ng; ++c) {
        const PlanGeometry& G = kGeometries[c];
        DevProgram prog;
        try {
            prog.passes = plan_for(3, all, P->N, P->dtype, G.tbits, G.lbits, -1, G.max_ops);
        } catch (const std::exception&) {
            continue;  // a geometry the planner cannot use for this circuit
        }
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        if (upload_program(ctx, prog) != SMOQ_OK) continue;
        smoq_status s = run_program(ctx, &st, prog, nullptr, nullptr);  // warm-up
        cudaEventRecord(e0, ctx->stream);
        if (!s) s = run_program(ctx, &st, prog, nullptr, nullptr);
        cudaEventRecord(e1, ctx->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (s || e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return s ? s : cuda_fail(ctx, e, "geometry tuning");
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        rep << "geometry tile " << G.tbits << " low " << G.lbits << " depth " << (G.max_ops ? G.max_ops : -1) << ": "
            << prog.passes.size() << " passes, " << ms << " ms\n";
        times[c] = ms;
    }
    const int best = pick_geometry(times, ng);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches = launches0;  // the tuning runs are not the caller's work
    ctx->tile_passes = passes0;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (best >= 0) {
        const PlanGeometry& G = kGeometries[best];
        P->tbits = G.tbits, P->lbits = G.lbits, P->max_ops = G.max_ops;
        rep << "-> geometry tile " << G.tbits << " low " << G.lbits << " depth " << (G.max_ops ? G.max_ops : -1) << "\n";
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_geometry[key] = best;
        tune_cache_store_locked(key, best);
    }
    ctx->tune_report += rep.str();
    return sync_check(ctx);
}

static smoq_status run_block(smoq_plan* P, smoq_state* st, smoq_plan::Block* B, std::vector<EventPair>* timing) {
    smoq_ctx* ctx = P->ctx;
    if (ctx->use_graphs && !timing) {
        if (!B->gexec || B->gptr != st->ptr || B->gbatch != st->batch) {
            if (B->gexec) cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
            cudaGraph_t g;
            CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            smoq_status s = run_program(ctx, st, B->prog, nullptr, nullptr);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (s) return s;
            if (e != cudaSuccess) return cuda_fail(ctx, e, "graph capture");
            e = cudaGraphInstantiate(&B->gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "graph instantiate");
            B->gptr = st->ptr;
            B->gbatch = st->batch;
            // capture counted launches that did not run
            ctx->launches -= B->kernels;
            ctx->tile_passes -= B->kernels;
        }
        CK(ctx, cudaGraphLaunch(B->gexec, ctx->stream));
        ctx->launches += B->kernels;
        ctx->tile_passes += B->kernels;
        return SMOQ_OK;
    }
    return run_program(ctx, st, B->prog, nullptr, timing);
}

extern "C" {

smoq_status smoq_precompute_trotter_gates(const double* bonds, int nb, const double* fields, int nf, double dt,
                                          smoq_trotter_gate* out, int* n_out) {
    // exp(-i dt (Jx XX + Jy YY + Jz ZZ)) is block diagonal on {00,11} and
    // {01,10} because XX, YY, ZZ commute: even block e^{-i Jz dt} exp(-i (Jx-Jy) dt sx),
    // odd block e^{+i Jz dt} exp(-i (Jx+Jy) dt sx); fields: exp(-i dt h.sigma)
    // = cos(|h| dt) I - i sin(|h| dt) h.sigma/|h|.
    if ((nb > 0 && !bonds) || (nf > 0 && !fields) || !out || !n_out) return SMOQ_ERR_BADINPUT;
    int n = 0;
    auto put = [](double* U, int dim, int r, int c, cd v) {
        U[2 * (c * dim + r)] = v.real();
        U[2 * (c * dim + r) + 1] = v.imag();
    };
    for (int t = 0; t < nb; ++t) {
        const double* b = bonds + 5 * t;
        smoq_trotter_gate& g = out[n++];
        std::memset(&g, 0, sizeof(g));
        g.nq = 2;
        g.q[0] = (int)b[0];
        g.q[1] = (int)b[1];
        const double a = (b[2] - b[3]) * dt, bb = (b[2] + b[3]) * dt;
        const cd pe = std::exp(cd(0, -b[4] * dt)), po = std::exp(cd(0, b[4] * dt));
        put(g.U, 4, 0, 0, pe * std::cos(a));
        put(g.U, 4, 3, 3, pe * std::cos(a));
        put(g.U, 4, 0, 3, pe * cd(0, -std::sin(a)));
        put(g.U, 4, 3, 0, pe * cd(0, -std::sin(a)));
        put(g.U, 4, 1, 1, po * std::cos(bb));
        put(g.U, 4, 2, 2, po * std::cos(bb));
        put(g.U, 4, 1, 2, po * cd(0, -std::sin(bb)));
        put(g.U, 4, 2, 1, po * cd(0, -std::sin(bb)));
    }
    for (int t = 0; t < nf; ++t) {
        const double* f = fields + 4 * t;
        const double hx = f[1], hy = f[2], hz = f[3];
        if (!(std::fabs(hx) > 1e-14 || std::fabs(hy) > 1e-14 || std::fabs(hz) > 1e-14)) continue;
        const double h = std::sqrt(hx * hx + hy * hy + hz * hz), c = std::cos(h * dt), s = std::sin(h * dt) / h;
        smoq_trotter_gate& g = out[n++];
        std::memset(&g, 0, sizeof(g));
        g.nq = 1;
        g.q[0] = (int)f[0];
        put(g.U, 2, 0, 0, cd(c, -s * hz));
        put(g.U, 2, 1, 1, cd(c, s * hz));
        put(g.U, 2, 0, 1, cd(0, -s) * cd(hx, -hy));
        put(g.U, 2, 1, 0, cd(0, -s) * cd(hx, hy));
    }
    *n_out = n;
    return SMOQ_OK;
}

smoq_status smoq_trotter_plan_create(smoq_ctx* ctx, int N, smoq_dtype dtype, const smoq_trotter_gate* gates, int n,
                                     int order, smoq_plan** out) {
    if (!ctx || !out || (n > 0 && !gates) || n < 0) return SMOQ_ERR_BADINPUT;
    if (order != 1 && order != 2) return fail(ctx, SMOQ_ERR_BADINPUT, "order must be 1 or 2");
    if (N < 1 || N > 40) return fail(ctx, SMOQ_ERR_BADINPUT, "N must be in 1..40");
    std::unique_ptr<smoq_plan> P(new smoq_plan());
    P->ctx = ctx;
    P->N = N;
    P->dtype = dtype;
    P->order = order;
    std::vector<GateIR> one;
    for (int i = 0; i < n; ++i) {
        const smoq_trotter_gate& g = gates[i];
        if (g.nq == 1) {
            if (g.q[0] < 0 || g.q[0] >= N) return fail(ctx, SMOQ_ERR_BADINPUT, "trotter gate qubit out of range");
            cd m[4];
            load_colmajor(g.U, 2, m);
            one.push_back(gate_1q(g.q[0], m));
        } else if (g.nq == 2) {
            if (g.q[0] < 0 || g.q[0] >= N || g.q[1] < 0 || g.q[1] >= N || g.q[0] == g.q[1])
                return fail(ctx, SMOQ_ERR_BADINPUT, "trotter gate qubits out of range");
            one.push_back(u2_gate(g.q[0], g.q[1], g.U, 0));
        } else {
            return fail(ctx, SMOQ_ERR_BADINPUT, "Gates with more than 2 qubits not supported");  // Trotter.jl:157
        }
    }
    P->step = one;
    if (order == 2) P->step.insert(P->step.end(), one.rbegin(), one.rend());
    *out = P.release();
    return SMOQ_OK;
}

smoq_status smoq_plan_destroy(smoq_plan* plan) {
    if (!plan) return SMOQ_ERR_BADINPUT;
    cudaStreamSynchronize(plan->ctx->stream);
    delete plan;
    return SMOQ_OK;
}

static const int kMaxBlockSteps = 10;

static smoq_status trotter_steps(smoq_plan* P, smoq_state* st, int n_steps, std::vector<EventPair>* timing) {
    while (n_steps > 0) {
        const int k = std::min(n_steps, kMaxBlockSteps);
        smoq_plan::Block* B = nullptr;
        if (smoq_status s = get_block(P, k, &B)) return s;
        if (smoq_status s = run_block(P, st, B, timing)) return s;
        n_steps -= k;
    }
    return SMOQ_OK;
}

static smoq_status check_plan_state(smoq_plan* P, smoq_state* st) {
    if (!P || check_state(st)) return SMOQ_ERR_BADINPUT;
    if (st->N != P->N || st->dtype != P->dtype) return fail(P->ctx, SMOQ_ERR_BADINPUT, "plan/state shape mismatch");
    if (st->ctx != P->ctx) return fail(P->ctx, SMOQ_ERR_BADINPUT, "plan and state belong to different contexts");
    return SMOQ_OK;
}

smoq_status smoq_trotter_step(smoq_plan* P, smoq_state* st, int n_steps) {
    if (smoq_status s = check_plan_state(P, st)) return s;
    if (n_steps < 0) return fail(P->ctx, SMOQ_ERR_BADINPUT, "n_steps < 0");
    std::vector<EventPair> timing;
    smoq_status s = trotter_steps(P, st, n_steps, P->ctx->kernel_timing ? &timing : nullptr);
    if (!timing.empty()) harvest_timing(P->ctx, timing);
    return s;
}

smoq_status smoq_trotter_run(smoq_plan* P, smoq_state* st, int steps, int record_every, double* z_out) {
    if (smoq_status s = check_plan_state(P, st)) return s;
    smoq_ctx* ctx = P->ctx;
    if (steps < 0 || record_every < 1 || !z_out) return fail(ctx, SMOQ_ERR_BADINPUT, "bad steps/record_every/z_out");
    const int N = P->N;
    const int nrec = steps / record_every + 1;
    const size_t per_rec = (size_t)st->batch * N;
    std::vector<uint64_t> zm(N);
    for (int i = 0; i < N; ++i) zm[i] = 1ull << i;
    // device record buffer, then the reduction partials
    const int per = 32;
    const size_t part = diag_reduce_scratch_doubles(st, std::min(N, per));
    if (smoq_status s = ensure_scratch(ctx, part + nrec * per_rec + (size_t)st->batch * per)) return s;
    double* d_rec = ctx->d_scratch + part;
    double* d_tmp = d_rec + nrec * per_rec;
    std::vector<EventPair> timing;
    std::vector<EventPair>* tp = ctx->kernel_timing ? &timing : nullptr;
    auto record = [&](int r) -> smoq_status {
        // <Z_i> of every state into d_rec[r][b][i]: 32 observables per reduction
        if (N <= per) {  // [b][i] layout straight into the record slot
            cudaError_t e = launch_diag_reduce(ctx, st, zm.data(), N, d_rec + r * per_rec);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "record reduction");
            return SMOQ_OK;
        }
        for (int o0 = 0; o0 < N; o0 += per) {
            const int k = std::min(per, N - o0);
            cudaError_t e = launch_diag_reduce(ctx, st, zm.data() + o0, k, d_tmp);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "record reduction");
            for (int b = 0; b < st->batch; ++b) {
                e = cudaMemcpyAsync(d_rec + r * per_rec + (size_t)b * N + o0, d_tmp + (size_t)b * k,
                                    k * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "record copy");
            }
        }
        return SMOQ_OK;
    };
    if (smoq_status s = record(0)) return s;
    int done = 0;
    for (int r = 1; r < nrec; ++r) {
        if (smoq_status s = trotter_steps(P, st, record_every, tp)) return s;
        done += record_every;
        if (smoq_status s = record(r)) return s;
    }
    if (steps > done)
        if (smoq_status s = trotter_steps(P, st, steps - done, tp)) return s;
    if (smoq_status s = fetch(ctx, d_rec, nrec * per_rec, z_out)) return s;
    harvest_timing(ctx, timing);
    return SMOQ_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Internal entry points shared with the other translation units (MCWF, VQE).
// ------------------------------------------------------------------------
smoq_status smoq_internal_fail(smoq_ctx* ctx, smoq_status s, const char* msg) { return fail(ctx, s, msg); }
smoq_status smoq_internal_cuda(smoq_ctx* ctx, cudaError_t e, const char* where) { return cuda_fail(ctx, e, where); }

smoq_status smoq_internal_plan_step(smoq_plan* plan, std::vector<GateIR>& out, int& N, int& dtype, int& order) {
    out = plan->step;
    N = plan->N;
    dtype = plan->dtype;
    order = plan->order;
    return SMOQ_OK;
}

// plan + upload a gate program for `st` (no launch); the handle owns it
// the passes of a one-use gate program (host only: reads the context's options,
// touches nothing else, so a planning thread may call it); throws on bad input.
// variational: a variational circuit's complex64 forward, compiled kernels with
// run-time coefficients
std::vector<Pass> smoq_internal_plan(smoq_ctx* ctx, int N, int dtype, const std::vector<GateIR>& gates,
                                     bool variational) {
    const bool rtc = variational && dtype == SMOQ_C64 && ctx->engine < 0 && jit_available();
    return plan_for(rtc ? 3 : engine_for(ctx, false, dtype), gates, N, dtype, tile_bits(ctx, dtype),
                    low_bits(ctx, dtype), -1, ctx->fusion_depth, rtc);
}

void smoq_internal_cap_fusion_depth(std::vector<Pass>& pl, int cap) { cap_fusion_depth(pl, cap); }

// upload planned passes (kernels resolved, ops on the device); the handle owns them
smoq_status smoq_internal_prepare_planned(smoq_ctx* ctx, std::vector<Pass>&& passes, void** handle) {
    std::unique_ptr<DevProgram> P(new DevProgram());
    P->passes = std::move(passes);
    if (smoq_status s = upload_program(ctx, *P)) return s;
    *handle = P.release();
    return SMOQ_OK;
}

smoq_status smoq_internal_prepare(smoq_ctx* ctx, smoq_state* st, const std::vector<GateIR>& gates,
                                  int epilogue_special, bool reusable, void** handle, bool variational) {
    std::unique_ptr<DevProgram> P(new DevProgram());
    // a variational circuit's complex64 forward: compiled kernels with run-time coefficients
    const bool rtc = variational && st->dtype == SMOQ_C64 && ctx->engine < 0 && jit_available();
    try {
        P->passes = plan_for(rtc ? 3 : engine_for(ctx, reusable, st->dtype), gates, st->N, st->dtype,
                             tile_bits(ctx, st->dtype), low_bits(ctx, st->dtype), epilogue_special, 0, rtc);
    } catch (const std::exception& ex) {
        return fail(ctx, SMOQ_ERR_BADINPUT, ex.what());
    }
    if (smoq_status s = upload_program(ctx, *P)) return s;
    *handle = P.release();
    return SMOQ_OK;
}

smoq_status smoq_internal_rerun(smoq_ctx* ctx, smoq_state* st, void* handle, const Epilogue* ep) {
    return run_program(ctx, st, *(DevProgram*)handle, ep, nullptr);
}

void smoq_internal_free_prog(void* handle) { delete (DevProgram*)handle; }

// tiles per state of the pass that carries the epilogue (else of the last pass)
int64_t smoq_internal_tiles_per_state(void* handle) {
    const DevProgram* P = (const DevProgram*)handle;
    for (const Pass& p : P->passes)
        if (p.epilogue) return (int64_t)1 << (p.g.N - p.g.T);
    return P->passes.empty() ? 1 : (int64_t)1 << (P->passes.back().g.N - P->passes.back().g.T);
}

// up to 32 Z-string sums of every state into d_out[b * nobs + o] (device)
smoq_status smoq_internal_zreduce(smoq_ctx* ctx, smoq_state* st, const uint64_t* zmasks, int nobs, double* d_out) {
    if (nobs < 1 || nobs > 32) return fail(ctx, SMOQ_ERR_BADINPUT, "at most 32 observables per reduction");
    if (smoq_status s = ensure_scratch(ctx, diag_reduce_scratch_doubles(st, nobs))) return s;
    CK(ctx, launch_diag_reduce(ctx, st, zmasks, nobs, d_out));
    return SMOQ_OK;
}

smoq_status smoq_internal_ops_to_ir(int N, const smoq_op* ops, int n, const double* theta, std::vector<GateIR>& out) {
    return ops_to_ir(nullptr, N, ops, n, theta, out);
}
int smoq_internal_tile_bits(smoq_ctx* ctx, int dtype) { return tile_bits(ctx, dtype); }
smoq_status smoq_internal_plan_step(smoq_plan* P, smoq_ctx** ctx, int* N, int* dtype, const std::vector<GateIR>** step) {
    if (!P || !P->ctx) return SMOQ_ERR_BADINPUT;
    *ctx = P->ctx;
    *N = P->N;
    *dtype = P->dtype;
    *step = &P->step;
    return SMOQ_OK;
}
int smoq_internal_low_bits(smoq_ctx* ctx, int dtype) { return low_bits(ctx, dtype); }

// host-only view of the geometry rule (pick_geometry)
extern "C" int smoq_debug_pick_geometry(const float* ms, int n) {
    if (!ms || n < 1 || n > 64) return -1;
    return pick_geometry(ms, n);
}

// noalloc.cu -- a Z-string expectation batch that allocates nothing.
//
// Who needs this: callers that may not allocate device memory when they call
// in.  Examples are a host application that hands the library fixed,
// pre-sized buffers and must keep its GPU footprint constant (a memory arena
// or a caller that already holds nearly all of HBM), code running where
// cudaMalloc/cudaFree would synchronise the device or wait on the allocator
// (callbacks, latency-bound control loops), and callers with no smoq_ctx at
// all (creating one allocates).  smoq_expect_zstrings needs a context whose
// scratch buffer grows with cudaMalloc; this variant takes the state and the
// output as caller-owned device pointers and keeps its per-block partial sums
// in a fixed array compiled into the library.
//
// The fixed array, g_noalloc_partials, holds kNoAllocMaxPartials doubles
// (512 KiB).  Every GPU that loads the library holds it until the process
// exits.  In host code the name g_noalloc_partials is only a host-side
// stand-in for the device array, not a device address: passing it to a
// kernel would fault or (where the GPU can reach host memory) silently use
// the wrong memory.  So, once per device and with that device current, the
// host looks up the array's device address with cudaGetSymbolAddress and
// passes that address to the kernels.  The lookup happens inside the first
// call made on each device; make that first call before any stream capture
// starts, because the lookup can load the library's device code.  The
// address is remembered together with the CUDA context that was current
// when it was looked up: after cudaDeviceReset the runtime makes a new
// primary context, the library's device code is loaded again (possibly at
// another address), and the next call sees the new context and looks the
// address up again instead of reusing the stale one.
//
// All calls on one device share the array.  Every slot the finishing kernel
// reads is written by the first kernel of the same call, so nothing carries
// over from an earlier call and nothing has to be cleared to zero; but two
// calls whose kernels can run at the same time on one device (different
// streams, or different host threads) race on the array and can return wrong
// values.  Issue such calls on one stream.
#include <cuda_runtime.h>
#include <stdio.h>
#include <mutex>
#include "k_common.cuh"

namespace {

constexpr int kNoAllocMaxPartials = 1 << 16;  // doubles (512 KiB) per GPU
constexpr int kNoAllocMaxObs = 32;
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxPartials];

std::mutex g_setup_mu;
// per device: the scratch array's device address and the CUDA context it
// belongs to (the address is only valid in that context)
double* g_partials_addr[kMaxDevices] = {};
void* g_partials_ctx[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry-point table (the library
// does not link libcuda itself); null when the driver does not provide it
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return fn;
}
void* current_context() {
    void* c = nullptr;
    if (CtxGetCurrentFn f = ctx_get_current())
        if (f(&c) != 0) c = nullptr;
    return c;
}

struct NoAllocMasks {
    uint64_t m[kNoAllocMaxObs];
};

// partials[(b * nblk + blk) * nobs + o] = this block's sum of
// |psi_i|^2 (-1)^{popc(i & zmask_o)} over state b, in FP64
template <typename R>
__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_partials_kernel(const typename smoq::CT<R>::T* psi, int N, NoAllocMasks zm, int nobs, double* partials) {
    const int64_t len = (int64_t)1 << N;
    const int64_t b = blockIdx.y;
    const int nblk = gridDim.x;
    const typename smoq::CT<R>::T* s = psi + b * len;
    double acc[kNoAllocMaxObs];
#pragma unroll
    for (int o = 0; o < kNoAllocMaxObs; ++o) acc[o] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)nblk * blockDim.x) {
        const double p = smoq::cabs2d(s[i]);
#pragma unroll
        for (int o = 0; o < kNoAllocMaxObs; ++o)
            if (o < nobs) acc[o] += (__popcll((uint64_t)i & zm.m[o]) & 1) ? -p : p;
    }
    __shared__ double red[kNoAllocThreads / 32][kNoAllocMaxObs];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < kNoAllocMaxObs; ++o) {
        if (o < nobs) {
            double x = acc[o];
            for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
            if (lane == 0) red[w][o] = x;
        }
    }
    __syncthreads();
    if (threadIdx.x < nobs) {
        double x = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) x += red[k][threadIdx.x];
        partials[((size_t)b * nblk + blockIdx.x) * nobs + threadIdx.x] = x;
    }
}

// out[b * nobs + o] = sum over blocks in a fixed order (deterministic)
__global__ void noalloc_finish_kernel(const double* partials, int64_t B, int nblk, int nobs, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * nobs) return;
    const int64_t b = i / nobs, o = i - b * nobs;
    double s = 0;
    for (int k = 0; k < nblk; ++k) s += partials[((size_t)b * nblk + k) * nobs + o];
    out[i] = s;
}

smoq_status reject(char* errbuf, size_t errlen, smoq_status s, const char* msg) {
    if (errbuf && errlen) snprintf(errbuf, errlen, "smoq_expect_zstrings_noalloc: %s", msg);
    return s;
}

}  // namespace

extern "C" smoq_status smoq_expect_zstrings_noalloc(const void* psi, int N, smoq_dtype dtype, int batch,
                                                     const uint64_t* zmasks, int nobs, double* out, void* stream,
                                                     char* errbuf, size_t errlen) {
    if (errbuf && errlen) errbuf[0] = '\0';
    if (!psi || !out || !zmasks) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "null pointer argument");
    if (((uintptr_t)psi & 15) != 0) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "psi must be 16-byte aligned");
    if (dtype != SMOQ_C64 && dtype != SMOQ_C128) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "bad dtype");
    if (N < 1 || N > 40) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "N must be in 1..40");
    if (batch < 1 || batch > 65535) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "batch must be in 1..65535");
    if (nobs < 1 || nobs > kNoAllocMaxObs)
        return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "nobs must be in 1..32 per call");
    if ((int64_t)batch * nobs > kNoAllocMaxPartials)
        return reject(errbuf, errlen, SMOQ_ERR_BADINPUT,
                      "batch * nobs exceeds the fixed scratch of 65536 partial sums");
    const uint64_t lim = N >= 64 ? ~0ull : ((1ull << N) - 1);
    NoAllocMasks zm;
    for (int o = 0; o < kNoAllocMaxObs; ++o) {
        zm.m[o] = o < nobs ? zmasks[o] : 0;
        if (o < nobs && (zmasks[o] & ~lim)) return reject(errbuf, errlen, SMOQ_ERR_BADINPUT, "zmask has bits beyond N");
    }

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return reject(errbuf, errlen, SMOQ_ERR_NOGPU, "no current CUDA device");
    if (dev < 0 || dev >= kMaxDevices) return reject(errbuf, errlen, SMOQ_ERR_UNSUPPORTED, "device index too large");
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        // set-up, once per device (and again if that device's context changed,
        // e.g. after cudaDeviceReset), with that device current
        void* cur = current_context();
        if (!g_partials_addr[dev] || !cur || cur != g_partials_ctx[dev]) {
            double* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_partials);
            if (e != cudaSuccess || !p) {
                if (errbuf && errlen)
                    snprintf(errbuf, errlen, "smoq_expect_zstrings_noalloc: cudaGetSymbolAddress failed: %s",
                             cudaGetErrorString(e));
                return SMOQ_ERR_CUDA;
            }
            g_partials_addr[dev] = p;
            // the lookup made the primary context current if nothing was; a null
            // context here (no driver entry point) leaves the address un-cached,
            // so every call looks it up again
            g_partials_ctx[dev] = current_context();
        }
        partials = g_partials_addr[dev];
    }

    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t len = (int64_t)1 << N;
    int64_t nblk = (len + kNoAllocThreads * 8 - 1) / (kNoAllocThreads * 8);
    int64_t cap = ((int64_t)sms * 4 + batch - 1) / batch;
    if (nblk > cap) nblk = cap;
    const int64_t fit = kNoAllocMaxPartials / ((int64_t)batch * nobs);  // >= 1 by the check above
    if (nblk > fit) nblk = fit;
    if (nblk < 1) nblk = 1;

    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid((unsigned)nblk, (unsigned)batch);
    if (dtype == SMOQ_C64)
        noalloc_partials_kernel<float><<<grid, kNoAllocThreads, 0, s>>>((const float2*)psi, N, zm, nobs, partials);
    else
        noalloc_partials_kernel<double><<<grid, kNoAllocThreads, 0, s>>>((const double2*)psi, N, zm, nobs, partials);
    const int64_t outs = (int64_t)batch * nobs;
    noalloc_finish_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, s>>>(partials, batch, (int)nblk, nobs, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "smoq_expect_zstrings_noalloc: launch failed: %s", cudaGetErrorString(e));
        return SMOQ_ERR_CUDA;
    }
    return SMOQ_OK;
}

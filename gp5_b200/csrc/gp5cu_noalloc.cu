// gp5cu_noalloc.cu - gp5cu_norm_noalloc: the field norm without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they need a norm, e.g. a
// host that keeps its fields in memory handed out by another allocator and forbids the
// library from allocating, or a monitoring hook that runs while the device is full.  The
// plan-based gp5cu_norm needs a plan, and a plan allocates (twiddles, k^2 tables, a work
// field, reduction slots); this entry point needs none of it.
//
// Where the scratch lives: the per-block partial sums, the last-block ticket and the result
// slot are one file-scope static __device__ array, g_norm_scratch, of kScratchBytes
// (33,024 bytes).  Every GPU that loads this library holds one copy until the process
// exits.  Host code may not pass the array's name to a kernel (on the host the name is only
// a stand-in, not a device address), so the first call on each device looks up the device
// address with cudaGetSymbolAddress, with that device current, and caches it.  Because of
// that look-up, make the first call on a device before any stream capture.  The cache is
// keyed by the device and the unique id of its current CUDA context: after a
// cudaDeviceReset (or any other re-creation of the context) the first call looks the
// address up again instead of using one from the destroyed context.
//
// Sharing: every call uses the same array and leaves the last call's contents in it; the
// ticket is cleared at the start of each call.  Calls whose kernels overlap on the GPU (for
// example on two streams at once) race on the array and must not be issued.  Each call reads
// the result back and synchronises `stream` before it returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/gp5cu.h"
#include "common.cuh"

namespace gp5 {
void set_last_error(const std::string &msg);
}

namespace {

using gp5::cpx;

constexpr int kThreadsNA = 256;
constexpr int kSitesPerThread = 16;
constexpr long long kSitesPerBlock = (long long)kThreadsNA * kSitesPerThread;  // 4096
constexpr int kMaxBlocksNA = 4096;
constexpr long long kMaxSites = kSitesPerBlock * kMaxBlocksNA;  // 16,777,216 = 256^3
// layout: [0, 8*kMaxBlocksNA) partial sums (double), then the ticket (unsigned) and the
// result (double), each in its own 128-byte slot
constexpr size_t kTicketOffset = sizeof(double) * kMaxBlocksNA;
constexpr size_t kResultOffset = kTicketOffset + 128;
constexpr size_t kScratchBytes = kResultOffset + 128;

static __device__ __align__(256) unsigned char g_norm_scratch[kScratchBytes];

static_assert(GP5_NOALLOC_MAX_SITES == kMaxSites, "header limit must match the scratch size");

__device__ __forceinline__ void neumaier_add(double &s, double &c, double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__device__ double block_sum_na(double v) {
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = (w == 0 && lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    if (w == 0)
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    return v;
}

// Block b sums |f|^2 over sites [b*4096, (b+1)*4096) of one component; the last block to
// finish adds the partials in index order and stores dV * total in the result slot.
template <typename Real>
__global__ void __launch_bounds__(kThreadsNA) k_norm_noalloc(const cpx<Real> *__restrict__ f, long long nsites,
                                                             double dV, unsigned char *scratch) {
    double *partials = reinterpret_cast<double *>(scratch);
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + kTicketOffset);
    double *result = reinterpret_cast<double *>(scratch + kResultOffset);
    const long long base = (long long)blockIdx.x * kSitesPerBlock;
    double acc = 0.0;
#pragma unroll 4
    for (int q = 0; q < kSitesPerThread; q++) {
        const long long s = base + (long long)q * kThreadsNA + threadIdx.x;
        if (s < nsites) {
            const cpx<Real> v = f[s];
            acc += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
        }
    }
    acc = block_sum_na(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    __threadfence();
    __shared__ bool last;
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0, c = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) neumaier_add(s, c, __ldcg(partials + b));
    s = block_sum_na(s);
    c = block_sum_na(c);
    if (threadIdx.x == 0) {
        *result = (s + c) * dV;
        *ticket = 0u;
    }
}

std::mutex g_mu;
// per device: the scratch address and the id of the context it was looked up in
void *g_scratch_addr[64] = {nullptr};
unsigned long long g_scratch_ctx[64] = {0};

int fail_na(int status, const std::string &msg) {
    gp5::set_last_error(msg);
    return status;
}

// Unique id of the calling thread's current CUDA context (0 if none can be had).  The driver
// functions come through cudaGetDriverEntryPoint, so the library needs no link to libcuda.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f1);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f2);
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}

}  // namespace

extern "C" int gp5cu_norm_noalloc(const void *dfield, int precision, const int shape[3], int ncomp, int comp,
                                  double dV, void *stream, double *out) {
    if (!dfield || !shape || !out) return fail_na(GP5_ERR_ARG, "NULL argument");
    if (precision != GP5_C128 && precision != GP5_C64)
        return fail_na(GP5_ERR_ARG, "precision must be GP5_C128 or GP5_C64");
    // one complex element: 16 bytes (double2) or 8 bytes (float2)
    const uintptr_t align = precision == GP5_C128 ? 16u : 8u;
    if (((uintptr_t)dfield & (align - 1)) != 0)
        return fail_na(GP5_ERR_ARG, precision == GP5_C128 ? "dfield is not 16-byte aligned"
                                                          : "dfield is not 8-byte aligned");
    if (ncomp < 1 || comp < 0 || comp >= ncomp) return fail_na(GP5_ERR_ARG, "component out of range");
    long long nsites = 1;
    for (int d = 0; d < 3; d++) {
        if (shape[d] < 1) return fail_na(GP5_ERR_ARG, "shape entries must be positive");
        // the limit is checked before each product, so the count never overflows
        if ((long long)shape[d] > kMaxSites / nsites)
            return fail_na(GP5_ERR_ARG, "gp5cu_norm_noalloc: the field exceeds the static scratch limit of " +
                                            std::to_string(kMaxSites) + " sites (GP5_NOALLOC_MAX_SITES); use gp5cu_norm");
        nsites *= shape[d];
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_na(GP5_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail_na(GP5_ERR_ARG, "device ordinal out of range");
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        const unsigned long long ctx = current_context_id();
        if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
            // set-up, once per device (and again for a new context), with that device current
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_norm_scratch);
            if (e != cudaSuccess || !ptr)
                return fail_na(GP5_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_addr[dev] = ptr;
            g_scratch_ctx[dev] = current_context_id();
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *sc = static_cast<unsigned char *>(scratch);
    // the ticket must start at zero: clear it (the result slot is overwritten by the kernel)
    e = cudaMemsetAsync(sc + kTicketOffset, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return fail_na(GP5_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const unsigned blocks = (unsigned)((nsites + kSitesPerBlock - 1) / kSitesPerBlock);
    const long long off = (long long)comp * nsites;
    if (precision == GP5_C128)
        k_norm_noalloc<double><<<blocks, kThreadsNA, 0, s>>>((const double2 *)dfield + off, nsites, dV, sc);
    else
        k_norm_noalloc<float><<<blocks, kThreadsNA, 0, s>>>((const float2 *)dfield + off, nsites, dV, sc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_na(GP5_ERR_CUDA, std::string("k_norm_noalloc: ") + cudaGetErrorString(e));
    double r = 0.0;
    e = cudaMemcpyAsync(&r, sc + kResultOffset, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_na(GP5_ERR_CUDA, std::string("norm read-back: ") + cudaGetErrorString(e));
    *out = r;
    return GP5_OK;
}

// mlp.cu - the learned warm start: a 3 -> 256 -> 256 -> 256 -> 64 GELU MLP whose GEMMs are
// hand-written tcgen05 (5th-generation tensor core) kernels: BF16 operands staged in shared
// memory, FP32 accumulators in tensor memory (TMEM), one elected thread issuing the MMAs.
// Forward, backward (input and weight gradients) and inference all run through the same
// GEMM; Adam keeps FP32 master weights and refreshes their BF16 copies after every update.
//
// No reference counterpart: the reference starts every solve from a Gaussian
// (python/test/regressionTests/LHY_imaginary.py:14).
//
// UMMA operands (both K-major, no swizzle): a tile of R rows x 64 K-values is stored as
// 8-row x 8-element "core matrices" of 128 bytes, core (r/8, k/8) at ((r/8)*8 + k/8)*128 bytes,
// element (r, k) at +(r%8)*16 + (k%8)*2.  The descriptor of one K=16 step then has
// LBO = 128 B (the second 8-element K half) and SBO = 1024 B (the next 8-row group).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "../../include/gp5cu.h"

namespace gp5 {
void set_last_error(const std::string &msg);
}

namespace {

using bf16 = __nv_bfloat16;

constexpr int kGemmThreads = 128;  // 4 warps: warp w owns TMEM lanes 32w..32w+31 (rows)
constexpr int kTileM = 128;
constexpr int kTileK = 64;
// default bound of the per-chunk MMA wait, and the fixed bound of the drain wait after a timeout
constexpr unsigned long long kWaitNs = GP5_GEMM_WAIT_DEFAULT_NS;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with the given parity; false once timeout_ns has passed.  The first
// probe does not block (test_wait), so a bound of 0 returns false whenever the phase is not
// complete at the call; later probes use try_wait.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned long long timeout_ns) {
    const uint32_t a = smem_u32(bar);
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        if (globaltimer_ns() - t0 >= timeout_ns) return false;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version 1 (sm_100); base offset 0, no swizzle
    return d;
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

struct GemmArgs {
    const bf16 *A;
    long long sam, sak;  // A(m, k) = A[m*sam + k*sak]
    const bf16 *B;
    long long sbn, sbk;  // B(n, k) = B[n*sbn + k*sbk]
    int M, N, K;
    // epilogue: v = acc (+ bias[n]); out32[m*ld + n] = beta*out32 + v; pre32 = v before GELU;
    // gelu: out32/out16 = GELU(v)
    const float *bias;
    float *out32;
    bf16 *out16;
    float *pre32;
    long long ld;
    float beta;
    int gelu;
    unsigned *err;
    // bound of each K chunk's MMA wait; on timeout the CTA drains its MMAs (fixed 2 s bound),
    // sets *err and returns
    unsigned long long wait_ns = kWaitNs;
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// Fills a rows x 64 K-major core-matrix tile from global memory (zeros outside the matrix).
__device__ void fill_tile(unsigned char *tile, int rows, const bf16 *src, long long srow, long long sk, int row0,
                          int rmax, int k0, int kmax) {
    const int units = rows * (kTileK / 8);
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int r = u / (kTileK / 8), kg = u % (kTileK / 8);
        const int gr = row0 + r;
        __align__(16) bf16 v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int gk = k0 + kg * 8 + e;
            v[e] = (gr < rmax && gk < kmax) ? src[(long long)gr * srow + (long long)gk * sk] : __float2bfloat16(0.f);
        }
        *reinterpret_cast<uint4 *>(tile + ((r / 8) * (kTileK / 8) + kg) * 128 + (r % 8) * 16) =
            *reinterpret_cast<const uint4 *>(v);
    }
}

// C tile (128 x NT) = A (128 x K) * B^T (NT x K), FP32 accumulators in TMEM.
template <int NT>
__global__ void __launch_bounds__(kGemmThreads, 1) k_gemm_tc(const GemmArgs a) {
    static_assert(NT == 64 || NT == 128 || NT == 256, "TMEM columns: power of two in [64, 256]");
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *ta = smem;                      // 128 x 64 bf16 = 16 KB
    unsigned char *tb = smem + kTileM * kTileK * 2;  // NT x 64 bf16
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * NT;
    const int warp = threadIdx.x / 32;

    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(NT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    const uint32_t idesc = instr_desc(NT);
    unsigned phase = 0;
    const int nk = (a.K + kTileK - 1) / kTileK;
    for (int kc = 0; kc < nk && !failed; kc++) {
        fill_tile(ta, kTileM, a.A, a.sam, a.sak, m0, a.M, kc * kTileK, a.K);
        fill_tile(tb, NT, a.B, a.sbn, a.sbk, n0, a.N, kc * kTileK, a.K);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy writes -> MMA
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < kTileK / 16; s++) {
                const uint64_t da = smem_desc(smem_u32(ta) + s * 256, 128, (kTileK / 8) * 128);
                const uint64_t db = smem_desc(smem_u32(tb) + s * 256, 128, (kTileK / 8) * 128);
                const uint32_t accum = (kc > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar))
                         : "memory");
        }
        // every thread waits for the MMAs before the tiles are overwritten or TMEM is read
        if (!mbar_wait(&bar, phase, a.wait_ns)) failed = 1;
        phase ^= 1u;
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (failed) {
        // the MMAs of the timed-out chunk may still be in flight: wait for them once more
        // (bounded) before the tensor memory is released
        mbar_wait(&bar, phase ^ 1u, kWaitNs);
        if (threadIdx.x == 0 && a.err) atomicOr(a.err, 1u);
    } else {
        // epilogue: thread (warp w, lane t) owns row m0 + 32w + t
        const int m = m0 + warp * 32 + (threadIdx.x % 32);
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 8) {
            uint32_t r[8];
            const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < a.M) {
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int n = n0 + c0 + e;
                    if (n >= a.N) continue;
                    float v = __uint_as_float(r[e]);
                    if (a.bias) v += a.bias[n];
                    const long long o = (long long)m * a.ld + n;
                    if (a.pre32) a.pre32[o] = v;
                    if (a.gelu) v = gelu_f(v);
                    if (a.out32) a.out32[o] = (a.beta != 0.f) ? a.beta * a.out32[o] + v : v;
                    if (a.out16) a.out16[o] = __float2bfloat16(v);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT) : "memory");
}

void launch_gemm(const GemmArgs &a, cudaStream_t s) {
    const int nt = a.N <= 64 ? 64 : (a.N <= 128 ? 128 : 256);
    const dim3 grid((a.M + kTileM - 1) / kTileM, (a.N + nt - 1) / nt);
    const size_t smem = (size_t)(kTileM + nt) * kTileK * 2;
    cudaError_t e;
    if (nt == 64) {
        cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_gemm_tc<64><<<grid, kGemmThreads, smem, s>>>(a);
    } else if (nt == 128) {
        cudaFuncSetAttribute(k_gemm_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_gemm_tc<128><<<grid, kGemmThreads, smem, s>>>(a);
    } else {
        cudaFuncSetAttribute(k_gemm_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_gemm_tc<256><<<grid, kGemmThreads, smem, s>>>(a);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) throw std::string("gemm launch: ") + cudaGetErrorString(e);
}

// ---- element-wise kernels --------------------------------------------------------------------
__global__ void k_to_bf16(const float *in, bf16 *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16(in[i]);
}

// dY = 2 (Y - T) / (B * 64) as BF16, and the per-block squared error (loss partials)
__global__ void k_mse_grad(const float *Y, const float *T, bf16 *dY, float *dY32, long long n, float scale,
                           double *loss) {
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        s += (double)d * d;
        const float g = 2.f * d * scale;
        dY[i] = __float2bfloat16(g);
        dY32[i] = g;
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// dH = dA * GELU'(pre), BF16 out
__global__ void k_gelu_back(const float *dA, const float *pre, bf16 *dH, float *dH32, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float x = pre[i];
        const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
        const float g = dA[i] * (cdf + x * pdf);
        dH[i] = __float2bfloat16(g);
        dH32[i] = g;
    }
}

// db[j] = sum_b d[b*width + j] (FP32, one thread per column)
__global__ void k_bias_grad(const float *d, float *db, int rows, int width) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= width) return;
    float s = 0.f;
    for (int b = 0; b < rows; b++) s += d[(long long)b * width + j];
    db[j] = s;
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, bf16 *w16, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (w16) w16[i] = __float2bfloat16(wi);
    }
}

}  // namespace

// ---- the network ------------------------------------------------------------------------------
struct gp5cu_mlp {
    static constexpr int IN = 3, H = 256, OUT = 64, L = 4;
    int dev = 0;
    cudaStream_t stream = nullptr;
    int fan_in[L] = {IN, H, H, H}, fan_out[L] = {H, H, H, OUT};
    long long woff[L], boff[L], nparam = 0;
    float *p32 = nullptr, *g32 = nullptr, *m32 = nullptr, *v32 = nullptr;  // parameters, grads, Adam moments
    bf16 *p16 = nullptr;                                                 // BF16 copies
    unsigned *err = nullptr;
    double *loss = nullptr;
    unsigned long long wait_ns = GP5_GEMM_WAIT_DEFAULT_NS;  // per-chunk MMA wait bound of its GEMMs
    int cap = 0;  // batch capacity of the buffers below
    bf16 *x16 = nullptr, *act16[L] = {}, *d16 = nullptr;
    float *pre[L] = {}, *act32 = nullptr, *y32 = nullptr, *t32 = nullptr, *d32a = nullptr, *d32b = nullptr;
    long long step = 0;
};

namespace {

void ck(cudaError_t e, const char *w) {
    if (e != cudaSuccess) throw std::string(w) + ": " + cudaGetErrorString(e);
}

void ensure_batch(gp5cu_mlp *n, int B) {
    if (B <= n->cap) return;
    auto fr = [](void *p) {
        if (p) cudaFree(p);
    };
    fr(n->x16);
    fr(n->d16);
    fr(n->act32);
    fr(n->y32);
    fr(n->t32);
    fr(n->d32a);
    fr(n->d32b);
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        fr(n->act16[l]);
        fr(n->pre[l]);
    }
    const int H = gp5cu_mlp::H;
    ck(cudaMalloc(&n->x16, sizeof(bf16) * B * gp5cu_mlp::IN), "cudaMalloc");
    ck(cudaMalloc(&n->d16, sizeof(bf16) * B * H), "cudaMalloc");
    ck(cudaMalloc(&n->act32, sizeof(float) * B * H), "cudaMalloc");
    ck(cudaMalloc(&n->y32, sizeof(float) * B * gp5cu_mlp::OUT), "cudaMalloc");
    ck(cudaMalloc(&n->t32, sizeof(float) * B * gp5cu_mlp::OUT), "cudaMalloc");
    ck(cudaMalloc(&n->d32a, sizeof(float) * B * H), "cudaMalloc");
    ck(cudaMalloc(&n->d32b, sizeof(float) * B * H), "cudaMalloc");
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        ck(cudaMalloc(&n->act16[l], sizeof(bf16) * B * H), "cudaMalloc");
        ck(cudaMalloc(&n->pre[l], sizeof(float) * B * H), "cudaMalloc");
    }
    n->cap = B;
}

void refresh_bf16(gp5cu_mlp *n) {
    k_to_bf16<<<256, 256, 0, n->stream>>>(n->p32, n->p16, n->nparam);
    ck(cudaGetLastError(), "k_to_bf16");
}

// forward of B samples already in x16; output in y32, activations kept for backward
void forward(gp5cu_mlp *n, int B) {
    const bf16 *in = n->x16;
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        GemmArgs a{};
        a.A = in;
        a.sam = n->fan_in[l];
        a.sak = 1;
        a.B = n->p16 + n->woff[l];  // W[out][in]: B(n, k) = W[n*in + k]
        a.sbn = n->fan_in[l];
        a.sbk = 1;
        a.M = B;
        a.N = n->fan_out[l];
        a.K = n->fan_in[l];
        a.bias = n->p32 + n->boff[l];
        a.ld = n->fan_out[l];
        a.err = n->err;
        a.wait_ns = n->wait_ns;
        if (l < gp5cu_mlp::L - 1) {
            a.pre32 = n->pre[l];
            a.gelu = 1;
            a.out16 = n->act16[l];
        } else {
            a.out32 = n->y32;
        }
        launch_gemm(a, n->stream);
        in = n->act16[l];
    }
}

// backward of the MSE loss against t32 (B samples); gradients into g32
void backward(gp5cu_mlp *n, int B) {
    const int OUT = gp5cu_mlp::OUT, H = gp5cu_mlp::H;
    ck(cudaMemsetAsync(n->loss, 0, sizeof(double), n->stream), "memset");
    k_mse_grad<<<128, 256, 0, n->stream>>>(n->y32, n->t32, n->d16, n->d32a, (long long)B * OUT,
                                           1.f / ((float)B * OUT), n->loss);
    ck(cudaGetLastError(), "k_mse_grad");
    for (int l = gp5cu_mlp::L - 1; l >= 0; l--) {
        const int fin = n->fan_in[l], fout = n->fan_out[l];
        const bf16 *xin = l == 0 ? n->x16 : n->act16[l - 1];
        // dW[o][i] = sum_b d[b][o] * x[b][i]: M = fout, N = fin, K = B
        GemmArgs gw{};
        gw.A = n->d16;
        gw.sam = 1;
        gw.sak = fout;
        gw.B = xin;
        gw.sbn = 1;
        gw.sbk = fin;
        gw.M = fout;
        gw.N = fin;
        gw.K = B;
        gw.out32 = n->g32 + n->woff[l];
        gw.ld = fin;
        gw.err = n->err;
        gw.wait_ns = n->wait_ns;
        launch_gemm(gw, n->stream);
        k_bias_grad<<<(fout + 255) / 256, 256, 0, n->stream>>>(n->d32a, n->g32 + n->boff[l], B, fout);
        ck(cudaGetLastError(), "k_bias_grad");
        if (l == 0) break;
        // dX[b][i] = sum_o d[b][o] W[o][i]: M = B, N = fin, K = fout; B(n=i, k=o) = W[o*fin + i]
        GemmArgs gx{};
        gx.A = n->d16;
        gx.sam = fout;
        gx.sak = 1;
        gx.B = n->p16 + n->woff[l];
        gx.sbn = 1;
        gx.sbk = fin;
        gx.M = B;
        gx.N = fin;
        gx.K = fout;
        gx.out32 = n->d32b;
        gx.ld = fin;
        gx.err = n->err;
        gx.wait_ns = n->wait_ns;
        launch_gemm(gx, n->stream);
        // through the GELU of layer l-1
        k_gelu_back<<<256, 256, 0, n->stream>>>(n->d32b, n->pre[l - 1], n->d16, n->d32a, (long long)B * fin);
        ck(cudaGetLastError(), "k_gelu_back");
        (void)H;
    }
}

// A bounded device wait ran out: reported as GP5_ERR_TIMEOUT.
struct WaitTimeout {
    std::string msg;
};

// Reads the GEMM error flag of the net's stream; a set flag is cleared (so the next call on
// the handle starts clean) and reported as a timeout.
void check_err(gp5cu_mlp *n) {
    unsigned e = 0;
    ck(cudaMemcpyAsync(&e, n->err, sizeof(unsigned), cudaMemcpyDeviceToHost, n->stream), "read err");
    ck(cudaStreamSynchronize(n->stream), "sync");
    if (e) {
        ck(cudaMemsetAsync(n->err, 0, sizeof(unsigned), n->stream), "clear err");
        ck(cudaStreamSynchronize(n->stream), "sync");
        throw WaitTimeout{"tensor-core GEMM: a bounded mbarrier wait ran out"};
    }
}

void upload_xt(gp5cu_mlp *n, const float *x, const float *t, int B) {
    ensure_batch(n, B);
    std::vector<bf16> xb((size_t)B * gp5cu_mlp::IN);
    for (size_t i = 0; i < xb.size(); i++) xb[i] = __float2bfloat16(x[i]);
    ck(cudaMemcpyAsync(n->x16, xb.data(), sizeof(bf16) * xb.size(), cudaMemcpyHostToDevice, n->stream), "upload");
    if (t)
        ck(cudaMemcpyAsync(n->t32, t, sizeof(float) * B * gp5cu_mlp::OUT, cudaMemcpyHostToDevice, n->stream),
           "upload");
    ck(cudaStreamSynchronize(n->stream), "sync");  // xb goes out of scope
}

int fail_m(int st, const std::string &m) {
    gp5::set_last_error(m);
    return st;
}

}  // namespace

#define MLP_TRY try {
#define MLP_CATCH                                   \
    }                                               \
    catch (const WaitTimeout &e) {                  \
        return fail_m(GP5_ERR_TIMEOUT, e.msg);      \
    }                                               \
    catch (const std::string &e) {                  \
        return fail_m(GP5_ERR_CUDA, e);             \
    }                                               \
    return GP5_OK;

extern "C" {

int gp5cu_mlp_create(gp5cu_mlp **out, int device, unsigned long long seed) {
    if (!out) return fail_m(GP5_ERR_ARG, "out is NULL");
    *out = nullptr;
    gp5cu_mlp *n = new gp5cu_mlp();
    try {
    n->dev = device;
    ck(cudaSetDevice(device), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    long long off = 0;
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        n->woff[l] = off;
        off += (long long)n->fan_in[l] * n->fan_out[l];
        n->boff[l] = off;
        off += n->fan_out[l];
    }
    n->nparam = off;
    ck(cudaMalloc(&n->p32, sizeof(float) * off), "cudaMalloc");
    ck(cudaMalloc(&n->g32, sizeof(float) * off), "cudaMalloc");
    ck(cudaMalloc(&n->m32, sizeof(float) * off), "cudaMalloc");
    ck(cudaMalloc(&n->v32, sizeof(float) * off), "cudaMalloc");
    ck(cudaMalloc(&n->p16, sizeof(bf16) * off), "cudaMalloc");
    ck(cudaMalloc(&n->err, sizeof(unsigned)), "cudaMalloc");
    ck(cudaMalloc(&n->loss, sizeof(double)), "cudaMalloc");
    ck(cudaMemset(n->err, 0, sizeof(unsigned)), "memset");
    ck(cudaMemset(n->m32, 0, sizeof(float) * off), "memset");
    ck(cudaMemset(n->v32, 0, sizeof(float) * off), "memset");
    // He-style uniform initialisation (seeded), zero biases
    std::vector<float> h(off, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        const float lim = std::sqrt(6.f / (float)n->fan_in[l]) * (l == gp5cu_mlp::L - 1 ? 0.5f : 1.f);
        std::uniform_real_distribution<float> U(-lim, lim);
        for (long long i = 0; i < (long long)n->fan_in[l] * n->fan_out[l]; i++) h[n->woff[l] + i] = U(rng);
    }
    ck(cudaMemcpy(n->p32, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice), "upload");
    refresh_bf16(n);
    ck(cudaStreamSynchronize(n->stream), "sync");
    *out = n;
    } catch (const std::string &e) {
        gp5cu_mlp_destroy(n);  // frees whatever was allocated before the failure
        return fail_m(GP5_ERR_CUDA, e);
    }
    return GP5_OK;
}

int gp5cu_mlp_destroy(gp5cu_mlp *n) {
    if (!n) return GP5_OK;
    cudaSetDevice(n->dev);
    if (n->stream) cudaStreamSynchronize(n->stream);
    void *ptrs[] = {n->p32, n->g32, n->m32, n->v32, n->p16, n->err, n->loss, n->x16, n->d16, n->act32,
                    n->y32, n->t32, n->d32a, n->d32b};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int l = 0; l < gp5cu_mlp::L; l++) {
        if (n->act16[l]) cudaFree(n->act16[l]);
        if (n->pre[l]) cudaFree(n->pre[l]);
    }
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return GP5_OK;
}

long long gp5cu_mlp_num_params(const gp5cu_mlp *n) { return n ? n->nparam : 0; }

int gp5cu_mlp_set_wait_bound(gp5cu_mlp *n, unsigned long long ns) {
    if (!n) return fail_m(GP5_ERR_ARG, "NULL argument");
    n->wait_ns = ns;
    return GP5_OK;
}

int gp5cu_mlp_get_params(gp5cu_mlp *n, float *host) {
    if (!n || !host) return fail_m(GP5_ERR_ARG, "NULL argument");
    MLP_TRY
    ck(cudaSetDevice(n->dev), "cudaSetDevice");
    ck(cudaMemcpyAsync(host, n->p32, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->stream), "download");
    ck(cudaStreamSynchronize(n->stream), "sync");
    MLP_CATCH
}

int gp5cu_mlp_set_params(gp5cu_mlp *n, const float *host) {
    if (!n || !host) return fail_m(GP5_ERR_ARG, "NULL argument");
    MLP_TRY
    ck(cudaSetDevice(n->dev), "cudaSetDevice");
    ck(cudaMemcpyAsync(n->p32, host, sizeof(float) * n->nparam, cudaMemcpyHostToDevice, n->stream), "upload");
    refresh_bf16(n);
    ck(cudaStreamSynchronize(n->stream), "sync");
    MLP_CATCH
}

int gp5cu_mlp_forward(gp5cu_mlp *n, const float *x, int B, float *y) {
    if (!n || !x || !y || B < 1) return fail_m(GP5_ERR_ARG, "invalid argument");
    MLP_TRY
    ck(cudaSetDevice(n->dev), "cudaSetDevice");
    upload_xt(n, x, nullptr, B);
    forward(n, B);
    ck(cudaMemcpyAsync(y, n->y32, sizeof(float) * B * gp5cu_mlp::OUT, cudaMemcpyDeviceToHost, n->stream), "download");
    check_err(n);
    MLP_CATCH
}

int gp5cu_mlp_gradients(gp5cu_mlp *n, const float *x, const float *t, int B, float *grad, double *loss) {
    if (!n || !x || !t || !grad || !loss || B < 1) return fail_m(GP5_ERR_ARG, "invalid argument");
    MLP_TRY
    ck(cudaSetDevice(n->dev), "cudaSetDevice");
    upload_xt(n, x, t, B);
    forward(n, B);
    backward(n, B);
    double l = 0;
    ck(cudaMemcpyAsync(grad, n->g32, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->stream), "download");
    ck(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream), "download");
    check_err(n);
    *loss = l / ((double)B * gp5cu_mlp::OUT);
    MLP_CATCH
}

int gp5cu_mlp_train(gp5cu_mlp *n, const float *x, const float *t, int count, int epochs, int batch, float lr,
                    unsigned long long seed, float *loss_history) {
    if (!n || !x || !t || count < 1 || epochs < 1 || batch < 1) return fail_m(GP5_ERR_ARG, "invalid argument");
    MLP_TRY
    ck(cudaSetDevice(n->dev), "cudaSetDevice");
    const int IN = gp5cu_mlp::IN, OUT = gp5cu_mlp::OUT;
    const int B = batch < count ? batch : count;
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::mt19937_64 rng(seed);
    std::vector<float> xb((size_t)B * IN), tb((size_t)B * OUT);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        double ep_loss = 0;
        int nb = 0;
        for (int s0 = 0; s0 + B <= count; s0 += B) {
            for (int b = 0; b < B; b++) {
                const int i = order[s0 + b];
                for (int c = 0; c < IN; c++) xb[(size_t)b * IN + c] = x[(size_t)i * IN + c];
                for (int c = 0; c < OUT; c++) tb[(size_t)b * OUT + c] = t[(size_t)i * OUT + c];
            }
            upload_xt(n, xb.data(), tb.data(), B);
            forward(n, B);
            backward(n, B);
            n->step++;
            const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
            k_adam<<<256, 256, 0, n->stream>>>(n->p32, n->g32, n->m32, n->v32, n->p16, n->nparam, lr, b1, b2, eps,
                                               c1, c2);
            ck(cudaGetLastError(), "k_adam");
            double l = 0;
            ck(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream), "download");
            check_err(n);
            ep_loss += l / ((double)B * OUT);
            nb++;
        }
        if (loss_history) loss_history[ep] = (float)(ep_loss / (nb > 0 ? nb : 1));
    }
    MLP_CATCH
}

int gp5cu_gemm_bf16(const void *A, long long sam, long long sak, const void *B, long long sbn, long long sbk, float *C,
                    long long ldc, int M, int N, int K, void *stream) {
    if (!A || !B || !C || M < 1 || N < 1 || K < 1) return fail_m(GP5_ERR_ARG, "invalid argument");
    MLP_TRY
    unsigned *err = nullptr;
    ck(cudaMalloc(&err, sizeof(unsigned)), "cudaMalloc");
    unsigned e = 0;
    try {
        ck(cudaMemsetAsync(err, 0, sizeof(unsigned), (cudaStream_t)stream), "memset");
        GemmArgs a{};
        a.A = (const bf16 *)A;
        a.sam = sam;
        a.sak = sak;
        a.B = (const bf16 *)B;
        a.sbn = sbn;
        a.sbk = sbk;
        a.M = M;
        a.N = N;
        a.K = K;
        a.out32 = C;
        a.ld = ldc;
        a.err = err;
        for (int n0 = 0; n0 < N; n0 += 256) {  // N tiles of 256 per launch group
            GemmArgs b = a;
            b.B = a.B + (long long)n0 * sbn;
            b.N = N - n0 < 256 ? N - n0 : 256;
            b.out32 = C + n0;
            launch_gemm(b, (cudaStream_t)stream);
        }
        ck(cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, (cudaStream_t)stream), "read err");
        ck(cudaStreamSynchronize((cudaStream_t)stream), "sync");
    } catch (...) {
        cudaStreamSynchronize((cudaStream_t)stream);
        cudaFree(err);  // the flag buffer is released on every path
        throw;
    }
    cudaFree(err);
    if (e) throw WaitTimeout{"tensor-core GEMM: a bounded mbarrier wait ran out"};
    MLP_CATCH
}

}  // extern "C"

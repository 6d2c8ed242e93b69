// gp5cu_cluster.cu - droplet decomposition: connected components of the sites whose density
// exceeds a cutoff, 26-connected with periodic boundaries, as gp::decompose::decompose
// (src/cluster.cpp:17-83) labels them for the gpCpp `decomposition` class
// (src/gpCpp.cpp:289-313).
//
// Reference semantics kept: a site with |psi_c|^2 <= cutoff gets -1; the clusters are numbered
// 1, 2, ... in the order in which a scan over (i, j, k) with i slowest and k fastest meets their
// first site; the other components' labels are 0.
//
// GPU form: lock-free union-find.  Labels live in "scan-key" order (key = (i*ny + j)*nz + k), a
// union always links the larger root under the smaller (atomicMin), so every cluster's root is
// its smallest key, i.e. the site at which the reference's scan starts it.  Ranking the roots by
// key (per-block counts, a host prefix over the blocks, a block scan) gives the reference's
// numbers.  Scratch: the plan's work field (parent and root-id arrays, 8 bytes per site) and its
// partials buffer (per-block counts); nothing is allocated per call.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "plan.hpp"

namespace gp5 {
namespace {

constexpr int kCcThreads = 256;
constexpr int kRankBlock = 1024;  // keys per ranking block

__device__ __forceinline__ long long scan_key(long long s, int nx, int ny, int nz) {
    const long long i = s % nx, j = (s / nx) % ny, k = s / ((long long)nx * ny);
    return (i * ny + j) * nz + k;
}

template <typename Real>
__global__ void k_cc_init(const cpx<Real> *__restrict__ psi, long long nsites, int nx, int ny, int nz, double cutoff,
                          int *__restrict__ parent) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nsites;
         s += (long long)gridDim.x * blockDim.x) {
        const double re = (double)psi[s].x, im = (double)psi[s].y;
        const double d = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
        const long long key = scan_key(s, nx, ny, nz);
        parent[key] = d > cutoff ? (int)key : -1;
    }
}

__device__ __forceinline__ int cc_find(const int *parent, int x) {
    int p = ((volatile const int *)parent)[x];
    while (p != x) {
        x = p;
        p = ((volatile const int *)parent)[x];
    }
    return x;
}

__device__ __forceinline__ void cc_union(int *parent, int a, int b) {
    while (true) {
        a = cc_find(parent, a);
        b = cc_find(parent, b);
        if (a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(&parent[b], a);
        if (old == b) return;  // b was a root and now hangs under a
        b = old;               // b was linked meanwhile: merge its new parent instead
    }
}

// each foreground site unites with its 13 neighbours of positive offset order (the other 13
// unite with it); periodic in every direction
__global__ void k_cc_union(int *parent, long long nkeys, int nx, int ny, int nz) {
    for (long long key = blockIdx.x * (long long)blockDim.x + threadIdx.x; key < nkeys;
         key += (long long)gridDim.x * blockDim.x) {
        if (parent[key] < 0) continue;
        const int k = (int)(key % nz), j = (int)((key / nz) % ny), i = (int)(key / ((long long)nz * ny));
        for (int di = 0; di <= 1; di++)
            for (int dj = -1; dj <= 1; dj++)
                for (int dk = -1; dk <= 1; dk++) {
                    if (di == 0 && (dj < 0 || (dj == 0 && dk <= 0))) continue;
                    const int i2 = (i + di) % nx;
                    const int j2 = (j + dj + ny) % ny;
                    const int k2 = (k + dk + nz) % nz;
                    const long long n = ((long long)i2 * ny + j2) * nz + k2;
                    if (((volatile const int *)parent)[n] >= 0) cc_union(parent, (int)key, (int)n);
                }
    }
}

__global__ void k_cc_flatten(int *parent, long long nkeys) {
    for (long long key = blockIdx.x * (long long)blockDim.x + threadIdx.x; key < nkeys;
         key += (long long)gridDim.x * blockDim.x)
        if (parent[key] >= 0) parent[key] = cc_find(parent, (int)key);
}

// roots per block of kRankBlock keys
__global__ void k_cc_count(const int *__restrict__ parent, long long nkeys, int *__restrict__ counts) {
    __shared__ int warp_n[kRankBlock / 32];
    const long long key = (long long)blockIdx.x * kRankBlock + threadIdx.x;
    const bool root = key < nkeys && parent[key] == (int)key;
    const unsigned b = __ballot_sync(0xffffffffu, root);
    if ((threadIdx.x & 31) == 0) warp_n[threadIdx.x >> 5] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kRankBlock / 32; w++) t += warp_n[w];
        counts[blockIdx.x] = t;
    }
}

// root id = 1 + roots before it in key order
__global__ void k_cc_rank(const int *__restrict__ parent, long long nkeys, const int *__restrict__ offsets,
                          int *__restrict__ rootid) {
    __shared__ int warp_n[kRankBlock / 32];
    const long long key = (long long)blockIdx.x * kRankBlock + threadIdx.x;
    const bool root = key < nkeys && parent[key] == (int)key;
    const unsigned b = __ballot_sync(0xffffffffu, root);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_n[w] = __popc(b);
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; q++) before += warp_n[q];
    if (root) rootid[key] = offsets[blockIdx.x] + before + __popc(b & ((1u << lane) - 1u)) + 1;
}

// labels in the field's layout (x fastest, component slowest)
__global__ void k_cc_write(const int *__restrict__ parent, const int *__restrict__ rootid, long long nsites, int nx,
                           int ny, int nz, int ncomp, int comp, int *__restrict__ labels) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nsites;
         s += (long long)gridDim.x * blockDim.x) {
        const int p = parent[scan_key(s, nx, ny, nz)];
        for (int c = 0; c < ncomp; c++) labels[s + c * nsites] = c != comp ? 0 : (p < 0 ? -1 : rootid[p]);
    }
}

}  // namespace
}  // namespace gp5

using namespace gp5;

extern "C" int gp5cu_decompose(gp5cu_plan *p, const void *dfield, int comp, double cutoff, int *dlabels,
                               int *nclusters) {
    try {
        if (!p || !dfield || !dlabels || !nclusters) fail(GP5_ERR_ARG, "NULL argument");
        if (comp < 0 || comp >= p->ncomp) fail(GP5_ERR_ARG, "component out of range");
        if (p->nsolve != 1) fail(GP5_ERR_UNSUPPORTED, "decomposition of batched plans");
        if (p->nsites >= (1ll << 31)) fail(GP5_ERR_UNSUPPORTED, "more than 2^31 sites");
        check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
        const long long n = p->nsites;
        const int nx = p->shape[0], ny = p->shape[1], nz = p->shape[2];
        int *parent = static_cast<int *>(p->work);  // 8 bytes per site fit in one field
        int *rootid = parent + n;
        const long long nb = (n + kRankBlock - 1) / kRankBlock;
        if ((size_t)(2 * nb) * sizeof(int) > sizeof(double) * (size_t)kNRed * (size_t)p->max_blocks)
            fail(GP5_ERR_UNSUPPORTED, "grid too large for the ranking scratch");
        int *counts = reinterpret_cast<int *>(p->partials), *offsets = counts + nb;
        const int grid = (int)std::min<long long>((n + kCcThreads - 1) / kCcThreads, (long long)p->sms * 16);
        cudaStream_t s = p->stream;
        if (p->prec == GP5_C128)
            k_cc_init<double><<<grid, kCcThreads, 0, s>>>((const cpx<double> *)dfield + comp * n, n, nx, ny, nz, cutoff,
                                                          parent);
        else
            k_cc_init<float><<<grid, kCcThreads, 0, s>>>((const cpx<float> *)dfield + comp * n, n, nx, ny, nz, cutoff,
                                                         parent);
        k_cc_union<<<grid, kCcThreads, 0, s>>>(parent, n, nx, ny, nz);
        k_cc_flatten<<<grid, kCcThreads, 0, s>>>(parent, n);
        k_cc_count<<<(unsigned)nb, kRankBlock, 0, s>>>(parent, n, counts);
        check_cuda(cudaGetLastError(), "decomposition launch");
        std::vector<int> h((size_t)nb);
        check_cuda(cudaMemcpyAsync(h.data(), counts, sizeof(int) * nb, cudaMemcpyDeviceToHost, s), "download");
        check_cuda(cudaStreamSynchronize(s), "sync");
        long long total = 0;
        for (long long b = 0; b < nb; b++) {
            const int c = h[(size_t)b];
            h[(size_t)b] = (int)total;
            total += c;
        }
        check_cuda(cudaMemcpyAsync(offsets, h.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s), "upload");
        k_cc_rank<<<(unsigned)nb, kRankBlock, 0, s>>>(parent, n, offsets, rootid);
        k_cc_write<<<grid, kCcThreads, 0, s>>>(parent, rootid, n, nx, ny, nz, p->ncomp, comp, dlabels);
        check_cuda(cudaGetLastError(), "decomposition launch");
        check_cuda(cudaStreamSynchronize(s), "sync");  // h is read by the upload above
        *nclusters = (int)total;
    } catch (const Gp5Error &e) {
        set_last_error(e.msg);
        return e.status;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return GP5_ERR_CUDA;
    }
    return GP5_OK;
}

extern "C" int gp5cu_decompose_host(gp5cu_plan *p, const void *dfield, int comp, double cutoff, int *labels,
                                    int *nclusters) {
    if (!p || !labels) {
        set_last_error("NULL argument");
        return GP5_ERR_ARG;
    }
    int *d = nullptr;
    const size_t bytes = sizeof(int) * (size_t)p->nsites * (size_t)p->ncomp;
    cudaSetDevice(p->dev);
    if (cudaMalloc(&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("cudaMalloc of the label buffer failed");
        return GP5_ERR_NOMEM;
    }
    int st = gp5cu_decompose(p, dfield, comp, cutoff, d, nclusters);
    if (st == GP5_OK && cudaMemcpy(labels, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_last_error("label download failed");
        st = GP5_ERR_CUDA;
    }
    cudaFree(d);
    return st;
}

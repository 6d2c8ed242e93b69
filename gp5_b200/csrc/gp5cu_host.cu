// gp5cu_host.cu - the C ABI (include/gp5cu.h): plans, functionals, steppers.
//
// Host logic only; the kernels and their launch sequences live in launch_impl.cuh.  Every
// entry point catches the library's internal errors and returns a status code; the message
// is kept per thread for gp5cu_last_error().
#include <array>
#include <cstdio>
#include <sys/stat.h>
#include <unistd.h>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "plan.hpp"

namespace gp5 {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

[[noreturn]] void fail(int status, const std::string &msg) { throw Gp5Error{status, msg}; }

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        const int st = (e == cudaErrorMemoryAllocation) ? GP5_ERR_NOMEM : GP5_ERR_CUDA;
        fail(st, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

__global__ void k_set_scalars(DevScalars *ds, int n) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        ds[q].sigma[0] = ds[q].sigma[1] = 1.0;
        ds[q].alpha[0][0] = ds[q].alpha[0][1] = ds[q].alpha[1][0] = ds[q].alpha[1][1] = 1.0;
        ds[q].status = 0u;
    }
}

void smem_opt_in(const void *kernel, size_t bytes, int dev) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    std::lock_guard<std::mutex> lock(mu);
    size_t &have = done[{kernel, dev}];
    if (have >= bytes) return;
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
               "cudaFuncSetAttribute");
    have = bytes;
}

int resident_blocks(const void *kernel, int threads, size_t smem, int dev) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({kernel, dev});
    if (it != cache.end()) return it->second;
    int nb = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (nb < 1) nb = 1;
    cache[{kernel, dev}] = nb;
    return nb;
}

void ProfRec::record(cudaStream_t s, int kind) {
    if (idx >= ev.size()) {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        ev.push_back(e);
        kinds.push_back(kind);
    }
    kinds[idx] = kind;
    check_cuda(cudaEventRecord(ev[idx], s), "cudaEventRecord");
    idx++;
}

void set_scalars(cudaStream_t s, DevScalars *ds, int n) {
    k_set_scalars<<<1, 128, 0, s>>>(ds, n);
    check_cuda(cudaGetLastError(), "k_set_scalars");
}

// Factorisation into the radices of the shared-memory engine: 8 and 4 first, then 2, the
// small odd primes with dedicated butterflies, then any remaining prime up to 61.
static bool factorize(int n, LineSchedule &s) {
    s.n = n;
    s.np = 0;
    int m = n;
    auto push = [&](int r) {
        if (s.np >= kMaxPasses) return false;
        s.rad[s.np++] = r;
        m /= r;
        return true;
    };
    while (m % 8 == 0) if (!push(8)) return false;
    while (m % 4 == 0) if (!push(4)) return false;
    while (m % 2 == 0) if (!push(2)) return false;
    while (m % 3 == 0) if (!push(3)) return false;
    while (m % 5 == 0) if (!push(5)) return false;
    for (int p = 7; p < kMaxRadix && m > 1; p += 2) {
        while (m % p == 0) if (!push(p)) return false;
    }
    return m == 1;
}

template <typename Real> static void *upload_twiddles(int n) {
    std::vector<cpx<Real>> h(n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int j = 0; j < n; j++) {
        const long double a = twopi * (long double)j / (long double)n;
        h[j] = mk<Real>((Real)cosl(a), (Real)(-sinl(a)));
    }
    void *d = nullptr;
    check_cuda(cudaMalloc(&d, sizeof(cpx<Real>) * n), "cudaMalloc twiddles");
    check_cuda(cudaMemcpy(d, h.data(), sizeof(cpx<Real>) * n, cudaMemcpyHostToDevice), "upload twiddles");
    return d;
}

void build_axis_plan(gp5cu_plan *p, int d) {
    AxisPlan &ap = p->ax[d];
    const int n = p->shape[d];
    ap.n = n;
    ap.reg = (n == 32 || n == 64 || n == 128 || n == 256 || n == 512);
    switch (n) {
        case 32: ap.reg_threads = RegCfgAll<32>::T, ap.reg_threads1 = RegCfgAll<32, 1>::T; break;
        case 64: ap.reg_threads = RegCfgAll<64>::T, ap.reg_threads1 = RegCfgAll<64, 1>::T; break;
        case 128: ap.reg_threads = RegCfgAll<128>::T, ap.reg_threads1 = RegCfgAll<128, 1>::T; break;
        case 256: ap.reg_threads = RegCfgAll<256>::T, ap.reg_threads1 = RegCfgAll<256, 1>::T; break;
        case 512: ap.reg_threads = RegCfgAll<512>::T, ap.reg_threads1 = RegCfgAll<512, 1>::T; break;
        default: ap.reg_threads = ap.reg_threads1 = 0;
    }
    if (!factorize(n, ap.sched))
        fail(GP5_ERR_UNSUPPORTED, "axis length " + std::to_string(n) + " has a prime factor > 61");
    ap.tw = p->prec == GP5_C128 ? upload_twiddles<double>(n) : upload_twiddles<float>(n);
    const size_t eb = p->elem_bytes;
    const size_t budget = 96 * 1024;
    long long lines = (long long)(budget / (2 * (size_t)(n + 1) * eb));
    if (lines < 1) {
        lines = 1;
        if (2 * (size_t)(n + 1) * eb > 200 * 1024)
            fail(GP5_ERR_UNSUPPORTED, "axis length " + std::to_string(n) + " too long for one tile");
    }
    ap.smem_lines = (int)std::min<long long>(lines, 64);
}

}  // namespace gp5

using namespace gp5;

// ---------------------------------------------------------------------------------------------
#define GP5_TRY try {
#define GP5_CATCH                                  \
    }                                              \
    catch (const Gp5Error &e) {                    \
        set_last_error(e.msg);                     \
        return e.status;                           \
    }                                              \
    catch (const std::exception &e) {              \
        set_last_error(e.what());                  \
        return GP5_ERR_ARG;                        \
    }                                              \
    return GP5_OK;

static void use_device(const gp5cu_plan *p) { check_cuda(cudaSetDevice(p->dev), "cudaSetDevice"); }

static void require(bool cond, const std::string &msg) {
    if (!cond) fail(GP5_ERR_ARG, msg);
}

static void check_field_ptr(const void *ptr, const char *name) {
    require(ptr != nullptr, std::string(name) + " is NULL");
    require(((uintptr_t)ptr & 15u) == 0, std::string(name) + " is not 16-byte aligned");
}

static void sync_and_check(gp5cu_plan *p, DevScalars *ds) {
    check_cuda(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
    if (ds) {
        unsigned st = 0;
        check_cuda(cudaMemcpy(&st, &ds->status, sizeof(unsigned), cudaMemcpyDeviceToHost), "read status");
        if (st & DS_NONFINITE) fail(GP5_ERR_NONFINITE, "a reduction met NaN/Inf (norm blow-up)");
        if (st & DS_TIMEOUT) fail(GP5_ERR_TIMEOUT, "a bounded device wait ran out");
    }
}

template <class F> static void dispatch(const gp5cu_plan *p, F &&f) {
    if (p->prec == GP5_C128) f((double)0);
    else f((float)0);
}

// Geometry of one solve (gp::discretization for one rank, src/geometry.h:88-90): Fourier
// steps 2 pi / L, cell-centred positions, dV as the product of the space steps in axis order
// (src/geometry.cpp:206-210); the kinetic factor is that of the Laplacian (-1/N^3).
static SolveParams geometry_params(const int shape[3], const double left[3], const double right[3]) {
    SolveParams S{};
    double dv = 1.0;
    long long n = 1;
    for (int d = 0; d < 3; d++) {
        const double L = right[d] - left[d];
        S.dk[d] = 2 * M_PI / L;
        S.left[d] = left[d];
        S.dx[d] = L / shape[d];
        dv *= S.dx[d];
        n *= shape[d];
    }
    S.dV = dv;
    S.kin[0] = S.kin[1] = -1.0 / (double)n;
    S.active = 1;
    return S;
}

// A plan for nsolve independent solves of one grid (boxes may differ per solve).
// Choices of the autotuner, kept in memory and in a JSON file: GP5_AUTOTUNE_CACHE names it
// (empty: no file), default $XDG_CACHE_HOME/gp5_b200/autotune.json or
// ~/.cache/gp5_b200/autotune.json.  Two kinds of entries:
//   "radix|<device>|<nx>x<ny>x<nz>|c<ncomp>|<c128|c64>|build <date time>": the radix schedule
//     (0/1) of the five tuned passes of gp5cu_plan_get_tiles and of the stage boundary, whose
//     entry also carries (bit 1) the bulk-copy ring feed: its tiles have other line counts, so
//     its per-tile partial sums fold in another order.  The
//     schedules round differently, so they are chosen once per grid and precision and every
//     plan of that grid uses them, whatever its number of solves (a batch is then bitwise a
//     set of single solves);
//   "<device>|<nx>x<ny>x<nz>|c<ncomp>|<c128|c64>|s<nsolve>|r<radices>|build <date time>": the
//     five thread counts of gp5cu_plan_get_tiles for those schedules (they change no result
//     bit).
// GP5_AUTOTUNE=0 keeps the default shapes and schedule 0; GP5_RADIX=0 or 1 fixes the schedule
// of every tuned pass and of the boundary (the thread counts are still tuned); GP5_RING=0 or 1
// then fixes the boundary's feed.
static std::mutex g_tune_mu;
static std::map<std::string, std::vector<int>> g_tune_cache;
static bool g_tune_loaded = false;

static std::string tune_cache_path() {
    const char *e = std::getenv("GP5_AUTOTUNE_CACHE");
    if (e) return std::string(e);
    const char *x = std::getenv("XDG_CACHE_HOME");
    if (x && *x) return std::string(x) + "/gp5_b200/autotune.json";
    const char *h = std::getenv("HOME");
    if (h && *h) return std::string(h) + "/.cache/gp5_b200/autotune.json";
    return std::string();
}

// reads entries "key": [integers]; anything else in the file is skipped
static void tune_cache_load(const std::string &path) {
    FILE *f = path.empty() ? nullptr : std::fopen(path.c_str(), "rb");
    if (!f) return;
    std::string txt;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, n);
    std::fclose(f);
    size_t pos = 0;
    while ((pos = txt.find('"', pos)) != std::string::npos) {
        const size_t end = txt.find('"', pos + 1);
        if (end == std::string::npos) break;
        const std::string key = txt.substr(pos + 1, end - pos - 1);
        size_t q = txt.find_first_not_of(" \t\r\n:", end + 1);
        if (q == std::string::npos || txt[q] != '[') {
            pos = end + 1;
            continue;
        }
        const size_t close = txt.find(']', q);
        if (close == std::string::npos) break;
        std::vector<int> v;
        const char *c = txt.c_str() + q + 1;
        const char *stop = txt.c_str() + close;
        while (c < stop) {
            char *next = nullptr;
            const long x = std::strtol(c, &next, 10);
            if (next == c) break;
            v.push_back((int)x);
            c = next;
            while (c < stop && (*c == ' ' || *c == ',' || *c == '\n' || *c == '\t' || *c == '\r')) c++;
        }
        const bool is_radix = key.compare(0, 6, "radix|") == 0;
        bool ok = (int)v.size() == (is_radix ? kTunedPasses + 1 : kTunedPasses);
        for (size_t q = 0; q < v.size(); q++) {
            const int x = v[q];
            // radix entries: 0/1 per tuned pass; the boundary's entry also carries the ring bit
            const int hi = (is_radix && (int)q == kTunedPasses) ? 3 : 1;
            ok = ok && (is_radix ? (x >= 0 && x <= hi) : (x == 0 || x == 128 || x == 256 || x == 512));
        }
        if (ok) g_tune_cache[key] = v;
        pos = close + 1;
    }
}

static void tune_cache_store(const std::string &path) {
    if (path.empty()) return;
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos) {  // create the directory chain
        for (size_t p = 1; p <= slash; p++)
            if (path[p] == '/' || p == slash) mkdir(path.substr(0, p == slash ? slash : p).c_str(), 0755);
    }
    const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return;  // the cache is an optimisation: a read-only location just keeps it in memory
    std::fprintf(f, "{\n");
    size_t i = 0;
    for (const auto &kv : g_tune_cache) {
        std::fprintf(f, "  \"%s\": [", kv.first.c_str());
        for (size_t k = 0; k < kv.second.size(); k++) std::fprintf(f, "%s%d", k ? ", " : "", kv.second[k]);
        std::fprintf(f, "]%s\n", ++i < g_tune_cache.size() ? "," : "");
    }
    std::fprintf(f, "}\n");
    std::fclose(f);
    std::rename(tmp.c_str(), path.c_str());
}

static std::string grid_key(const gp5cu_plan *p) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, p->dev);
    std::string name(prop.name);
    for (char &ch : name)
        if (ch == '"' || ch == '|' || ch == '\\') ch = '_';
    return name + "|" + std::to_string(p->shape[0]) + "x" + std::to_string(p->shape[1]) + "x" +
           std::to_string(p->shape[2]) + "|c" + std::to_string(p->ncomp) + "|" + (p->prec == GP5_C128 ? "c128" : "c64");
}

static const char *kBuildStamp = "|build " __DATE__ " " __TIME__;  // another build tunes afresh

static std::vector<int> radix_vector(const gp5cu_plan *p) {
    std::vector<int> v(kTunedPasses + 1);
    for (int q = 0; q < kTunedPasses; q++) v[q] = p->radix[kTunedAxis[q]][kTunedMode[q]];
    v[kTunedPasses] = p->radix_boundary;
    return v;
}

static void apply_radix(gp5cu_plan *p, const std::vector<int> &v) {
    for (int q = 0; q < kTunedPasses; q++) p->radix[kTunedAxis[q]][kTunedMode[q]] = p->ax[kTunedAxis[q]].reg ? v[q] : 0;
    p->radix_boundary = p->ax[0].reg ? v[kTunedPasses] : 0;
}

static void apply_threads(gp5cu_plan *p, const std::vector<int> &v) {
    for (int q = 0; q < kTunedPasses; q++) {
        const int t = v[q];
        const int axis = kTunedAxis[q];
        const AxisPlan &ap = p->ax[axis];
        const int T = p->radix[axis][kTunedMode[q]] == 0 ? ap.reg_threads : ap.reg_threads1;
        p->tile_threads[axis][kTunedMode[q]] = (t != 0 && ap.reg && T > 0 && t % T == 0) ? t : 0;
    }
}

void autotune_plan(gp5cu_plan *p, bool force) {
    const char *env = std::getenv("GP5_AUTOTUNE");
    if (!force && env && std::string(env) == "0") return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const std::string path = tune_cache_path();
    if (!g_tune_loaded) {
        tune_cache_load(path);
        g_tune_loaded = true;
    }
    const std::string rkey = "radix|" + grid_key(p) + kBuildStamp;
    bool have_radix = false;
    const char *fixed = std::getenv("GP5_RADIX");
    if (fixed && (std::string(fixed) == "0" || std::string(fixed) == "1")) {
        apply_radix(p, std::vector<int>(kTunedPasses + 1, std::atoi(fixed)));
        const char *ring = std::getenv("GP5_RING");
        if (ring && std::string(ring) == "1" && p->ax[0].reg) p->radix_boundary |= 2;
        have_radix = true;
    } else {
        // a forced re-tune times the thread counts again but keeps the grid's schedules, so
        // that every plan of the grid keeps rounding the same way
        auto it = g_tune_cache.find(rkey);
        if (it != g_tune_cache.end()) {
            apply_radix(p, it->second);
            have_radix = true;
        }
    }
    auto thread_key = [&] {
        std::string r;
        for (int x : radix_vector(p)) r += std::to_string(x);
        return grid_key(p) + "|s" + std::to_string(p->nsolve) + "|r" + r + kBuildStamp;
    };
    if (have_radix && !force) {
        auto it = g_tune_cache.find(thread_key());
        if (it != g_tune_cache.end()) {
            apply_threads(p, it->second);
            return;
        }
    }
    if (p->prec == GP5_C128) Launch<double>::autotune(p, 3, !have_radix);
    else Launch<float>::autotune(p, 3, !have_radix);
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    if (!have_radix) g_tune_cache[rkey] = radix_vector(p);
    std::vector<int> v(kTunedPasses);
    for (int q = 0; q < kTunedPasses; q++) v[q] = p->tile_threads[kTunedAxis[q]][kTunedMode[q]];
    g_tune_cache[thread_key()] = v;
    tune_cache_store(path);
}

gp5cu_plan *create_plan(const int shape[3], const double *const *lefts, const double *const *rights, int nsolve,
                        int ncomp, int precision, int device) {
    require(ncomp == 1 || ncomp == 2, "ncomp must be 1 or 2");
    require(precision == GP5_C128 || precision == GP5_C64, "precision must be GP5_C128 or GP5_C64");
    require(nsolve >= 1 && nsolve <= 4096, "between 1 and 4096 solves per plan");
    for (int d = 0; d < 3; d++) require(shape[d] >= 2 && shape[d] <= 4096, "each axis length must be in [2, 4096]");
    for (int q = 0; q < nsolve; q++)
        for (int d = 0; d < 3; d++) require(rights[q][d] > lefts[q][d], "domain right must exceed left on every axis");
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    require(device >= 0 && device < ndev, "device ordinal out of range");
    gp5cu_plan *p = new gp5cu_plan();
    try {
        p->dev = device;
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        for (int d = 0; d < 3; d++) {
            p->shape[d] = shape[d];
            p->left[d] = lefts[0][d];
            p->right[d] = rights[0][d];
        }
        p->ncomp = ncomp;
        p->prec = precision;
        {
            const char *pdl = std::getenv("GP5_PDL");
            p->pdl = !(pdl && std::string(pdl) == "0");
            // defaults from the 256^3 step on a B200: the reversed boundary order saves 2% in
            // both precisions; the evict-first hints save another 2% in complex64 and cost 1%
            // in complex128
            const char *l2o = std::getenv("GP5_L2ORDER");
            p->l2_order = l2o ? std::string(l2o) == "1" : true;
            const char *sa = std::getenv("GP5_STREAM_AUX");
            p->stream_aux = sa ? std::string(sa) == "1" : precision == GP5_C64;
            // complex64 fields above L2 run their y/z passes on two x-slabs (measured 2% faster
            // at 256^3; complex128 and more slabs measured slower)
            const long long fbytes = (long long)shape[0] * shape[1] * shape[2] * ncomp *
                                     (precision == GP5_C128 ? 16LL : 8LL) * nsolve;
            if (precision == GP5_C64 && fbytes >= (100LL << 20) && shape[0] % 64 == 0) p->yz_slabs = 2;
            const char *yz = std::getenv("GP5_YZ_SLABS");
            if (yz) {
                const int v = std::atoi(yz);
                // slabs must split x evenly into whole tiles (x a power of two >= 32 per slab)
                if (v >= 1 && shape[0] % v == 0 && (shape[0] / v) % 32 == 0) p->yz_slabs = v;
            }
            const char *ks = std::getenv("GP5_KIN_SCHEME");
            if (ks && std::string(ks) == "1") p->kin_scheme = 1;
        }
        p->nsites = (long long)shape[0] * shape[1] * shape[2];
        p->nsolve = nsolve;
        p->solve_stride = p->nsites * ncomp;
        p->elem_bytes = precision == GP5_C128 ? 16 : 8;
        p->field_bytes = (size_t)p->nsites * ncomp * p->elem_bytes;
        p->sp_host.resize(nsolve);
        for (int q = 0; q < nsolve; q++) p->sp_host[q] = geometry_params(shape, lefts[q], rights[q]);
        p->dV = p->sp_host[0].dV;
        check_cuda(cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        p->stream = p->own_stream;
        for (int d = 0; d < 3; d++) build_axis_plan(p, d);
        check_cuda(cudaMalloc(&p->work, p->field_bytes * nsolve), "cudaMalloc work");
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        p->sms = sms;
        p->pw_blocks = sms * 8;
        p->pw_bps = std::max(1, p->pw_blocks / nsolve);
        // partial-sum slots per solve: the most blocks any kernel gives one solve (at worst one
        // line per tile)
        long long mb = p->pw_bps;
        for (int d = 0; d < 3; d++) {
            const long long lines_total = d == 0 ? (long long)shape[1] * shape[2] * ncomp
                                                 : (d == 1 ? (long long)shape[0] * shape[2] * ncomp
                                                           : (long long)shape[0] * shape[1] * ncomp);
            mb = std::max(mb, lines_total);
        }
        p->max_blocks = mb;
        check_cuda(cudaMalloc(&p->partials, sizeof(double) * kNRed * mb * nsolve), "cudaMalloc partials");
        check_cuda(cudaMalloc(&p->counter, sizeof(unsigned) * nsolve), "cudaMalloc counter");
        check_cuda(cudaMemset(p->counter, 0, sizeof(unsigned) * nsolve), "memset counter");
        check_cuda(cudaMalloc(&p->ds, sizeof(DevScalars) * nsolve), "cudaMalloc scalars");
        check_cuda(cudaMemset(p->ds, 0, sizeof(DevScalars) * nsolve), "memset scalars");
        check_cuda(cudaMalloc(&p->sp_lap, sizeof(SolveParams) * nsolve), "cudaMalloc params");
        check_cuda(cudaMemcpy(p->sp_lap, p->sp_host.data(), sizeof(SolveParams) * nsolve, cudaMemcpyHostToDevice),
                   "upload params");
        check_cuda(cudaMalloc(&p->dmax, sizeof(unsigned long long)), "cudaMalloc dmax");
        set_scalars(p->stream, p->ds, nsolve);
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
        autotune_plan(p, false);
    } catch (...) {
        gp5cu_plan_destroy(p);
        throw;
    }
    return p;
}

extern "C" {

int gp5cu_version(void) { return 10000; }

const char *gp5cu_status_string(int status) {
    switch (status) {
        case GP5_OK: return "ok";
        case GP5_ERR_ARG: return "invalid argument";
        case GP5_ERR_CUDA: return "CUDA error";
        case GP5_ERR_NONFINITE: return "non-finite value in a reduction";
        case GP5_ERR_TIMEOUT: return "device wait timed out";
        case GP5_ERR_UNSUPPORTED: return "unsupported";
        case GP5_ERR_STATE: return "invalid state";
        case GP5_ERR_NOMEM: return "out of device memory";
        case GP5_ERR_IO: return "file error";
        default: return "unknown status";
    }
}

const char *gp5cu_last_error(void) { return g_last_error.c_str(); }

int gp5cu_plan_create(gp5cu_plan **out, const int shape[3], const double left[3], const double right[3],
                      int ncomp, int precision, int device) {
    GP5_TRY
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    require(shape && left && right, "shape/left/right must not be NULL");
    *out = create_plan(shape, &left, &right, 1, ncomp, precision, device);
    GP5_CATCH
}

int gp5cu_plan_destroy(gp5cu_plan *p) {
    if (!p) return GP5_OK;
    cudaSetDevice(p->dev);
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (int d = 0; d < 3; d++) cudaFree(p->ax[d].tw);
    cudaFree(p->sp_lap);
    cudaFree(p->work);
    cudaFree(p->partials);
    cudaFree(p->counter);
    cudaFree(p->ds);
    cudaFree(p->dmax);
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
    delete p;
    return GP5_OK;
}

int gp5cu_plan_autotune(gp5cu_plan *p) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    use_device(p);
    autotune_plan(p, true);
    GP5_CATCH
}

int gp5cu_plan_get_tiles(const gp5cu_plan *p, int threads[5]) {
    GP5_TRY
    require(p != nullptr && threads != nullptr, "NULL argument");
    for (int q = 0; q < kTunedPasses; q++) threads[q] = p->tile_threads[kTunedAxis[q]][kTunedMode[q]];
    GP5_CATCH
}

int gp5cu_plan_set_tiles(gp5cu_plan *p, const int threads[5]) {
    GP5_TRY
    require(p != nullptr && threads != nullptr, "NULL argument");
    for (int q = 0; q < kTunedPasses; q++) {
        const int t = threads[q];
        require(t == 0 || t == 128 || t == 256 || t == 512, "tile threads must be 0, 128, 256 or 512");
        const AxisPlan &ap = p->ax[kTunedAxis[q]];
        const int T = p->radix[kTunedAxis[q]][kTunedMode[q]] == 0 ? ap.reg_threads : ap.reg_threads1;
        require(t == 0 || (ap.reg && t % T == 0), "tile threads do not fit this axis");
    }
    for (int q = 0; q < kTunedPasses; q++) p->tile_threads[kTunedAxis[q]][kTunedMode[q]] = threads[q];
    GP5_CATCH
}

int gp5cu_plan_get_radix(const gp5cu_plan *p, int radix[6]) {
    GP5_TRY
    require(p != nullptr && radix != nullptr, "NULL argument");
    for (int q = 0; q < kTunedPasses; q++) radix[q] = p->radix[kTunedAxis[q]][kTunedMode[q]];
    radix[kTunedPasses] = p->radix_boundary;
    GP5_CATCH
}

int gp5cu_plan_set_radix(gp5cu_plan *p, const int radix[6]) {
    GP5_TRY
    require(p != nullptr && radix != nullptr, "NULL argument");
    for (int q = 0; q < kTunedPasses; q++) require(radix[q] == 0 || radix[q] == 1, "radix schedules are 0 or 1");
    require(radix[kTunedPasses] >= 0 && radix[kTunedPasses] <= 3,
            "the stage boundary's choice is 0-3 (bit 0 schedule, bit 1 bulk-copy ring)");
    for (int q = 0; q < kTunedPasses; q++) {
        const int axis = kTunedAxis[q], mode = kTunedMode[q];
        const AxisPlan &ap = p->ax[axis];
        p->radix[axis][mode] = ap.reg ? radix[q] : 0;
        // a thread count that does not fit the new schedule falls back to the default shape
        const int T = p->radix[axis][mode] == 0 ? ap.reg_threads : ap.reg_threads1;
        if (p->tile_threads[axis][mode] != 0 && (T == 0 || p->tile_threads[axis][mode] % T != 0))
            p->tile_threads[axis][mode] = 0;
    }
    p->radix_boundary = p->ax[0].reg ? radix[kTunedPasses] : 0;
    GP5_CATCH
}

int gp5cu_plan_set_wait_bound(gp5cu_plan *p, unsigned long long ns) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    p->ring_wait_ns = ns;
    GP5_CATCH
}

int gp5cu_plan_set_stream(gp5cu_plan *p, void *stream) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    use_device(p);
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    p->stream = stream ? (cudaStream_t)stream : p->own_stream;
    GP5_CATCH
}

int gp5cu_plan_synchronize(gp5cu_plan *p) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    use_device(p);
    check_cuda(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
    GP5_CATCH
}

size_t gp5cu_field_bytes(const gp5cu_plan *p) { return p ? p->field_bytes : 0; }

int gp5cu_field_alloc(gp5cu_plan *p, void **dfield) {
    GP5_TRY
    require(p && dfield, "NULL argument");
    use_device(p);
    *dfield = nullptr;
    check_cuda(cudaMalloc(dfield, p->field_bytes), "cudaMalloc field");
    check_cuda(cudaMemsetAsync(*dfield, 0, p->field_bytes, p->stream), "memset field");
    GP5_CATCH
}

int gp5cu_field_free(gp5cu_plan *p, void *dfield) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    use_device(p);
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    check_cuda(cudaFree(dfield), "cudaFree");
    GP5_CATCH
}

int gp5cu_upload(gp5cu_plan *p, void *dfield, const void *host) {
    GP5_TRY
    require(p && host, "NULL argument");
    check_field_ptr(dfield, "dfield");
    use_device(p);
    check_cuda(cudaMemcpyAsync(dfield, host, p->field_bytes, cudaMemcpyHostToDevice, p->stream), "upload");
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    GP5_CATCH
}

int gp5cu_download(gp5cu_plan *p, const void *dfield, void *host) {
    GP5_TRY
    require(p && host, "NULL argument");
    check_field_ptr(dfield, "dfield");
    use_device(p);
    check_cuda(cudaMemcpyAsync(host, dfield, p->field_bytes, cudaMemcpyDeviceToHost, p->stream), "download");
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    GP5_CATCH
}

int gp5cu_upload_c128(gp5cu_plan *p, void *dfield, const double *host) {
    GP5_TRY
    require(p && host, "NULL argument");
    check_field_ptr(dfield, "dfield");
    use_device(p);
    if (p->prec == GP5_C128) return gp5cu_upload(p, dfield, host);
    const size_t n = (size_t)p->nsites * p->ncomp;
    double *tmp = nullptr;
    check_cuda(cudaMalloc(&tmp, n * 16), "cudaMalloc staging");
    try {
        check_cuda(cudaMemcpyAsync(tmp, host, n * 16, cudaMemcpyHostToDevice, p->stream), "upload");
        Launch<float>::convert(p, tmp, dfield, nullptr, nullptr, (long long)n);
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
    } catch (...) {
        cudaFree(tmp);
        throw;
    }
    cudaFree(tmp);
    GP5_CATCH
}

int gp5cu_download_c128(gp5cu_plan *p, const void *dfield, double *host) {
    GP5_TRY
    require(p && host, "NULL argument");
    check_field_ptr(dfield, "dfield");
    use_device(p);
    if (p->prec == GP5_C128) return gp5cu_download(p, dfield, host);
    const size_t n = (size_t)p->nsites * p->ncomp;
    double *tmp = nullptr;
    check_cuda(cudaMalloc(&tmp, n * 16), "cudaMalloc staging");
    try {
        Launch<float>::convert(p, nullptr, nullptr, dfield, tmp, (long long)n);
        check_cuda(cudaMemcpyAsync(host, tmp, n * 16, cudaMemcpyDeviceToHost, p->stream), "download");
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
    } catch (...) {
        cudaFree(tmp);
        throw;
    }
    cudaFree(tmp);
    GP5_CATCH
}

int gp5cu_fft(gp5cu_plan *p, const void *src, void *dst, int direction) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    check_field_ptr(src, "src");
    check_field_ptr(dst, "dst");
    require(direction == GP5_FORWARD || direction == GP5_BACKWARD, "direction must be GP5_FORWARD or GP5_BACKWARD");
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::fft(p, src, dst, direction); });
    GP5_CATCH
}

int gp5cu_laplacian(gp5cu_plan *p, const void *src, void *dst) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    check_field_ptr(src, "src");
    check_field_ptr(dst, "dst");
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::laplacian(p, src, dst); });
    GP5_CATCH
}

int gp5cu_norm(gp5cu_plan *p, const void *field, int comp, double *out) {
    GP5_TRY
    require(p && out, "NULL argument");
    check_field_ptr(field, "field");
    require(comp >= 0 && comp < p->ncomp, "component out of range");
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::norm(p, field, comp, 0.0, p->ds); });
    double s = 0;
    check_cuda(cudaMemcpyAsync(&s, &p->ds->sums[0], sizeof(double), cudaMemcpyDeviceToHost, p->stream), "read");
    sync_and_check(p, p->ds);
    *out = s * p->dV;
    GP5_CATCH
}

int gp5cu_normalize(gp5cu_plan *p, void *field, int comp, double N) {
    GP5_TRY
    require(p != nullptr, "plan is NULL");
    check_field_ptr(field, "field");
    require(comp >= 0 && comp < p->ncomp, "component out of range");
    require(N > 0, "normalisation must be positive");
    use_device(p);
    dispatch(p, [&](auto r) {
        Launch<decltype(r)>::norm(p, field, comp, N, p->ds);
        Launch<decltype(r)>::scale(p, field, comp, p->ds, false);
    });
    GP5_CATCH
}

int gp5cu_init_gaussian(gp5cu_plan *p, void *field, int comp, const double sigma[3]) {
    GP5_TRY
    require(p && sigma, "NULL argument");
    check_field_ptr(field, "field");
    require(comp >= 0 && comp < p->ncomp, "component out of range");
    require(p->nsolve == 1, "plan carries several solves");
    for (int q = 0; q < 3; q++) require(sigma[q] > 0 && std::isfinite(sigma[q]), "widths must be positive and finite");
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::init_gaussian(p, field, comp, sigma); });
    GP5_CATCH
}

int gp5cu_max_density(gp5cu_plan *p, const void *field, double *out) {
    GP5_TRY
    require(p && out, "NULL argument");
    check_field_ptr(field, "field");
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::max_density(p, field); });
    unsigned long long bits = 0;
    check_cuda(cudaMemcpyAsync(&bits, p->dmax, sizeof(bits), cudaMemcpyDeviceToHost, p->stream), "read");
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    double v;
    memcpy(&v, &bits, sizeof(v));
    *out = v;
    GP5_CATCH
}

void gp5cu_functional_desc_init(gp5cu_functional_desc *d) {
    if (!d) return;
    memset(d, 0, sizeof(*d));
    d->kind = GP5_FUNC_LHY;
    d->c3 = -3.0;
    d->c4 = 2.5;
    d->masses[0] = d->masses[1] = 1.0;
    d->potential = GP5_POT_NONE;
}

// Parameters of the functional on top of the plan's geometry, for every solve of the plan.
extern "C++" {
void fill_functional_params(const gp5cu_plan *p, const gp5cu_functional_desc &d, SolveParams &S) {
    for (int c = 0; c < 2; c++) {
        const double m = (d.kind == GP5_FUNC_GP && c < p->ncomp) ? d.masses[c] : 1.0;
        require(m > 0, "masses must be positive");
        // -1/2 (1/m) IFFT(-K^2 FFT)/N^3 = IFFT(K^2 FFT) * (0.5/m/N^3)
        S.kin[c] = 0.5 * (1.0 / m) / (double)p->nsites;
    }
    S.c3 = d.c3;
    S.c4 = d.c4;
    S.g00 = d.couplings[0];
    S.g01 = d.couplings[1];
    S.g11 = d.couplings[3];
    S.la = d.alpha;
    S.lb = d.beta;
    S.le = d.eta;
    for (int c = 0; c < 2; c++)
        for (int k = 0; k < 3; k++)  // w*w as in externalPotential.cpp:26
            S.om2[c][k] = (d.potential == GP5_POT_HARMONIC && c < p->ncomp) ? d.omegas[c][k] * d.omegas[c][k] : 0.0;
}
}  // extern "C++"

extern "C++" {
void upload_params(const std::vector<SolveParams> &h, SolveParams **dptr) {
    if (!*dptr) check_cuda(cudaMalloc(dptr, sizeof(SolveParams) * h.size()), "cudaMalloc params");
    check_cuda(cudaMemcpy(*dptr, h.data(), sizeof(SolveParams) * h.size(), cudaMemcpyHostToDevice), "upload params");
}
}  // extern "C++"

int gp5cu_functional_create(gp5cu_plan *p, const gp5cu_functional_desc *desc, gp5cu_functional **out) {
    GP5_TRY
    require(p && desc && out, "NULL argument");
    *out = nullptr;
    require(desc->kind >= GP5_FUNC_GP && desc->kind <= GP5_FUNC_LHY_UNLOCKED, "unknown functional kind");
    require(desc->kind != GP5_FUNC_LHY_UNLOCKED || p->ncomp == 2, "the unlocked LHY functional needs 2 components");
    require(desc->kind != GP5_FUNC_LHY || p->ncomp == 1, "the LHY droplet functional has 1 component");
    require(desc->potential >= GP5_POT_NONE && desc->potential <= GP5_POT_ARRAY, "unknown potential kind");
    require(desc->potential != GP5_POT_ARRAY || desc->dpotential != nullptr, "potential array is NULL");
    use_device(p);
    gp5cu_functional *f = new gp5cu_functional();
    f->plan = p;
    f->desc = *desc;
    try {
        f->sp_host = p->sp_host;
        for (auto &S : f->sp_host) fill_functional_params(p, *desc, S);
        upload_params(f->sp_host, &f->sp);
    } catch (...) {
        gp5cu_functional_destroy(f);
        throw;
    }
    *out = f;
    GP5_CATCH
}

int gp5cu_functional_destroy(gp5cu_functional *f) {
    if (!f) return GP5_OK;
    cudaSetDevice(f->plan->dev);
    cudaStreamSynchronize(f->plan->stream);
    cudaFree(f->sp);
    delete f;
    return GP5_OK;
}

int gp5cu_apply_H(gp5cu_functional *f, const void *src, void *dst) {
    GP5_TRY
    require(f != nullptr, "functional is NULL");
    check_field_ptr(src, "src");
    check_field_ptr(dst, "dst");
    require(src != dst, "src and dst must differ");
    gp5cu_plan *p = f->plan;
    use_device(p);
    dispatch(p, [&](auto r) { Launch<decltype(r)>::apply_h(f, src, dst, false); });
    GP5_CATCH
}

int gp5cu_observables(gp5cu_functional *f, const void *field, gp5cu_observables_t *out) {
    GP5_TRY
    require(f && out, "NULL argument");
    check_field_ptr(field, "field");
    gp5cu_plan *p = f->plan;
    use_device(p);
    set_scalars(p->stream, p->ds, p->nsolve);
    dispatch(p, [&](auto r) {
        // H psi lands in the workspace (read then written element by element by one thread)
        Launch<decltype(r)>::apply_h(f, field, p->work, true);
        Launch<decltype(r)>::residual(p, field, p->work, p->ds, f->sp);
    });
    double s[8];
    check_cuda(cudaMemcpyAsync(s, p->ds->sums, sizeof(s), cudaMemcpyDeviceToHost, p->stream), "read sums");
    sync_and_check(p, p->ds);
    const double dV = p->dV;
    out->norm = s[0] * dV;
    out->ekin = s[1] * dV;
    out->epot = s[2] * dV;
    out->eint = s[3] * dV;
    out->energy = out->ekin + out->epot + out->eint;
    out->mu = s[4] / s[0];
    out->residual = sqrt(s[5] / s[0]);
    GP5_CATCH
}

int gp5cu_stepper_create(gp5cu_functional *f, int kind, double dt, int imaginary, gp5cu_stepper **out) {
    GP5_TRY
    require(f && out, "NULL argument");
    *out = nullptr;
    require(kind == GP5_STEP_EULER || kind == GP5_STEP_RK4, "stepper kind must be GP5_STEP_EULER or GP5_STEP_RK4");
    require(std::isfinite(dt), "time step must be finite");
    gp5cu_plan *p = f->plan;
    use_device(p);
    gp5cu_stepper *st = new gp5cu_stepper();
    st->func = f;
    st->kind = kind;
    st->dt = dt;
    st->imaginary = imaginary ? 1 : 0;
    // gpCpp.cpp:217-224: (dt, 0) imaginary, (0, dt) real
    st->tre = imaginary ? dt : 0.0;
    st->tim = imaginary ? 0.0 : dt;
    st->sround = p->prec == GP5_C64;  // unbiased rounding of the complex64 state update
    try {
        check_cuda(cudaMalloc(&st->Ka, p->field_bytes * p->nsolve), "cudaMalloc k buffers");
        if (kind == GP5_STEP_RK4) check_cuda(cudaMalloc(&st->Kb, p->field_bytes * p->nsolve), "cudaMalloc k buffers");
        check_cuda(cudaMalloc(&st->ds, sizeof(DevScalars) * p->nsolve), "cudaMalloc scalars");
        check_cuda(cudaMemset(st->ds, 0, sizeof(DevScalars) * p->nsolve), "memset scalars");
        set_scalars(p->stream, st->ds, p->nsolve);
        st->sp_host = f->sp_host;
        for (auto &S : st->sp_host) {
            S.tre = st->tre;
            S.tim = st->tim;
        }
        upload_params(st->sp_host, &st->sp);
    } catch (...) {
        gp5cu_stepper_destroy(st);
        throw;
    }
    *out = st;
    GP5_CATCH
}

int gp5cu_stepper_destroy(gp5cu_stepper *st) {
    if (!st) return GP5_OK;
    cudaSetDevice(st->func->plan->dev);
    cudaStreamSynchronize(st->func->plan->stream);
    drop_graph(st);
    if (st->up) cudaStreamSynchronize(st->up);
    if (st->down) cudaStreamSynchronize(st->down);
    for (int b = 0; b < gp5cu_stepper::kHostStates; b++) {
        if (st->ev_up[b]) cudaEventDestroy(st->ev_up[b]);
        if (st->ev_done[b]) cudaEventDestroy(st->ev_done[b]);
        if (st->ev_down[b]) cudaEventDestroy(st->ev_down[b]);
    }
    if (st->up) cudaStreamDestroy(st->up);
    if (st->down) cudaStreamDestroy(st->down);
    cudaFree(st->Ka);
    cudaFree(st->Kb);
    cudaFree(st->T);
    cudaFree(st->ds);
    cudaFree(st->phase_exp);
    cudaFree(st->dstate);
    for (void *d : st->dstate_more) cudaFree(d);
    cudaFree(st->comp);
    cudaFree(st->sp);
    delete st;
    return GP5_OK;
}

extern "C++" {
void drop_graph(gp5cu_stepper *st) {
    if (st->exec) cudaGraphExecDestroy(st->exec);
    st->exec = nullptr;
    st->graph_field = nullptr;
    for (int a = 0; a < gp5cu_stepper::kAltGraphs; a++) {
        if (st->exec_alt[a]) cudaGraphExecDestroy(st->exec_alt[a]);
        st->exec_alt[a] = nullptr;
        st->graph_field_alt[a] = nullptr;
    }
}
}  // extern "C++"

int gp5cu_stepper_set_renormalization(gp5cu_stepper *st, int n, const double *N) {
    GP5_TRY
    require(st != nullptr, "stepper is NULL");
    const gp5cu_plan *p = st->func->plan;
    if (n == 0) {
        st->renorm = false;
    } else {
        require(N != nullptr, "N is NULL");
        require(n == p->ncomp, "one normalisation per component is required");
        for (int c = 0; c < n; c++) require(N[c] > 0, "normalisations must be positive");
        st->renorm = true;
        st->N[0] = N[0];
        st->N[1] = n > 1 ? N[1] : 0.0;
    }
    for (auto &S : st->sp_host) {
        S.Nt[0] = st->renorm ? st->N[0] : 0.0;
        S.Nt[1] = st->renorm ? st->N[1] : 0.0;
    }
    upload_params(st->sp_host, &st->sp);
    drop_graph(st);
    GP5_CATCH
}

int gp5cu_stepper_set_compensation(gp5cu_stepper *st, int on) {
    GP5_TRY
    require(st != nullptr, "stepper is NULL");
    gp5cu_plan *p = st->func->plan;
    if (on) require(p->prec == GP5_C64, "the compensated update is for complex64 plans");
    use_device(p);
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    drop_graph(st);
    if (on) {
        const size_t bytes = p->field_bytes / 2 * (size_t)p->nsolve;  // BF16 pair per element
        if (!st->comp) check_cuda(cudaMalloc(&st->comp, bytes), "cudaMalloc compensation");
        check_cuda(cudaMemset(st->comp, 0, bytes), "memset compensation");
        st->compensate = true;
    } else {
        cudaFree(st->comp);
        st->comp = nullptr;
        st->compensate = false;
    }
    st->comp_field = nullptr;
    GP5_CATCH
}

int gp5cu_stepper_set_stochastic_rounding(gp5cu_stepper *st, int on) {
    GP5_TRY
    require(st != nullptr, "stepper is NULL");
    gp5cu_plan *p = st->func->plan;
    if (on) require(p->prec == GP5_C64, "stochastic rounding is for complex64 plans");
    use_device(p);
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    drop_graph(st);
    st->sround = on != 0;
    GP5_CATCH
}

int gp5cu_stepper_set_phase_constraint(gp5cu_stepper *st, const void *dphase) {
    GP5_TRY
    require(st != nullptr, "stepper is NULL");
    gp5cu_plan *p = st->func->plan;
    use_device(p);
    drop_graph(st);
    if (!dphase) {
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
        cudaFree(st->phase_exp);
        st->phase_exp = nullptr;
    } else {
        check_field_ptr(dphase, "dphase");
        if (!st->phase_exp) check_cuda(cudaMalloc(&st->phase_exp, p->field_bytes), "cudaMalloc phase");
        dispatch(p, [&](auto r) { Launch<decltype(r)>::phase_exp(p, dphase, st->phase_exp); });
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
    }
    GP5_CATCH
}

// The merged stage-boundary path runs when one component is stepped and the x axis uses the
// register engine; otherwise each stage is five passes with separate prologue/epilogue.
extern "C++" {
bool merged_path(const gp5cu_plan *p) { return p->ncomp == 1 && p->ax[0].reg; }
}  // extern "C++"

extern "C++" {
int queue_step(gp5cu_stepper *st, void *field, bool merged, bool prologue) {
    int n = 0;
    dispatch(st->func->plan, [&](auto r) {
        n = merged ? Launch<decltype(r)>::step_merged(st, field, prologue) : Launch<decltype(r)>::step(st, field);
    });
    return n;
}
}  // extern "C++"

// Captures ksteps steps into a CUDA graph bound to this field; kernels are configured in a dry
// pass first so that no attribute call happens during the capture.
extern "C++" {
void build_graph(gp5cu_stepper *st, void *field, bool merged, int ksteps) {
    gp5cu_plan *p = st->func->plan;
    drop_graph(st);
    capture_graph(st, field, merged, ksteps);
}

// Captures into the primary graph slot only (the alternate slot is kept).
void capture_graph(gp5cu_stepper *st, void *field, bool merged, int ksteps) {
    gp5cu_plan *p = st->func->plan;
    if (st->exec) cudaGraphExecDestroy(st->exec);
    st->exec = nullptr;
    st->graph_field = nullptr;
    p->dry = true;
    try {
        queue_step(st, field, merged, false);
    } catch (...) {
        p->dry = false;
        throw;
    }
    p->dry = false;
    cudaGraph_t g = nullptr;
    check_cuda(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int n = 0;
    try {
        for (int k = 0; k < ksteps; k++) n = queue_step(st, field, merged, false);
    } catch (...) {
        cudaStreamEndCapture(p->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(p->stream, &g), "end capture");
    cudaError_t e = cudaGraphInstantiate(&st->exec, g, 0);
    cudaGraphDestroy(g);
    check_cuda(e, "cudaGraphInstantiate");
    st->graph_field = field;
    st->graph_merged = merged;
    st->graph_steps = ksteps;
    st->launches_per_step = n;
}
}  // extern "C++"

// Queues nsteps steps of `field` on the plan stream (no synchronisation).  The three most
// recent fields keep their captured one-step graphs.
static void enqueue_advance(gp5cu_stepper *st, void *field, int nsteps) {
    gp5cu_plan *p = st->func->plan;
    const bool merged = merged_path(p);
    if (compensation_active(st) && st->comp_field != field) {
        // the correction belongs to one state: a new state starts from zero
        check_cuda(cudaMemsetAsync(st->comp, 0, p->field_bytes / 2 * (size_t)p->nsolve, p->stream), "memset");
        st->comp_field = field;
    }
    auto fits = [&](cudaGraphExec_t e, void *f, bool m, int k) { return e && f == field && m == merged && k == 1; };
    if (!fits(st->exec, st->graph_field, st->graph_merged, st->graph_steps)) {
        constexpr int NA = gp5cu_stepper::kAltGraphs;
        int hit = -1;
        for (int a = 0; a < NA && hit < 0; a++)
            if (fits(st->exec_alt[a], st->graph_field_alt[a], st->graph_merged_alt[a], st->graph_steps_alt[a])) hit = a;
        // least recently used last: a hit leaves its slot, a miss drops the last one
        const int from = hit >= 0 ? hit : NA - 1;
        cudaGraphExec_t e = st->exec_alt[from];
        void *f = st->graph_field_alt[from];
        const bool m = st->graph_merged_alt[from];
        const int k = st->graph_steps_alt[from];
        if (hit < 0 && e) cudaGraphExecDestroy(e);
        for (int a = from; a > 0; a--) {
            st->exec_alt[a] = st->exec_alt[a - 1];
            st->graph_field_alt[a] = st->graph_field_alt[a - 1];
            st->graph_merged_alt[a] = st->graph_merged_alt[a - 1];
            st->graph_steps_alt[a] = st->graph_steps_alt[a - 1];
        }
        st->exec_alt[0] = st->exec;
        st->graph_field_alt[0] = st->graph_field;
        st->graph_merged_alt[0] = st->graph_merged;
        st->graph_steps_alt[0] = st->graph_steps;
        st->exec = nullptr;
        st->graph_field = nullptr;
        if (hit >= 0) {
            st->exec = e;
            st->graph_field = f;
            st->graph_merged = m;
            st->graph_steps = k;
        } else {
            capture_graph(st, field, merged, 1);
        }
    }
    set_scalars(p->stream, st->ds, p->nsolve);
    if (merged) {
        // forward x transform of psi, consumed by the first graph step
        p->dry = false;
        dispatch(p, [&](auto r) { Launch<decltype(r)>::prologue(st, field); });
    }
    for (int i = 0; i < nsteps; i++) {
        check_cuda(cudaGraphLaunch(st->exec, p->stream), "cudaGraphLaunch");
        st->t += st->dt;
    }
    if (st->renorm) {
        // materialise the pending normalisation of the last step (stepper.cpp:67)
        dispatch(p, [&](auto r) { Launch<decltype(r)>::scale(p, field, -1, st->ds, true); });
    }
}

int gp5cu_stepper_advance(gp5cu_stepper *st, void *field, int nsteps) {
    GP5_TRY
    require(st != nullptr, "stepper is NULL");
    check_field_ptr(field, "field");
    require(nsteps >= 0, "nsteps must be >= 0");
    gp5cu_plan *p = st->func->plan;
    use_device(p);
    if (nsteps == 0) return GP5_OK;
    enqueue_advance(st, field, nsteps);
    sync_and_check(p, st->ds);
    GP5_CATCH
}

int gp5cu_stepper_get_time(const gp5cu_stepper *st, double *t) {
    if (!st || !t) {
        set_last_error("NULL argument");
        return GP5_ERR_ARG;
    }
    *t = st->t;
    return GP5_OK;
}

int gp5cu_stepper_set_time(gp5cu_stepper *st, double t) {
    if (!st) {
        set_last_error("stepper is NULL");
        return GP5_ERR_ARG;
    }
    st->t = t;
    return GP5_OK;
}

int gp5cu_stepper_advance_host(gp5cu_stepper *st, const void *host_in, void *host_out, int nsteps) {
    GP5_TRY
    require(st && host_in && host_out, "NULL argument");
    require(nsteps >= 0, "nsteps must be >= 0");
    gp5cu_plan *p = st->func->plan;
    use_device(p);
    if (!st->dstate) check_cuda(cudaMalloc(&st->dstate, p->field_bytes), "cudaMalloc state");
    check_cuda(cudaMemcpyAsync(st->dstate, host_in, p->field_bytes, cudaMemcpyHostToDevice, p->stream), "upload");
    st->comp_field = nullptr;  // a new state: its correction starts from zero
    const int rc = gp5cu_stepper_advance(st, st->dstate, nsteps);
    if (rc != GP5_OK) return rc;
    check_cuda(cudaMemcpyAsync(host_out, st->dstate, p->field_bytes, cudaMemcpyDeviceToHost, p->stream), "download");
    check_cuda(cudaStreamSynchronize(p->stream), "sync");
    GP5_CATCH
}

int gp5cu_stepper_advance_host_many(gp5cu_stepper *st, int nstates, const void *const *host_in,
                                    void *const *host_out, int nsteps) {
    GP5_TRY
    require(st && host_in && host_out, "NULL argument");
    require(nstates >= 0 && nsteps >= 0, "nstates and nsteps must be >= 0");
    for (int i = 0; i < nstates; i++) require(host_in[i] && host_out[i], "NULL host buffer");
    gp5cu_plan *p = st->func->plan;
    require(p->nsolve == 1, "host-buffer stepping needs a single-solve plan");
    use_device(p);
    if (nstates == 0) return GP5_OK;
    const size_t fb = p->field_bytes;
    constexpr int NB = gp5cu_stepper::kHostStates;
    // as many device states as there are host states, up to NB
    const int nbuf = nstates < NB ? nstates : NB;
    if (!st->dstate) check_cuda(cudaMalloc(&st->dstate, fb), "cudaMalloc state");
    for (int b = 1; b < nbuf; b++)
        if (!st->dstate_more[b - 1]) check_cuda(cudaMalloc(&st->dstate_more[b - 1], fb), "cudaMalloc state");
    if (!st->up) {
        check_cuda(cudaStreamCreateWithFlags(&st->up, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaStreamCreateWithFlags(&st->down, cudaStreamNonBlocking), "cudaStreamCreate");
        for (int b = 0; b < NB; b++) {
            check_cuda(cudaEventCreateWithFlags(&st->ev_up[b], cudaEventDisableTiming), "cudaEventCreate");
            check_cuda(cudaEventCreateWithFlags(&st->ev_done[b], cudaEventDisableTiming), "cudaEventCreate");
            check_cuda(cudaEventCreateWithFlags(&st->ev_down[b], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
    void *dbuf[NB] = {st->dstate};
    for (int b = 1; b < NB; b++) dbuf[b] = st->dstate_more[b - 1];
    // the plan stream's earlier work (for example the last call's steps) comes first
    check_cuda(cudaEventRecord(st->ev_done[0], p->stream), "cudaEventRecord");
    check_cuda(cudaStreamWaitEvent(st->up, st->ev_done[0], 0), "cudaStreamWaitEvent");
    double t_after = st->t;
    for (int i = 0; i < nstates; i++) {
        const int b = i % nbuf;
        // buffer b is free once state i-nbuf has been downloaded from it
        if (i >= nbuf) check_cuda(cudaStreamWaitEvent(st->up, st->ev_down[b], 0), "cudaStreamWaitEvent");
        check_cuda(cudaMemcpyAsync(dbuf[b], host_in[i], fb, cudaMemcpyHostToDevice, st->up), "upload");
        check_cuda(cudaEventRecord(st->ev_up[b], st->up), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(p->stream, st->ev_up[b], 0), "cudaStreamWaitEvent");
        st->comp_field = nullptr;  // a new state: its compensation starts from zero
        const double t0 = st->t;
        if (nsteps > 0) enqueue_advance(st, dbuf[b], nsteps);
        if (i == 0) t_after = st->t;
        st->t = t0;
        check_cuda(cudaEventRecord(st->ev_done[b], p->stream), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(st->down, st->ev_done[b], 0), "cudaStreamWaitEvent");
        check_cuda(cudaMemcpyAsync(host_out[i], dbuf[b], fb, cudaMemcpyDeviceToHost, st->down), "download");
        check_cuda(cudaEventRecord(st->ev_down[b], st->down), "cudaEventRecord");
    }
    check_cuda(cudaStreamSynchronize(st->down), "sync");
    sync_and_check(p, st->ds);
    st->t = t_after;  // the states are independent: the stepper's time advances once
    GP5_CATCH
}

int gp5cu_stepper_launches_per_step(const gp5cu_stepper *st) { return st ? st->launches_per_step : 0; }

int gp5cu_stepper_profile(gp5cu_stepper *st, void *field, int nrep, double *ms, int *kinds, int cap,
                          int *nlaunch) {
    GP5_TRY
    require(st && ms && kinds && nlaunch, "NULL argument");
    check_field_ptr(field, "field");
    require(nrep >= 1, "nrep must be >= 1");
    gp5cu_plan *p = st->func->plan;
    use_device(p);
    ProfRec rec;
    p->prof = &rec;
    try {
        set_scalars(p->stream, st->ds, p->nsolve);
        const bool merged = merged_path(p);
        if (merged) {
            p->prof = nullptr;
            dispatch(p, [&](auto r) { Launch<decltype(r)>::prologue(st, field); });
            p->prof = &rec;
        }
        std::vector<double> acc;
        int n = 0;
        for (int r = 0; r < nrep; r++) {
            rec.idx = 0;
            rec.record(p->stream, -1);
            n = queue_step(st, field, merged, false);
            st->t += st->dt;
            check_cuda(cudaStreamSynchronize(p->stream), "sync");
            if (acc.empty()) acc.assign(rec.idx - 1, 0.0);
            for (size_t i = 1; i < rec.idx; i++) {
                float t = 0;
                check_cuda(cudaEventElapsedTime(&t, rec.ev[i - 1], rec.ev[i]), "cudaEventElapsedTime");
                acc[i - 1] += t;
            }
        }
        (void)n;
        const int m = (int)acc.size();
        *nlaunch = m;
        for (int i = 0; i < m && i < cap; i++) {
            ms[i] = acc[i] / nrep;
            kinds[i] = rec.kinds[i + 1];
        }
        if (st->renorm) dispatch(p, [&](auto r) { Launch<decltype(r)>::scale(p, field, -1, st->ds, true); });
        sync_and_check(p, st->ds);
    } catch (...) {
        p->prof = nullptr;
        for (auto e : rec.ev) cudaEventDestroy(e);
        throw;
    }
    p->prof = nullptr;
    for (auto e : rec.ev) cudaEventDestroy(e);
    GP5_CATCH
}

}  // extern "C"

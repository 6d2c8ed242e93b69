// launch_impl.cuh - precision-templated launchers: tile geometry, engine dispatch and the
// kernel sequences of the transforms, the H application and one stepper step.
// Included once per precision (gp5cu_f64.cu, gp5cu_f32.cu).
#pragma once

#include <algorithm>
#include <cstdio>
#include <utility>

#include "ops.cuh"
#include "plan.hpp"
#include "ring.cuh"

namespace gp5 {

constexpr int kThreads = 256;

inline TileGeom make_geom(const gp5cu_plan *p, int axis, int lines, bool pow2_bx, long long *tiles) {
    TileGeom g{};
    g.nx = p->shape[0];
    g.ny = p->shape[1];
    g.nz = p->shape[2];
    g.nc = p->ncomp;
    g.axis = axis;
    g.n = p->shape[axis];
    g.estride = axis == 0 ? 1 : (axis == 1 ? (long long)g.nx : (long long)g.nx * g.ny);
    long long tps = 0;
    if (axis == 0) {
        g.lines = lines;
        g.bx = g.bo = 1;
        g.tiles_x = 1;
        g.n_other = (long long)g.ny * g.nz * g.nc;
        tps = (g.n_other + lines - 1) / lines;
    } else {
        int bx = std::min(lines, g.nx);
        if (pow2_bx) {
            int b = 1;
            while (b * 2 <= bx) b *= 2;
            bx = b;
        }
        const int bo = lines / bx;
        g.lines = bx * bo;
        g.bx = bx;
        g.bo = bo;
        // the plan's x range (a slab of consecutive x values, or all of them)
        g.x0 = p->xr_n > 0 ? p->xr0 : 0;
        g.xend = p->xr_n > 0 ? p->xr0 + p->xr_n : g.nx;
        g.tiles_x = (g.xend - g.x0 + bx - 1) / bx;
        g.n_other = axis == 1 ? (long long)g.nz * g.nc : (long long)g.ny * g.nc;
        tps = (long long)g.tiles_x * ((g.n_other + bo - 1) / bo);
    }
    g.nsolve = p->nsolve;
    g.tiles_per_solve = tps;
    g.solve_stride = p->solve_stride;
    g.ntiles = tps * p->nsolve;
    *tiles = g.ntiles;
    return g;
}
inline RedSlot red_slot(const gp5cu_plan *p) { return RedSlot{p->partials, p->counter}; }

// Opt a kernel in to more than 48 KB of dynamic shared memory, once per (kernel, device,
// size); the bookkeeping is keyed by the kernel's address.
void smem_opt_in(const void *kernel, size_t bytes, int dev);

// CTAs of a kernel resident per SM (cached per kernel and device).
int resident_blocks(const void *kernel, int threads, size_t smem, int dev);

// Launch on the plan's stream with programmatic stream serialisation (unless the plan turned
// it off): in a captured graph the launch gets a programmatic edge from its predecessor, and
// the kernel's pdl_enter() keeps every read behind the predecessor's completion.
template <typename... KArgs, typename... Args>
inline void launch_k(const gp5cu_plan *p, void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem,
                     Args &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = p->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = p->pdl ? 1 : 0;
    check_cuda(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...), "kernel launch");
}

template <class K> inline void ensure_smem(K kernel, size_t bytes, int dev) {
    if (bytes > 48 * 1024) smem_opt_in((const void *)kernel, bytes, dev);
}

template <typename Real, int N, bool CONTIG, int MODE, class Op, int TH, int S>
void launch_reg_th(gp5cu_plan *p, int axis, const Op &op) {
    using V = cpx<Real>;
    constexpr int LINES = RegTile<Real, N, CONTIG, MODE, TH, S>::LINES,
                  THREADS = RegTile<Real, N, CONTIG, MODE, TH, S>::THREADS;
    long long tiles = 0;
    TileGeom g = make_geom(p, axis, LINES, true, &tiles);
    g.reverse = (MODE == MODE_INV_TURN_FWD && p->l2_order) ? 1 : 0;
    const size_t smem = CONTIG ? (size_t)LINES * LayContig<N, S>::LD * sizeof(V) : (size_t)LINES * N * sizeof(V);
    auto kern = k_axis_reg<Real, N, CONTIG, MODE, Op, TH, S>;
    ensure_smem(kern, smem, p->dev);
    if (p->dry) return;
    launch_k(p, kern, (unsigned)tiles, THREADS, smem, g, op, (const V *)p->ax[axis].tw, red_slot(p));
    if (p->prof) p->prof->record(p->stream, axis * 10 + MODE);
}

// Tile shapes of the strided (y/z) passes: the plan's autotuned threads per CTA (0: the
// default rule of RegTile).  These passes carry no reductions, so the thread count does not
// change any result bit.
template <typename Real, int N, bool CONTIG, int MODE, class Op, int S>
void launch_reg_s(gp5cu_plan *p, int axis, const Op &op) {
    if constexpr (!CONTIG && (MODE == MODE_FWD || MODE == MODE_INV || MODE == MODE_FWD_MID_INV)) {
        constexpr int T = RegCfgAll<N, S>::T, DEF = RegTile<Real, N, CONTIG, MODE, 0, S>::THREADS;
        switch (p->tile_threads[axis][MODE]) {
            case 128: if constexpr (128 % T == 0 && DEF != 128) { launch_reg_th<Real, N, CONTIG, MODE, Op, 128, S>(p, axis, op); return; } break;
            case 256: if constexpr (256 % T == 0 && DEF != 256) { launch_reg_th<Real, N, CONTIG, MODE, Op, 256, S>(p, axis, op); return; } break;
            case 512: if constexpr (512 % T == 0 && DEF != 512) { launch_reg_th<Real, N, CONTIG, MODE, Op, 512, S>(p, axis, op); return; } break;
            default: break;
        }
    }
    launch_reg_th<Real, N, CONTIG, MODE, Op, 0, S>(p, axis, op);
}

// The stage boundary on the bulk-copy ring (ring.cuh): one persistent CTA per SM (its shared
// memory holds the ring).  Returns false when the ring does not serve this configuration
// (tile shape, or the compensated complex64 update, whose BF16 stream is not staged).
template <typename Real, int N, int S, class Op> bool launch_ring(gp5cu_plan *, const Op &) { return false; }
template <typename Real, int N, int S, bool RED>
bool launch_ring(gp5cu_plan *p, const OpStageOut<Real, RED, true> &op) {
    using RT = RingTile<Real, N, S>;
    if constexpr (!RT::OK) {
        return false;
    } else {
        if (op.P.comp) return false;
        long long tiles = 0;
        TileGeom g = make_geom(p, 0, RT::LINES, true, &tiles);
        g.reverse = p->l2_order ? 1 : 0;
        auto kern = k_boundary_ring<Real, N, S, RED>;
        ensure_smem(kern, RT::SMEM, p->dev);
        if (p->dry) return true;
        const unsigned grid = (unsigned)std::min<long long>(tiles, p->sms);
        launch_k(p, kern, grid, RT::THREADS, RT::SMEM, g, op, (const cpx<Real> *)p->ax[0].tw, red_slot(p),
                 p->ring_wait_ns);
        if (p->prof) p->prof->record(p->stream, MODE_INV_TURN_FWD);
        return true;
    }
}

// Radix schedule: the plan's choice for the strided passes and for the stage boundary (the
// other x passes keep schedule 0).  The boundary's choice also selects its operand feed: bit 0
// the schedule, bit 1 the bulk-copy ring instead of register loads.
template <typename Real, int N, bool CONTIG, int MODE, class Op>
void launch_reg(gp5cu_plan *p, int axis, const Op &op) {
    if constexpr (MODE == MODE_INV_TURN_FWD) {
        if (p->radix_boundary & 2) {
            if ((p->radix_boundary & 1) ? launch_ring<Real, N, 1>(p, op) : launch_ring<Real, N, 0>(p, op)) return;
        }
    }
    if constexpr (!CONTIG || MODE == MODE_INV_TURN_FWD) {
        const int s = MODE == MODE_INV_TURN_FWD ? (p->radix_boundary & 1) : p->radix[axis][MODE];
        if (s == 1) {
            launch_reg_s<Real, N, CONTIG, MODE, Op, 1>(p, axis, op);
            return;
        }
    }
    launch_reg_s<Real, N, CONTIG, MODE, Op, 0>(p, axis, op);
}

template <typename Real, bool CONTIG, int MODE, class Op>
void launch_smem(gp5cu_plan *p, int axis, const Op &op) {
    using V = cpx<Real>;
    const AxisPlan &ap = p->ax[axis];
    long long tiles = 0;
    TileGeom g = make_geom(p, axis, ap.smem_lines, false, &tiles);
    const int ld = CONTIG ? g.n + 1 : g.lines;
    const size_t bufsz = CONTIG ? (size_t)g.lines * ld : (size_t)g.lines * g.n;
    const size_t smem = 2 * bufsz * sizeof(V);
    auto kern = k_axis_smem<Real, CONTIG, MODE, Op>;
    ensure_smem(kern, smem, p->dev);
    if (p->dry) return;
    launch_k(p, kern, (unsigned)tiles, kThreads, smem, g, ap.sched, op, (const V *)ap.tw, red_slot(p));
    if (p->prof) p->prof->record(p->stream, axis * 10 + MODE);
}

template <typename Real, bool CONTIG, int MODE, class Op>
void launch_axis(gp5cu_plan *p, int axis, const Op &op) {
    const AxisPlan &ap = p->ax[axis];
    if constexpr (MODE == MODE_INV_TURN_FWD) {
        // the stage-boundary kernel exists for the register engine only
        switch (ap.n) {
            case 32: launch_reg<Real, 32, CONTIG, MODE>(p, axis, op); return;
            case 64: launch_reg<Real, 64, CONTIG, MODE>(p, axis, op); return;
            case 128: launch_reg<Real, 128, CONTIG, MODE>(p, axis, op); return;
            case 256: launch_reg<Real, 256, CONTIG, MODE>(p, axis, op); return;
            case 512: launch_reg<Real, 512, CONTIG, MODE>(p, axis, op); return;
            default: fail(GP5_ERR_UNSUPPORTED, "stage boundary kernel needs a power-of-two x axis in [32, 512]");
        }
    }
    if (ap.reg) {
        switch (ap.n) {
            case 32: launch_reg<Real, 32, CONTIG, MODE>(p, axis, op); return;
            case 64: launch_reg<Real, 64, CONTIG, MODE>(p, axis, op); return;
            case 128: launch_reg<Real, 128, CONTIG, MODE>(p, axis, op); return;
            case 256: launch_reg<Real, 256, CONTIG, MODE>(p, axis, op); return;
            case 512: launch_reg<Real, 512, CONTIG, MODE>(p, axis, op); return;
            default: break;
        }
    }
    launch_smem<Real, CONTIG, MODE>(p, axis, op);
}

// Point-wise kernel over the sites of every solve: pw_bps blocks per solve.
template <class Op> void launch_pointwise(gp5cu_plan *p, const Op &op) {
    if (p->dry) return;
    launch_k(p, k_pointwise<Op>, (unsigned)(p->pw_bps * p->nsolve), kThreads, 0, p->nsites, p->pw_bps, op,
             red_slot(p));
    if (p->prof) p->prof->record(p->stream, 90);
}

template <typename Real>
__global__ void __launch_bounds__(256) k_max_density(const cpx<Real> *f, long long nsites, int ncomp,
                                                     unsigned long long *out) {
    double m = 0.0;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nsites;
         s += (long long)gridDim.x * blockDim.x) {
        for (int c = 0; c < ncomp; c++) {
            const cpx<Real> v = f[s + (long long)c * nsites];
            const double n = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
            m = fmax(m, n);
        }
    }
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    __shared__ double wm[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wm[w] = m;
    __syncthreads();
    if (w == 0) {
        m = lane < (int)(blockDim.x >> 5) ? wm[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
        if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// psi_c = exp(-(ax x^2 + ay y^2 + az z^2)) + 0i at the cell centres x = left + (i + 1/2) dx
// (initGaussian, src/geometry.cpp:251-276); arithmetic in FP64, rounded to Real once.
template <typename Real>
__global__ void __launch_bounds__(256) k_init_gaussian(cpx<Real> *f, int nx, int ny, long long nsites, double x0,
                                                       double y0, double z0, double dx, double dy, double dz,
                                                       double ax, double ay, double az) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nsites;
         s += (long long)gridDim.x * blockDim.x) {
        const long long jk = s / nx;
        const int i = (int)(s - jk * nx), j = (int)(jk % ny), k = (int)(jk / ny);
        // uncontracted, in the reference's order: only exp() rounds differently from the host
        const double x = __dadd_rn(x0, __dmul_rn(i + 0.5, dx)), y = __dadd_rn(y0, __dmul_rn(j + 0.5, dy)),
                     z = __dadd_rn(z0, __dmul_rn(k + 0.5, dz));
        const double t = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(ax, x), x), __dmul_rn(__dmul_rn(ay, y), y)),
                                   __dmul_rn(__dmul_rn(az, z), z));
        f[s] = mk<Real>((Real)exp(-t), (Real)0);
    }
}

template <typename Real>
__global__ void __launch_bounds__(256) k_phase_exp(const Real *phase, cpx<Real> *out, long long n) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        Real sn, cs;
        sincos(phase[s], &sn, &cs);
        out[s] = mk<Real>(cs, sn);
    }
}

// ---- transforms ----------------------------------------------------------------------------
template <typename Real> void Launch<Real>::fft(gp5cu_plan *p, const void *src, void *dst, int dir) {
    using V = cpx<Real>;
    const V *s = (const V *)src;
    V *d = (V *)dst;
    if (dir == GP5_FORWARD) {
        OpStageIn<Real, false> in{s, nullptr, d, p->ds, p->sp_lap, 0, 0.0, 1};
        launch_axis<Real, true, MODE_FWD>(p, 0, in);
        OpCopy<Real> cp{d, d, nullptr};
        launch_axis<Real, false, MODE_FWD>(p, 1, cp);
        launch_axis<Real, false, MODE_FWD>(p, 2, cp);
    } else {
        OpCopy<Real> first{s, d, nullptr};
        launch_axis<Real, true, MODE_INV>(p, 0, first);
        OpCopy<Real> cp{d, d, nullptr};
        launch_axis<Real, false, MODE_INV>(p, 1, cp);
        launch_axis<Real, false, MODE_INV>(p, 2, cp);
    }
}

// x fwd, y fwd, z fwd * K^2 kin * z inv, y inv; the x inverse is left to the caller.
template <typename Real>
static void kinetic_passes(gp5cu_plan *p, const void *src, void *w, const SolveParams *sp, DevScalars *ds) {
    using V = cpx<Real>;
    OpStageIn<Real, false> in{(const V *)src, nullptr, (V *)w, ds, sp, 0, 0.0, 1};
    launch_axis<Real, true, MODE_FWD>(p, 0, in);
    OpCopy<Real> cp{(const V *)w, (V *)w, p->nsolve > 1 ? sp : nullptr};
    launch_axis<Real, false, MODE_FWD>(p, 1, cp);
    OpKinetic<Real> kin{(const V *)w, (V *)w, sp, p->shape[0], p->shape[1], p->shape[2]};
    launch_axis<Real, false, MODE_FWD_MID_INV>(p, 2, kin);
    launch_axis<Real, false, MODE_INV>(p, 1, cp);
}

// whether the ring kernel has a tile shape for the plan's x length and schedule s
template <typename Real> bool ring_serves(const gp5cu_plan *p, int s) {
    if (!p->ax[0].reg) return false;
    switch (p->shape[0]) {
        case 32: return s ? RingTile<Real, 32, 1>::OK : RingTile<Real, 32, 0>::OK;
        case 64: return s ? RingTile<Real, 64, 1>::OK : RingTile<Real, 64, 0>::OK;
        case 128: return s ? RingTile<Real, 128, 1>::OK : RingTile<Real, 128, 0>::OK;
        case 256: return s ? RingTile<Real, 256, 1>::OK : RingTile<Real, 256, 0>::OK;
        case 512: return s ? RingTile<Real, 512, 1>::OK : RingTile<Real, 512, 0>::OK;
        default: return false;
    }
}

template <typename Real> void Launch<Real>::autotune(gp5cu_plan *p, int nrep, bool radix) {
    using V = cpx<Real>;
    V *w = (V *)p->work;
    check_cuda(cudaMemsetAsync(w, 0, p->field_bytes * p->nsolve, p->stream), "memset work");
    OpCopy<Real> cp{w, w, p->nsolve > 1 ? p->sp_lap : nullptr};
    OpKinetic<Real> kin{w, w, p->sp_lap, p->shape[0], p->shape[1], p->shape[2]};
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    auto run = [&](int q) {
        const int axis = kTunedAxis[q];
        switch (kTunedMode[q]) {
            case MODE_FWD: launch_axis<Real, false, MODE_FWD>(p, axis, cp); break;
            case MODE_INV: launch_axis<Real, false, MODE_INV>(p, axis, cp); break;
            default: launch_axis<Real, false, MODE_FWD_MID_INV>(p, axis, kin); break;
        }
    };
    auto timed = [&](auto &&fn) {
        fn();  // configure and warm
        check_cuda(cudaEventRecord(e0, p->stream), "cudaEventRecord");
        for (int r = 0; r < nrep; r++) fn();
        check_cuda(cudaEventRecord(e1, p->stream), "cudaEventRecord");
        check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        return ms;
    };
    try {
        for (int q = 0; q < kTunedPasses; q++) {
            const int axis = kTunedAxis[q], mode = kTunedMode[q];
            p->tile_threads[axis][mode] = 0;
            if (!p->ax[axis].reg) continue;  // the shared-memory engine has one tile shape
            float best = 0.f;
            int best_th = 0, best_s = p->radix[axis][mode];
            for (int s = 0; s < 2; s++) {
                if (!radix && s != p->radix[axis][mode]) continue;
                const int T = s == 0 ? p->ax[axis].reg_threads : p->ax[axis].reg_threads1;
                for (int th : {128, 256, 512}) {
                    if (th % T != 0) continue;
                    p->radix[axis][mode] = s;
                    p->tile_threads[axis][mode] = th;
                    const float ms = timed([&] { run(q); });
                    if (best_th == 0 || ms < best) {
                        best = ms;
                        best_th = th;
                        best_s = s;
                    }
                }
            }
            p->radix[axis][mode] = best_s;
            p->tile_threads[axis][mode] = best_th;
        }
        if (radix && p->ax[0].reg) {
            // the stage boundary's schedule, timed on the work field alone (every operand of the
            // RK stage epilogue points at it; each element is read and written by one thread)
            EpiParams<Real> P{};
            P.nsites = p->nsites;
            P.mode = EPI_RK3;
            P.psi = w;
            P.psi_out = w;
            P.kprev = w;
            P.kout = w;
            P.kacc = w;
            P.ds = p->ds;
            P.sp = p->sp_lap;
            P.fkind = FK_LHY;
            P.nx = p->shape[0];
            P.ny = p->shape[1];
            P.nz = p->shape[2];
            P.slot = 1;
            P.cfac = 0.5;
            P.cnfac = 1.0;
            P.turn = 1;
            P.stream_aux = p->stream_aux ? 1 : 0;
            OpStageOut<Real, false, true> op{w, P};
            // schedules 0 / 1 with register loads, then on the bulk-copy ring where it serves
            float best = 0.f;
            int best_b = 0;
            for (int b = 0; b < 4; b++) {
                if ((b & 2) && !ring_serves<Real>(p, b & 1)) continue;
                p->radix_boundary = b;
                const float ms = timed([&] { launch_axis<Real, true, MODE_INV_TURN_FWD>(p, 0, op); });
                if (b == 0 || ms < best) {
                    best = ms;
                    best_b = b;
                }
            }
            p->radix_boundary = best_b;
            check_cuda(cudaMemsetAsync(w, 0, p->field_bytes * p->nsolve, p->stream), "memset work");
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

template <typename Real> void Launch<Real>::laplacian(gp5cu_plan *p, const void *src, void *dst) {
    using V = cpx<Real>;
    kinetic_passes<Real>(p, src, p->work, p->sp_lap, p->ds);
    OpCopy<Real> last{(const V *)p->work, (V *)dst, nullptr};
    launch_axis<Real, true, MODE_INV>(p, 0, last);
}

template <typename Real> static EpiParams<Real> base_epi(gp5cu_functional *f) {
    const gp5cu_plan *p = f->plan;
    const gp5cu_functional_desc &d = f->desc;
    EpiParams<Real> P{};
    P.nsites = p->nsites;
    P.fkind = d.kind;
    P.has_g = d.has_couplings;
    P.pot = d.potential;
    P.nx = p->shape[0];
    P.ny = p->shape[1];
    P.nz = p->shape[2];
    P.varr = (const Real *)d.dpotential;
    P.sp = f->sp;
    return P;
}

template <typename Real>
static void epilogue(gp5cu_plan *p, const EpiParams<Real> &P, bool red) {
    using V = cpx<Real>;
    if (p->ncomp == 1) {
        if (red) {
            OpStageOut<Real, true> op{(const V *)p->work, P};
            launch_axis<Real, true, MODE_INV>(p, 0, op);
        } else {
            OpStageOut<Real, false> op{(const V *)p->work, P};
            launch_axis<Real, true, MODE_INV>(p, 0, op);
        }
    } else {
        OpCopy<Real> cp{(const V *)p->work, (V *)p->work, P.sp};
        launch_axis<Real, true, MODE_INV>(p, 0, cp);
        EpiParams<Real> Q = P;
        Q.tsrc = (const V *)p->work;
        if (red) launch_pointwise(p, OpSiteEpilogue<Real, 2, true>{Q, p->solve_stride});
        else launch_pointwise(p, OpSiteEpilogue<Real, 2, false>{Q, p->solve_stride});
    }
}

template <typename Real>
void Launch<Real>::apply_h(gp5cu_functional *f, const void *src, void *dst, bool obs) {
    using V = cpx<Real>;
    gp5cu_plan *p = f->plan;
    kinetic_passes<Real>(p, src, p->work, f->sp, p->ds);
    EpiParams<Real> P = base_epi<Real>(f);
    P.mode = obs ? EPI_OBS : EPI_H;
    P.psi = (const V *)src;
    P.kout = (V *)dst;
    P.ds = p->ds;
    epilogue<Real>(p, P, obs);
}

// One preconditioned gradient iteration of every live solve of the plan (single component;
// OpPrecondIn / OpPrecond / OpPrecondOut): H psi into hbuf with mu per solve, the residual's
// transform with the shifted inverse kinetic operator in k-space, the update of psi with its
// norm, then the normalisation.  sp_norm: parameters holding the target N and dV per solve.
template <typename Real>
void Launch<Real>::precond_iter(gp5cu_functional *f, const SolveParams *sp_norm, void *psi, void *hbuf,
                                double theta) {
    using V = cpx<Real>;
    gp5cu_plan *p = f->plan;
    apply_h(f, psi, hbuf, true);
    OpPrecondIn<Real> in{(const V *)hbuf, (const V *)psi, (V *)p->work, p->ds, f->sp};
    launch_axis<Real, true, MODE_FWD>(p, 0, in);
    OpCopy<Real> cp{(const V *)p->work, (V *)p->work, p->nsolve > 1 ? f->sp : nullptr};
    launch_axis<Real, false, MODE_FWD>(p, 1, cp);
    OpPrecond<Real> pc{(const V *)p->work, (V *)p->work, f->sp, p->ds, p->shape[0], p->shape[1], p->shape[2],
                       (double)p->nsites};
    launch_axis<Real, false, MODE_FWD_MID_INV>(p, 2, pc);
    launch_axis<Real, false, MODE_INV>(p, 1, cp);
    OpPrecondOut<Real> out{(const V *)p->work, (V *)psi, p->ds, sp_norm, theta};
    launch_axis<Real, true, MODE_INV>(p, 0, out);
    scale(p, psi, 0, p->ds, false);
}

template <typename Real>
void Launch<Real>::residual(gp5cu_plan *p, const void *psi, const void *hpsi, DevScalars *ds, const SolveParams *sp) {
    using V = cpx<Real>;
    OpResidual<Real> op{(const V *)psi, (const V *)hpsi, p->nsites, p->solve_stride, p->ncomp, ds, sp};
    launch_pointwise(p, op);
}

template <typename Real>
void Launch<Real>::norm(gp5cu_plan *p, const void *field, int comp, double Ntarget, DevScalars *ds) {
    using V = cpx<Real>;
    OpNorm<Real> op{(const V *)field, p->nsites, p->solve_stride, comp, p->ncomp, ds, Ntarget, p->dV};
    launch_pointwise(p, op);
}

template <typename Real>
void Launch<Real>::scale(gp5cu_plan *p, void *field, int comp, DevScalars *ds, bool from_sigma) {
    using V = cpx<Real>;
    OpScale<Real> op{(V *)field, p->nsites, p->solve_stride, comp, p->ncomp, ds, from_sigma ? 1 : 0};
    launch_pointwise(p, op);
}

template <typename Real> void Launch<Real>::max_density(gp5cu_plan *p, const void *field) {
    check_cuda(cudaMemsetAsync(p->dmax, 0, sizeof(unsigned long long), p->stream), "memset");
    k_max_density<Real><<<p->pw_blocks, kThreads, 0, p->stream>>>((const cpx<Real> *)field,
                                                                    p->nsites * p->nsolve, p->ncomp, p->dmax);
    check_cuda(cudaGetLastError(), "k_max_density launch");
}

template <typename Real>
void Launch<Real>::convert(gp5cu_plan *p, const double *in128, void *out, const void *in, double *out128,
                           long long n) {
    OpConvert<Real> op{(const double2 *)in128, (cpx<Real> *)out, (const cpx<Real> *)in, (double2 *)out128};
    k_pointwise<OpConvert<Real>><<<p->pw_blocks, kThreads, 0, p->stream>>>(n, p->pw_blocks, op, red_slot(p));
    check_cuda(cudaGetLastError(), "convert launch");
}

template <typename Real> void Launch<Real>::init_gaussian(gp5cu_plan *p, void *field, int comp, const double sigma[3]) {
    double a[3], d[3];
    for (int q = 0; q < 3; q++) {
        a[q] = 1.0 / (2 * sigma[q] * sigma[q]);
        d[q] = (p->right[q] - p->left[q]) / p->shape[q];
    }
    cpx<Real> *f = (cpx<Real> *)field + (long long)comp * p->nsites;
    k_init_gaussian<Real><<<p->pw_blocks, kThreads, 0, p->stream>>>(f, p->shape[0], p->shape[1], p->nsites,
                                                                     p->left[0], p->left[1], p->left[2], d[0],
                                                                     d[1], d[2], a[0], a[1], a[2]);
    check_cuda(cudaGetLastError(), "init_gaussian launch");
}

template <typename Real> void Launch<Real>::phase_exp(gp5cu_plan *p, const void *phase, void *out) {
    k_phase_exp<Real><<<p->pw_blocks, kThreads, 0, p->stream>>>((const Real *)phase, (cpx<Real> *)out,
                                                                 p->nsites * p->ncomp * p->nsolve);
    check_cuda(cudaGetLastError(), "phase_exp launch");
}

// ---- one stepper step ----------------------------------------------------------------------
// Five-pass form (RK4, stepper.cpp:46-71): four stages of
//   x fwd [u~ = sigma psi0 - c k_{s-1}, |u~|^2]  y fwd  z fwd*K^2/(2mN^3)*z inv  y inv
//   x inv [k_s = H(alpha u~); RK bookkeeping; psi1 on the last stage]
// Buffers: psi (in/out, in place), work (transform), Ka (k1, then the running sum
// k1 + 2k2 + 2k3), Kb (k2, then k3).  Used when the stage boundary cannot be merged.
template <typename Real> int Launch<Real>::step(gp5cu_stepper *st, void *field) {
    using V = cpx<Real>;
    gp5cu_functional *f = st->func;
    gp5cu_plan *p = f->plan;
    V *psi = (V *)field;
    V *W = (V *)p->work;
    V *Ka = (V *)st->Ka;
    V *Kb = (V *)st->Kb;
    const bool rk4 = st->kind == GP5_STEP_RK4;
    const int nst = rk4 ? 4 : 1;
    int launches = 0;
    for (int s = 1; s <= nst; s++) {
        double cfac = 0;
        const V *kprev = nullptr;
        if (rk4 && s > 1) {
            cfac = (s == 4) ? 1.0 : 0.5;
            kprev = (s == 2) ? Ka : Kb;
        }
        const bool red_in = st->renorm && rk4 && s > 1;
        if (red_in) {
            OpStageIn<Real, true> in{psi, kprev, W, st->ds, st->sp, 1, cfac, s & 1};
            launch_axis<Real, true, MODE_FWD>(p, 0, in);
        } else {
            OpStageIn<Real, false> in{psi, kprev, W, st->ds, st->sp, st->renorm ? 1 : 0, cfac, s & 1};
            launch_axis<Real, true, MODE_FWD>(p, 0, in);
        }
        OpCopy<Real> cp{W, W, p->nsolve > 1 ? st->sp : nullptr};  // only a batch needs the active flags
        launch_axis<Real, false, MODE_FWD>(p, 1, cp);
        OpKinetic<Real> kin{W, W, st->sp, p->shape[0], p->shape[1], p->shape[2]};
        launch_axis<Real, false, MODE_FWD_MID_INV>(p, 2, kin);
        launch_axis<Real, false, MODE_INV>(p, 1, cp);
        launches += 4;

        EpiParams<Real> P = base_epi<Real>(f);
        P.sp = st->sp;
        P.ds = st->ds;
        P.psi = psi;
        P.psi_out = psi;
        P.kprev = kprev;
        P.kacc = Ka;
        P.use_sigma = st->renorm ? 1 : 0;
        P.use_alpha = red_in ? 1 : 0;
        P.slot = s & 1;
        P.cfac = cfac;
        P.phase_exp = nullptr;
        if (!rk4) {
            P.mode = EPI_EULER;
            P.dfac = 1.0;
        } else {
            P.mode = EPI_RK1 + (s - 1);
            P.kout = (s == 1) ? Ka : Kb;
            P.dfac = 1. / 6;
        }
        const bool last = (s == nst);
        if (last) {
            P.phase_exp = (const V *)st->phase_exp;
            P.renorm_out = st->renorm ? 1 : 0;
            if (compensation_active(st)) P.comp = (__nv_bfloat162 *)st->comp;
            P.sround = st->sround ? 1 : 0;
        }
        epilogue<Real>(p, P, last && st->renorm);
        launches += (p->ncomp == 1) ? 1 : 2;
    }
    return launches;
}

template <typename Real> void Launch<Real>::prologue(gp5cu_stepper *st, void *field) {
    using V = cpx<Real>;
    gp5cu_plan *p = st->func->plan;
    if (p->kin_scheme == 1) return;  // the per-axis scheme's first stage reads the state itself
    OpStageIn<Real, false> in{(const V *)field, nullptr, (V *)p->work, st->ds, st->sp, 0, 0.0, 1};
    launch_axis<Real, true, MODE_FWD>(p, 0, in);
}

// RK4 / Euler with the stage boundaries merged: after the prologue transform of psi (once
// per advance call), every stage is y fwd, z fwd*K^2/(2mN^3)*z inv, y inv, then one x kernel
// that inverts x, finishes stage s (k_s, RK bookkeeping, psi1 after the last stage), forms the
// input of the next stage (u~_{s+1} = sigma psi0 - c_{s+1} k_s, or psi1) and transforms it
// forward in x.  Field transfers per RK4 step: 47 instead of 54; 16 launches instead of 20.
template <typename Real> int Launch<Real>::step_merged(gp5cu_stepper *st, void *field, bool prologue) {
    using V = cpx<Real>;
    gp5cu_functional *f = st->func;
    gp5cu_plan *p = f->plan;
    if (p->kin_scheme == 1) return step_axes(st, field);
    V *psi = (V *)field;
    V *W = (V *)p->work;
    V *Ka = (V *)st->Ka;
    V *Kb = (V *)st->Kb;
    const bool rk4 = st->kind == GP5_STEP_RK4;
    const int nst = rk4 ? 4 : 1;
    int launches = 0;
    if (prologue) {
        Launch<Real>::prologue(st, field);
        launches++;
    }
    // The y forward, z (forward * K^2 * inverse) and y inverse passes run on slabs of
    // consecutive x values, one slab after the other (p->yz_slabs of them): a slab's field
    // stays in L2 from its y forward pass to its y inverse pass, so only the first reads and
    // the last writes it in HBM.
    const int slabs = std::max(1, p->yz_slabs);
    const int sw = p->shape[0] / slabs;
    for (int s = 1; s <= nst; s++) {
        OpCopy<Real> cp{W, W, p->nsolve > 1 ? st->sp : nullptr};  // only a batch needs the active flags
        OpKinetic<Real> kin{W, W, st->sp, p->shape[0], p->shape[1], p->shape[2]};
        for (int b = 0; b < slabs; b++) {
            if (slabs > 1) {
                p->xr0 = b * sw;
                p->xr_n = sw;
            }
            launch_axis<Real, false, MODE_FWD>(p, 1, cp);
            launch_axis<Real, false, MODE_FWD_MID_INV>(p, 2, kin);
            launch_axis<Real, false, MODE_INV>(p, 1, cp);
        }
        p->xr0 = p->xr_n = 0;
        EpiParams<Real> P = base_epi<Real>(f);
        P.sp = st->sp;
        P.ds = st->ds;
        P.psi = psi;
        P.psi_out = psi;
        P.kacc = Ka;
        P.use_sigma = st->renorm ? 1 : 0;
        P.use_alpha = st->renorm ? 1 : 0;
        P.slot = s & 1;
        P.u1_raw = (s == 1) ? 1 : 0;
        P.turn = 1;
        P.stream_aux = p->stream_aux ? 1 : 0;
        P.renorm_out = st->renorm ? 1 : 0;
        P.phase_exp = nullptr;
        P.comp = nullptr;
        if (s == nst && compensation_active(st)) P.comp = (__nv_bfloat162 *)st->comp;
        P.sround = st->sround ? 1 : 0;
        if (!rk4) {
            P.mode = EPI_EULER;
            P.kprev = nullptr;
            P.dfac = 1.0;
            P.phase_exp = (const V *)st->phase_exp;
        } else {
            P.mode = EPI_RK1 + (s - 1);
            P.kprev = (s == 1) ? nullptr : ((s == 2) ? Ka : Kb);
            P.kout = (s == 1) ? Ka : Kb;
            P.dfac = 1. / 6;
            P.cfac = (s == 1) ? 0.0 : ((s == 4) ? 1.0 : 0.5);      // u~_s = sigma psi0 - tau cfac k_{s-1}
            P.cnfac = (s < 4) ? ((s + 1 == 4) ? 1.0 : 0.5) : 0.0;  // u~_{s+1}
            if (s == 4) P.phase_exp = (const V *)st->phase_exp;
        }
        if (st->renorm) {
            OpStageOut<Real, true, true> op{W, P};
            launch_axis<Real, true, MODE_INV_TURN_FWD>(p, 0, op);
        } else {
            OpStageOut<Real, false, true> op{W, P};
            launch_axis<Real, true, MODE_INV_TURN_FWD>(p, 0, op);
        }
        launches += 1 + 3 * slabs;
    }
    return launches;
}

// RK4 / Euler with the kinetic term as per-axis spectral second derivatives (plan kin_scheme 1).
// Per stage s, u~_s the stage input (the state itself in the first stage, else what the
// previous boundary wrote to the work field U, in real space):
//   y pass    T  = IFFT_y(ky^2/(2 m Ny) FFT_y u~_s)            reads u~_s, writes T
//   z pass    T += IFFT_z(kz^2/(2 m Nz) FFT_z u~_s)            reads u~_s and T, writes T
//   boundary  u~_s again from psi and k_{s-1}; t = IFFT_x(kx^2/(2 m Nx) FFT_x u~_s) + T; the
//             stage epilogue of step_merged; u~_{s+1} to U (psi1 after the last stage)
// The three axis terms sum to the 3D operator because K^2 is separable and the axis transforms
// commute.  Field transfers per RK4 step: 5 per stage in the y/z passes and 4 + 6 + 7 + 5 in
// the boundaries, 42 instead of 47; 12 launches and no prologue.
template <typename Real> int Launch<Real>::step_axes(gp5cu_stepper *st, void *field) {
    using V = cpx<Real>;
    gp5cu_functional *f = st->func;
    gp5cu_plan *p = f->plan;
    V *psi = (V *)field;
    V *U = (V *)p->work;
    V *Ka = (V *)st->Ka;
    V *Kb = (V *)st->Kb;
    // allocated in the dry pass that precedes a graph capture, or by an eager step
    if (!st->T) check_cuda(cudaMalloc(&st->T, p->field_bytes * p->nsolve), "cudaMalloc kinetic terms");
    V *T = (V *)st->T;
    const bool rk4 = st->kind == GP5_STEP_RK4;
    const int nst = rk4 ? 4 : 1;
    const int slabs = std::max(1, p->yz_slabs);
    const int sw = p->shape[0] / slabs;
    int launches = 0;
    for (int s = 1; s <= nst; s++) {
        const V *u = s == 1 ? psi : U;
        OpDeriv<Real, 1, false> dy{u, T, st->sp, p->shape[0], p->shape[1], p->shape[2]};
        OpDeriv<Real, 2, true> dz{u, T, st->sp, p->shape[0], p->shape[1], p->shape[2]};
        for (int b = 0; b < slabs; b++) {
            if (slabs > 1) {
                p->xr0 = b * sw;
                p->xr_n = sw;
            }
            launch_axis<Real, false, MODE_FWD_MID_INV>(p, 1, dy);
            launch_axis<Real, false, MODE_FWD_MID_INV>(p, 2, dz);
        }
        p->xr0 = p->xr_n = 0;
        EpiParams<Real> P = base_epi<Real>(f);
        P.sp = st->sp;
        P.ds = st->ds;
        P.psi = psi;
        P.psi_out = psi;
        P.kacc = Ka;
        P.use_sigma = st->renorm ? 1 : 0;
        P.use_alpha = st->renorm ? 1 : 0;
        P.slot = s & 1;
        P.u1_raw = (s == 1) ? 1 : 0;
        P.turn = 1;
        P.stream_aux = p->stream_aux ? 1 : 0;
        P.renorm_out = st->renorm ? 1 : 0;
        P.phase_exp = nullptr;
        P.comp = nullptr;
        if (s == nst && compensation_active(st)) P.comp = (__nv_bfloat162 *)st->comp;
        P.sround = st->sround ? 1 : 0;
        if (!rk4) {
            P.mode = EPI_EULER;
            P.kprev = nullptr;
            P.dfac = 1.0;
            P.phase_exp = (const V *)st->phase_exp;
        } else {
            P.mode = EPI_RK1 + (s - 1);
            P.kprev = (s == 1) ? nullptr : ((s == 2) ? Ka : Kb);
            P.kout = (s == 1) ? Ka : Kb;
            P.dfac = 1. / 6;
            P.cfac = (s == 1) ? 0.0 : ((s == 4) ? 1.0 : 0.5);
            P.cnfac = (s < 4) ? ((s + 1 == 4) ? 1.0 : 0.5) : 0.0;
            if (s == 4) P.phase_exp = (const V *)st->phase_exp;
        }
        V *unext = s < nst ? U : nullptr;
        if (st->renorm) {
            OpStageAxes<Real, true> op{P, T, unext, p->shape[0], p->shape[1], p->shape[2]};
            launch_axis<Real, true, MODE_FWD_MID_INV>(p, 0, op);
        } else {
            OpStageAxes<Real, false> op{P, T, unext, p->shape[0], p->shape[1], p->shape[2]};
            launch_axis<Real, true, MODE_FWD_MID_INV>(p, 0, op);
        }
        launches += 1 + 2 * slabs;
    }
    return launches;
}

}  // namespace gp5

// passes.cuh - axis-pass kernels: one kernel = a batch of line FFTs along one axis, with
// the point-wise work of the stepper fused into its loads (prologue), into the middle of a
// forward+inverse pair (kinetic multiply), and into its stores (epilogue).
//
// Field layout: element (i, j, k, c) at i + nx*(j + ny*(k + nz*c)) (ColMajor, x fastest).
//   x axis: a line is contiguous; a tile is LINES consecutive lines.
//   y/z axes: a line has stride nx (y) or nx*ny (z); a tile is bx consecutive x values by bo
//     other lines, so that a warp's loads cover bx*16 contiguous bytes per position.
//
// Reductions: every op may accumulate up to 8 FP64 sums per thread.  A block folds them
// with a fixed-order shuffle tree, writes one partial per block, and the last block to
// finish (atomic ticket, no waiting) adds the partials in index order with Neumaier
// compensation and calls op.finalize.  The result is independent of block scheduling, so
// repeated runs are bitwise identical.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "fft_line.cuh"

namespace gp5 {

// MODE_INV_TURN_FWD: inverse transform, op.turn() per element (epilogue of one stage and
// prologue of the next), forward transform, op.post() stores.
enum PassMode : int { MODE_FWD = 0, MODE_INV = 1, MODE_FWD_MID_INV = 2, MODE_INV_TURN_FWD = 3 };

struct TileGeom {
    int nx, ny, nz, nc;
    int axis;           // 0 = x, 1 = y, 2 = z
    int n;              // line length
    long long estride;  // element stride along the line
    int lines;          // lines per tile
    int bx, bo;         // strided tiles: consecutive x lines, other lines
    int tiles_x;        // strided tiles: ceil(nx / bx)
    long long n_other;  // strided: number of (other) line groups; x axis: total lines
    long long ntiles;   // tiles of the launch: nsolve * tiles_per_solve
    int nsolve;                 // independent solves of this grid in the launch
    long long tiles_per_solve;  // tiles of one solve (consecutive tile indices)
    long long solve_stride;     // elements between the fields of consecutive solves
    int reverse;                // CTAs take the tiles from the last one down (L2 reuse order)
    int x0, xend;               // strided passes: the x range [x0, xend) the tiles cover
};

struct RedSlot {
    double *partials;   // [nsolve][tiles_per_solve][8]
    unsigned *counter;  // [nsolve], zero between launches
};

// Coordinates of one line: base offset (including the solve's offset) and fixed coordinates.
struct LineRef {
    long long base;
    int i, j, k, c;
    int solve;
    bool valid;
};

__device__ __forceinline__ LineRef line_ref(const TileGeom &g, long long tile_all, int line) {
    LineRef r;
    r.i = r.j = r.k = r.c = 0;
    r.solve = (int)(tile_all / g.tiles_per_solve);
    const long long tile = tile_all - (long long)r.solve * g.tiles_per_solve;
    if (g.axis == 0) {
        long long L = tile * g.lines + line;
        r.valid = L < g.n_other;
        if (!r.valid) L = 0;
        r.base = L * g.nx;
        r.j = (int)(L % g.ny);
        long long t = L / g.ny;
        r.k = (int)(t % g.nz);
        r.c = (int)(t / g.nz);
    } else {
        const long long tx = tile % g.tiles_x, to = tile / g.tiles_x;
        const int xo = line % g.bx, oo = line / g.bx;
        int i = g.x0 + (int)(tx * g.bx) + xo;
        long long o = to * g.bo + oo;
        r.valid = (i < g.xend) && (o < g.n_other);
        if (!r.valid) { i = 0; o = 0; }
        r.i = i;
        if (g.axis == 1) {  // o = k + nz*c
            r.k = (int)(o % g.nz);
            r.c = (int)(o / g.nz);
            r.base = i + (long long)g.nx * g.ny * o;
        } else {            // o = j + ny*c
            r.j = (int)(o % g.ny);
            r.c = (int)(o / g.ny);
            r.base = i + (long long)g.nx * r.j + (long long)g.nx * g.ny * g.nz * r.c;
        }
    }
    r.base += (long long)r.solve * g.solve_stride;
    return r;
}

__device__ __forceinline__ void set_pos(const TileGeom &g, LineRef &r, int pos) {
    if (g.axis == 0) r.i = pos;
    else if (g.axis == 1) r.j = pos;
    else r.k = pos;
}

// ---- reductions -------------------------------------------------------------------------
template <int K> __device__ __forceinline__ void warp_sum(double (&a)[K]) {
#pragma unroll
    for (int r = 0; r < K; r++) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a[r] += __shfl_down_sync(0xffffffffu, a[r], off);
    }
}

// Block sum in fixed order; result valid in thread 0.
template <int K> __device__ void block_sum(double (&a)[K]) {
    __shared__ double red[32 * (K > 0 ? K : 1)];
    warp_sum<K>(a);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < K; r++) red[w * K + r] = a[r];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int r = 0; r < K; r++) a[r] = lane < nw ? red[lane * K + r] : 0.0;
        warp_sum<K>(a);
    }
    __syncthreads();
}

__device__ __forceinline__ void neumaier(double &s, double &comp, double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) comp += (s - t) + x;
    else comp += (x - t) + s;
    s = t;
}

// Per-block partials, then the last block of the solve folds that solve's partials and calls
// op.finalize(sums, solve).  lb = block index within the solve, nb = blocks of the solve.
template <int K, class Op>
__device__ void reduce_and_finalize(const double *acc_in, const RedSlot &rs, const Op &op, int solve,
                                    long long lb, long long nb) {
    if constexpr (K > 0) {
        double acc[K];
#pragma unroll
        for (int r = 0; r < K; r++) acc[r] = acc_in[r];
        block_sum<K>(acc);
        double *part = rs.partials + (long long)solve * nb * K;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int r = 0; r < K; r++) part[lb * K + r] = acc[r];
        }
        __threadfence();
        __shared__ bool s_last;
        __syncthreads();
        if (threadIdx.x == 0) s_last = (atomicAdd(rs.counter + solve, 1u) == (unsigned)(nb - 1));
        __syncthreads();
        if (s_last) {
            __threadfence();
            double s[K], cp[K];
#pragma unroll
            for (int r = 0; r < K; r++) { s[r] = 0.0; cp[r] = 0.0; }
            for (long long b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
                for (int r = 0; r < K; r++) neumaier(s[r], cp[r], __ldcg(part + b * K + r));
            }
            block_sum<K>(s);
            block_sum<K>(cp);
            if (threadIdx.x == 0) {
                double tot[K];
#pragma unroll
                for (int r = 0; r < K; r++) tot[r] = s[r] + cp[r];
                op.finalize(tot, solve);
                rs.counter[solve] = 0u;
            }
        }
    }
}

// ---- L2 prefetch of a tile's input streams -------------------------------------------------
// cp.async.bulk.prefetch.L2 brings a contiguous range into L2 without registers or shared
// memory; a persistent CTA issues it for the tile it will process next, so that the DRAM
// reads of that tile overlap the transform of the current one.  Ranges that are not 16-byte
// aligned and sized are skipped (the prefetch is only a hint).
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes) {
    if ((((uintptr_t)p) & 15u) == 0 && (bytes & 15u) == 0 && bytes > 0)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L2 prefetch of every stream of a contiguous x tile that reads more than one array: one
// instruction per stream, issued by thread 0 at kernel start, so that all DRAM reads of the
// tile are in flight at once and the later register loads hit L2.  GP5_PREFETCH_AUX: 2 all
// streams, 1 the epilogue's streams only (not the transform input), 0 none (default: with the
// reversed boundary tile order the prefetch measured 1-2% slower at 256^3 in both precisions,
// and its lines were partly evicted before use: 8-18% extra DRAM reads in stages 2-4).
#ifndef GP5_PREFETCH_AUX
#define GP5_PREFETCH_AUX 0
#endif
template <typename V, class Op>
__device__ __forceinline__ void prefetch_aux(const TileGeom &g, long long tile, const Op &op) {
    if constexpr (GP5_PREFETCH_AUX == 0) return;
    const void *st[4];
    const int ns = op.streams(st);
    if (ns < 2 || threadIdx.x != 0 || g.axis != 0) return;
    const long long solve = tile / g.tiles_per_solve, lt = tile - solve * g.tiles_per_solve;
    const long long L0 = lt * g.lines;
    long long L1 = L0 + g.lines;
    if (L1 > g.n_other) L1 = g.n_other;
    const long long e0 = solve * g.solve_stride + L0 * g.nx, cnt = (L1 - L0) * g.nx;
    for (int q = GP5_PREFETCH_AUX == 1 ? 1 : 0; q < ns; q++)
        prefetch_l2(reinterpret_cast<const V *>(st[q]) + e0, (unsigned)(cnt * sizeof(V)));
}

// ops that provide the hoisted z-line k-space multiply (mid_line / mid_z)
// ops whose epilogue is long enough to run as a rolled loop (HEAVY_EPILOGUE)
template <class Op, class = void> struct heavy_epilogue : std::false_type {};
template <class Op> struct heavy_epilogue<Op, std::void_t<decltype(Op::HEAVY_EPILOGUE)>> : std::true_type {};

template <class Op, class = void> struct has_mid_z : std::false_type {};
template <class Op> struct has_mid_z<Op, std::void_t<decltype(Op::MID_Z)>> : std::true_type {};

// ---- register-engine kernel ----------------------------------------------------------------
// Threads: LINES lines x T threads per line (RegTile below); one tile per
// CTA.
// Tile shape: the passes with two transforms (forward*K^2*inverse, and the stage boundary)
// have the longest compute phase; they use 128-thread tiles so that several small CTAs share
// an SM and their load / transform / store phases interleave.  Copy passes use 256 threads.
#ifndef GP5_HEAVY_THREADS
#define GP5_HEAVY_THREADS 128
#endif
// TH > 0 overrides the rule (the autotuner's tile shapes for the strided y/z passes); S is the
// radix schedule (RegCfg).
template <typename Real, int N, bool CONTIG, int MODE, int TH = 0, int S = 0> struct RegTile {
    static constexpr int T = RegCfgAll<N, S>::T;
    static constexpr int THREADS =
        TH > 0 ? TH
               : ((MODE == MODE_FWD_MID_INV || MODE == MODE_INV_TURN_FWD) && GP5_HEAVY_THREADS / T >= 2 ? GP5_HEAVY_THREADS
                                                                                                      : 256);
    static_assert(THREADS % T == 0 && THREADS <= 1024, "a tile is a whole number of lines");
    static constexpr int LINES = THREADS / T;
    // register cap per thread: 128 for complex128.  complex64: the strided single-transform
    // passes and the stage boundary are bound by memory latency and trade registers for
    // resident CTAs (64: 8 CTAs of 128 threads, at most 8 bytes of spill); the other passes
    // keep 80.  (A cap of 96 for the complex128 strided copies measured slower: it spills.)
    static constexpr bool STRIDED_COPY = (MODE == MODE_FWD || MODE == MODE_INV) && !CONTIG;
#ifndef GP5_C64_CAP_COPY
#define GP5_C64_CAP_COPY 64
#endif
#ifndef GP5_C64_CAP_BOUNDARY
#define GP5_C64_CAP_BOUNDARY 64
#endif
#ifndef GP5_C64_CAP_OTHER
#define GP5_C64_CAP_OTHER 80
#endif
#ifndef GP5_C128_CAP
#define GP5_C128_CAP 128
#endif
#ifndef GP5_C128_CAP_LIGHT
#define GP5_C128_CAP_LIGHT 96
#endif
#ifndef GP5_C64_CAP_LIGHT
#define GP5_C64_CAP_LIGHT 64
#endif
    // a schedule with fewer elements per thread than S = 0 needs fewer registers: it is capped
    // lower so that more CTAs share an SM
    static constexpr bool LIGHT = RegCfg<N, S>::E < RegCfg<N, 0>::E;
    static constexpr int REGCAP = LIGHT ? (sizeof(Real) == 8 ? GP5_C128_CAP_LIGHT : GP5_C64_CAP_LIGHT)
                                        : (sizeof(Real) == 8 ? GP5_C128_CAP
                                                             : (STRIDED_COPY ? GP5_C64_CAP_COPY
                                                                             : (MODE == MODE_INV_TURN_FWD
                                                                                    ? GP5_C64_CAP_BOUNDARY
                                                                                    : GP5_C64_CAP_OTHER)));
    static constexpr int MINB_RAW = (65536 / REGCAP) / THREADS;
    static constexpr int MINB = MINB_RAW > 0 ? MINB_RAW : 1;
};

template <typename Real, int N, bool CONTIG, int MODE, class Op, int TH = 0, int S = 0>
__global__ void __launch_bounds__(RegTile<Real, N, CONTIG, MODE, TH, S>::THREADS,
                                  RegTile<Real, N, CONTIG, MODE, TH, S>::MINB)
k_axis_reg(const TileGeom g, Op op, const cpx<Real> *__restrict__ tw, const RedSlot rs) {
    using V = cpx<Real>;
    constexpr int E = RegCfg<N, S>::E, T = RegCfgAll<N, S>::T, LINES = RegTile<Real, N, CONTIG, MODE, TH, S>::LINES;
    constexpr int NB = Op::BATCH;
    static_assert(E % NB == 0, "batch must divide the elements per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *sm = reinterpret_cast<V *>(smem_raw);

    pdl_enter();
    // x lines are contiguous: a compile-time unit stride spares the 64-bit multiplies
    const long long es = CONTIG ? 1LL : g.estride;
    int tid, line;
    if (CONTIG) { tid = threadIdx.x % T; line = threadIdx.x / T; }
    else { line = threadIdx.x % LINES; tid = threadIdx.x / LINES; }

    double acc[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int r = 0; r < (Op::NRED > 0 ? Op::NRED : 1); r++) acc[r] = 0.0;

    const long long tile = g.reverse ? (long long)gridDim.x - 1 - blockIdx.x : (long long)blockIdx.x;
    const int solve = (int)(tile / g.tiles_per_solve);
    __shared__ typename Op::Ctx X;
    const void *streams[4];
    op.streams(streams);
    const V *__restrict__ src0 = reinterpret_cast<const V *>(streams[0]);
    if (CONTIG) prefetch_aux<V>(g, tile, op);
    {
        LineRef lr = line_ref(g, tile, line);
        // the solve's context and the tile's first stream are fetched together
        const unsigned long long cw = ctx_fetch(op.params(), op.scalars(), solve);
        V v[E];
#pragma unroll
        for (int m = 0; m < E; m++)
            v[m] = lr.valid ? src0[lr.base + (tid + T * m) * es] : mk<Real>(0, 0);
        if (op.params() || op.scalars()) {  // uniform: ops without per-solve data skip the barrier
            ctx_store(X, op.params(), op.scalars(), cw);
            __syncthreads();
            if (op.params() && !X.S.active) return;  // a finished solve's tiles return at once
        }
        if (lr.valid) {
#pragma unroll
            for (int m = 0; m < E; m++) {
                const int pos = tid + T * m;
                LineRef e = lr;
                set_pos(g, e, pos);
                const long long ge = lr.base + pos * es;
                v[m] = op.load(v[m], ge, e, acc, X);
            }
        }
        if constexpr (MODE == MODE_INV_TURN_FWD) {
            static_assert(CONTIG, "the stage boundary runs on x lines");
            LayContig<N, S> lay;
            reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            // The epilogue/prologue runs as a rolled loop over the thread's own elements staged
            // in shared memory: one copy of its code (the unrolled form overflowed the
            // instruction cache) and the transform registers are free meanwhile.  Each thread
            // reads back only what it wrote, so no barrier is needed around the loop.
#pragma unroll
            for (int m = 0; m < E; m++) sm[lay(line, tid + T * m)] = v[m];
            if (lr.valid) {
                const auto K = op.consts(X);  // once per tile, out of the element loop
#pragma unroll 1
                for (int m0 = 0; m0 < E; m0 += NB) {
                    typename Op::Pre pre[NB];
#pragma unroll
                    for (int j = 0; j < NB; j++) pre[j] = op.pre(lr.base + (tid + T * (m0 + j)) * es);
#pragma unroll
                    for (int j = 0; j < NB; j++) {
                        const int pos = tid + T * (m0 + j);
                        LineRef e = lr;
                        set_pos(g, e, pos);
                        const int si = lay(line, pos);
                        sm[si] = op.turn(lr.base + pos * es, e, sm[si], pre[j], acc, X, K);
                    }
                }
            }
#pragma unroll
            for (int m = 0; m < E; m++) v[m] = sm[lay(line, tid + T * m)];
            __syncthreads();
            reg_fft<N, S, -1>(v, tid, line, tw, sm, lay);
        } else if constexpr (CONTIG) {
            LayContig<N, S> lay;
            if (MODE == MODE_INV) reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            else reg_fft<N, S, -1>(v, tid, line, tw, sm, lay);
            if (MODE == MODE_FWD_MID_INV) {
#pragma unroll
                for (int m = 0; m < E; m++) {
                    LineRef e = lr;
                    set_pos(g, e, tid + T * m);
                    v[m] = op.mid(v[m], e, X);
                }
                __syncthreads();  // also a scheduling fence: keeps register pressure below 128
                reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            }
        } else {
            LayStrided lay{LINES};
            if (MODE == MODE_INV) reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            else reg_fft<N, S, -1>(v, tid, line, tw, sm, lay);
            if constexpr (MODE == MODE_FWD_MID_INV && has_mid_z<Op>::value) {
                if (g.axis == 2) {
                    // element m sits at tid + T*m < N/2 exactly when m < E/2, so the sign of
                    // its momentum index is known at compile time
                    const auto L = op.mid_line(lr, X);
#pragma unroll
                    for (int m = 0; m < E; m++) {
                        const int pos = tid + T * m;
                        v[m] = op.mid_z(v[m], m < E / 2 ? pos : pos - N, L);
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < E; m++) {
                        LineRef e = lr;
                        set_pos(g, e, tid + T * m);
                        v[m] = op.mid(v[m], e, X);
                    }
                }
                __syncthreads();  // also a scheduling fence: keeps register pressure below 128
                reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            } else if (MODE == MODE_FWD_MID_INV) {
#pragma unroll
                for (int m = 0; m < E; m++) {
                    LineRef e = lr;
                    set_pos(g, e, tid + T * m);
                    v[m] = op.mid(v[m], e, X);
                }
                __syncthreads();  // also a scheduling fence: keeps register pressure below 128
                reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
            }
        }
        if (lr.valid && MODE == MODE_INV_TURN_FWD) {
#pragma unroll
            for (int m = 0; m < E; m++) {
                const int pos = tid + T * m;
                LineRef e = lr;
                set_pos(g, e, pos);
                op.post(lr.base + pos * es, e, v[m], typename Op::Pre{}, acc, X);
            }
        } else if (CONTIG && heavy_epilogue<Op>::value) {
            // a long epilogue (the per-axis stage boundary) runs as a rolled loop over the
            // thread's own elements staged in shared memory, like the stage boundary's turn: one
            // copy of its code.  The transform's last exchange is behind a barrier, and each
            // thread reads back only what it wrote.
            LayContig<N, S> lay;
#pragma unroll
            for (int m = 0; m < E; m++) sm[lay(line, tid + T * m)] = v[m];
            if (lr.valid) {
#pragma unroll 1
                for (int m0 = 0; m0 < E; m0 += NB) {
                    typename Op::Pre pre[NB];
#pragma unroll
                    for (int j = 0; j < NB; j++) pre[j] = op.pre(lr.base + (tid + T * (m0 + j)) * es);
#pragma unroll
                    for (int j = 0; j < NB; j++) {
                        const int pos = tid + T * (m0 + j);
                        LineRef e = lr;
                        set_pos(g, e, pos);
                        op.post(lr.base + pos * es, e, sm[lay(line, pos)], pre[j], acc, X);
                    }
                }
            }
        } else if (lr.valid) {
            // epilogue in batches: the operand loads of NB elements are issued together
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += NB) {
                typename Op::Pre pre[NB];
#pragma unroll
                for (int j = 0; j < NB; j++) pre[j] = op.pre(lr.base + (tid + T * (m0 + j)) * es);
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const int pos = tid + T * (m0 + j);
                    LineRef e = lr;
                    set_pos(g, e, pos);
                    op.post(lr.base + pos * es, e, v[m0 + j], pre[j], acc, X);
                }
            }
        }
    }
    reduce_and_finalize<Op::NRED>(acc, rs, op, solve, tile - (long long)solve * g.tiles_per_solve,
                                  g.tiles_per_solve);
}

// ---- shared-memory-engine kernel (any length) ---------------------------------------------
struct LayContigRT {
    int ld;
    __device__ __forceinline__ int operator()(int line, int pos) const { return line * ld + pos; }
};

template <typename Real, bool CONTIG, int MODE, class Op>
__global__ void __launch_bounds__(256)
k_axis_smem(const TileGeom g, const LineSchedule ls, Op op, const cpx<Real> *__restrict__ tw,
            const RedSlot rs) {
    using V = cpx<Real>;
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = g.n, lines = g.lines;
    const int ld = CONTIG ? n + 1 : lines;
    const int bufsz = CONTIG ? lines * ld : lines * n;
    V *b0 = reinterpret_cast<V *>(smem_raw);
    V *b1 = b0 + bufsz;
    constexpr int K = Op::NRED > 0 ? Op::NRED : 1;
    double acc[K];
#pragma unroll
    for (int r = 0; r < K; r++) acc[r] = 0.0;

    const long long tile = g.reverse ? (long long)gridDim.x - 1 - blockIdx.x : (long long)blockIdx.x;
    const int solve = (int)(tile / g.tiles_per_solve);
    __shared__ typename Op::Ctx X;
    load_ctx(X, op.params(), op.scalars(), solve);
    __syncthreads();
    if (op.params() && !X.S.active) return;
    const void *streams[4];
    op.streams(streams);
    const V *__restrict__ src0 = reinterpret_cast<const V *>(streams[0]);
    auto lay_idx = [&](int line, int pos) { return CONTIG ? line * ld + pos : pos * lines + line; };
    const int total = lines * n;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        int line, pos;
        if (CONTIG) { pos = q % n; line = q / n; }
        else { line = q % lines; pos = q / lines; }
        LineRef lr = line_ref(g, tile, line);
        V val = mk<Real>(0, 0);
        if (lr.valid) {
            set_pos(g, lr, pos);
            const long long ge = lr.base + pos * g.estride;
            val = op.load(src0[ge], ge, lr, acc, X);
        }
        b0[lay_idx(line, pos)] = val;
    }
    __syncthreads();
    V *res;
    if (CONTIG) {
        LayContigRT lay{ld};
        res = (MODE == MODE_INV) ? smem_fft<1>(b0, b1, lines, ls, tw, lay)
                                 : smem_fft<-1>(b0, b1, lines, ls, tw, lay);
    } else {
        LayStrided lay{lines};
        res = (MODE == MODE_INV) ? smem_fft<1>(b0, b1, lines, ls, tw, lay)
                                 : smem_fft<-1>(b0, b1, lines, ls, tw, lay);
    }
    if (MODE == MODE_FWD_MID_INV) {
        for (int q = threadIdx.x; q < total; q += blockDim.x) {
            int line, pos;
            if (CONTIG) { pos = q % n; line = q / n; }
            else { line = q % lines; pos = q / lines; }
            LineRef lr = line_ref(g, tile, line);
            set_pos(g, lr, pos);
            const int s = lay_idx(line, pos);
            res[s] = op.mid(res[s], lr, X);
        }
        __syncthreads();
        V *other = (res == b0) ? b1 : b0;
        if (CONTIG) {
            LayContigRT lay{ld};
            res = smem_fft<1>(res, other, lines, ls, tw, lay);
        } else {
            LayStrided lay{lines};
            res = smem_fft<1>(res, other, lines, ls, tw, lay);
        }
    }
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        int line, pos;
        if (CONTIG) { pos = q % n; line = q / n; }
        else { line = q % lines; pos = q / lines; }
        LineRef lr = line_ref(g, tile, line);
        if (lr.valid) {
            set_pos(g, lr, pos);
            const long long ge = lr.base + pos * g.estride;
            const typename Op::Pre pre = op.pre(ge);
            op.post(ge, lr, res[lay_idx(line, pos)], pre, acc, X);
        }
    }
    reduce_and_finalize<Op::NRED>(acc, rs, op, solve, tile - (long long)solve * g.tiles_per_solve,
                                  g.tiles_per_solve);
}

// ---- point-wise kernel over all sites (reductions, scaling, conversions) -----------------
// Grid: nsolve * bps blocks; block b works on solve b / bps, sites of that solve strided by
// bps * blockDim.x.
template <class Op>
__global__ void __launch_bounds__(256) k_pointwise(const long long nsites, const int bps, Op op, const RedSlot rs) {
    pdl_enter();
    constexpr int K = Op::NRED > 0 ? Op::NRED : 1;
    const int solve = blockIdx.x / bps;
    const int lb = blockIdx.x - solve * bps;
    __shared__ typename Op::Ctx X;
    load_ctx(X, op.params(), op.scalars(), solve);
    __syncthreads();
    if (op.params() && !X.S.active) return;
    double acc[K];
#pragma unroll
    for (int r = 0; r < K; r++) acc[r] = 0.0;
    for (long long s = (long long)lb * blockDim.x + threadIdx.x; s < nsites; s += (long long)bps * blockDim.x)
        op.site(solve, s, acc, X);
    reduce_and_finalize<Op::NRED>(acc, rs, op, solve, lb, bps);
}

}  // namespace gp5

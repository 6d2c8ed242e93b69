// ring.cuh - the stage-boundary kernel fed by bulk copies: a persistent CTA per SM runs the
// x tiles of the boundary (inverse x, RK stage epilogue + next-stage prologue, forward x)
// while the tiles after it stream into a ring of shared-memory stages.
//
// Every tile is LINES consecutive x lines; each of its input streams (the transform buffer W,
// psi, k_{s-1}, the RK accumulator) is one contiguous range of LINES * N elements, copied by
// one cp.async.bulk (global -> shared, completion on the stage's mbarrier with a byte count).
// Thread 0 refills a stage as soon as every thread has finished reading it (the barrier
// before the forward transform), so GP5_RING_STAGES - 1 tiles are in flight while one is
// transformed.  The transform and the epilogue are those of the register engine
// (reg_fft, OpStageOut::turn / post); only the operand loads come from shared memory.
//
// Waits are bounded: a stage that has not arrived after `wait_ns` sets DS_TIMEOUT in the
// solve's status (and solve 0's), the CTA stops taking tiles, waits (bounded again, 2 s) for
// the copies it issued, so that none lands after the CTA has left, and returns.  No cluster,
// no multicast: each CTA copies into its own shared memory from this GPU's global memory.
#pragma once

#include "ops.cuh"
#include "passes.cuh"

namespace gp5 {

#ifndef GP5_RING_STAGES
#define GP5_RING_STAGES 3
#endif
constexpr int kRingStreamBytes = 16384;  // one stream of one tile
constexpr int kRingStreams = 4;
constexpr unsigned long long kRingDrainNs = GP5_RING_WAIT_DEFAULT_NS;  // bound of the final drain

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long ring_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void ring_bar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// one arrival (the barrier's only one per phase) announcing `bytes` of bulk copies
__device__ __forceinline__ void ring_expect(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// global -> this CTA's shared memory; both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void ring_copy(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// true once the phase of the given parity has completed, false after limit_ns (a limit of 0:
// after the first probe)
__device__ __forceinline__ bool ring_wait(unsigned long long *bar, unsigned parity, unsigned long long limit_ns) {
    const unsigned a = smem_addr(bar);
    unsigned ok = 0;
    asm volatile(
        "{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok || limit_ns == 0) return ok != 0;
    const unsigned long long t0 = ring_clock_ns();
    do {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    } while (ring_clock_ns() - t0 < limit_ns);
    return false;
}

// Tile shape: LINES lines of one stream fill kRingStreamBytes; threads = LINES x T.
template <typename Real, int N, int S> struct RingTile {
    using V = cpx<Real>;
    static constexpr int T = RegCfgAll<N, S>::T;
    static constexpr int LINES = kRingStreamBytes / (N * (int)sizeof(V));
    static constexpr int THREADS = LINES * T;
    static constexpr bool OK = LINES >= 1 && (THREADS == 128 || THREADS == 256);
    static constexpr int TILE = LINES * N;  // elements of one stream of one tile
    static constexpr size_t STAGE_ELEMS = (size_t)kRingStreams * TILE;
    static constexpr size_t SMEM =
        (size_t)GP5_RING_STAGES * STAGE_ELEMS * sizeof(V) + (size_t)LINES * LayContig<N, S>::LD * sizeof(V);
};

template <typename Real, int N, int S, bool RED>
__global__ void __launch_bounds__(RingTile<Real, N, S>::THREADS, 1)
    k_boundary_ring(const TileGeom g, const OpStageOut<Real, RED, true> op, const cpx<Real> *__restrict__ tw,
                    const RedSlot rs, const unsigned long long wait_ns) {
    using V = cpx<Real>;
    using RT = RingTile<Real, N, S>;
    using Op = OpStageOut<Real, RED, true>;
    constexpr int E = RegCfg<N, S>::E, T = RT::T, TILE = RT::TILE, ST = GP5_RING_STAGES;
    constexpr int NB = Op::BATCH;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    V *ring = reinterpret_cast<V *>(smem_raw);
    V *sm = ring + ST * RT::STAGE_ELEMS;  // exchange buffer of the transforms
    __shared__ __align__(8) unsigned long long full[ST];
    __shared__ SolveCtx X;
    __shared__ int s_abort;

    pdl_enter();
    const int tid = threadIdx.x % T, line = threadIdx.x / T;
    const void *streams[4];
    const int ns = op.streams(streams);
    const long long ntiles = g.ntiles, G = gridDim.x;
    // this CTA's tiles: blockIdx.x + k G (k = 0 .. mine-1), counted from the top when reversed
    const long long mine = (long long)blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
    auto tile_of = [&](long long k) {
        const long long t = blockIdx.x + k * G;
        return g.reverse ? ntiles - 1 - t : t;
    };
    auto issue = [&](long long k) {  // thread 0: the streams of tile k into stage k % ST
        const long long t = tile_of(k);
        const long long solve = t / g.tiles_per_solve, lt = t - solve * g.tiles_per_solve;
        const long long L0 = lt * RT::LINES;
        const long long L1 = L0 + RT::LINES < g.n_other ? L0 + RT::LINES : g.n_other;
        const unsigned bytes = (unsigned)((L1 - L0) * N * (long long)sizeof(V));
        const long long e0 = solve * g.solve_stride + L0 * N;
        V *stage = ring + (size_t)(k % ST) * RT::STAGE_ELEMS;
        ring_expect(&full[k % ST], bytes * (unsigned)ns);
        for (int q = 0; q < ns; q++)
            ring_copy(stage + (size_t)q * TILE, reinterpret_cast<const V *>(streams[q]) + e0, bytes, &full[k % ST]);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; s++) ring_bar_init(&full[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        for (long long k = 0; k < mine && k < ST; k++) issue(k);
    }
    __syncthreads();

    long long k = 0;
    for (; k < mine; k++) {
        const long long t = tile_of(k);
        const int solve = (int)(t / g.tiles_per_solve);
        const V *stage = ring + (size_t)(k % ST) * RT::STAGE_ELEMS;
        const unsigned long long cw = ctx_fetch(op.params(), op.scalars(), solve);
        const bool arrived = ring_wait(&full[k % ST], (unsigned)((k / ST) & 1), wait_ns);
        ctx_store(X, op.params(), op.scalars(), cw);
        if (!arrived) s_abort = 1;
        __syncthreads();
        if (s_abort) break;
        double acc[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
        for (int r = 0; r < (Op::NRED > 0 ? Op::NRED : 1); r++) acc[r] = 0.0;
        const LineRef lr = line_ref(g, t, line);
        const bool active = !op.params() || X.S.active;
        V v[E];
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = stage[line * N + tid + T * m];
        LayContig<N, S> lay;
        reg_fft<N, S, 1>(v, tid, line, tw, sm, lay);
#pragma unroll
        for (int m = 0; m < E; m++) sm[lay(line, tid + T * m)] = v[m];
        if (lr.valid && active) {
            // the stage epilogue, operands from the ring (streams 1..3: psi, k_{s-1}, accumulator)
            const StageK<Real> K = op.consts(X);
#pragma unroll 1
            for (int m0 = 0; m0 < E; m0 += NB) {
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const int pos = tid + T * (m0 + j);
                    const int o = line * N + pos;
                    EpiIn<Real> in;
                    in.psi = stage[TILE + o];
                    in.kprev = ns > 2 ? stage[2 * TILE + o] : mk<Real>(0, 0);
                    in.kacc = ns > 3 ? stage[3 * TILE + o] : mk<Real>(0, 0);
                    in.lo = mk<Real>(0, 0);
                    LineRef e = lr;
                    set_pos(g, e, pos);
                    const int si = lay(line, pos);
                    sm[si] = op.turn(lr.base + pos, e, sm[si], in, acc, X, K);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = sm[lay(line, tid + T * m)];
        __syncthreads();
        // every thread is past its reads of this stage: refill it with the tile ST ahead
        if (threadIdx.x == 0 && k + ST < mine) issue(k + ST);
        reg_fft<N, S, -1>(v, tid, line, tw, sm, lay);
        if (lr.valid && active) {
#pragma unroll
            for (int m = 0; m < E; m++) {
                const int pos = tid + T * m;
                LineRef e = lr;
                set_pos(g, e, pos);
                op.post(lr.base + pos, e, v[m], EpiIn<Real>{}, acc, X);
            }
        }
        // a finished solve of a batch takes no part in the reductions (uniform over the CTA)
        if (active)
            reduce_and_finalize<Op::NRED>(acc, rs, op, solve, t - (long long)solve * g.tiles_per_solve,
                                          g.tiles_per_solve);
        __syncthreads();  // the exchange buffer and X are free for the next tile
    }
    if (s_abort && threadIdx.x == 0) {
        const long long t = tile_of(k);
        const int solve = (int)(t / g.tiles_per_solve);
        if (op.scalars()) {
            atomicOr(&const_cast<DevScalars *>(op.scalars())[solve].status, (unsigned)DS_TIMEOUT);
            atomicOr(&const_cast<DevScalars *>(op.scalars())[0].status, (unsigned)DS_TIMEOUT);
        }
        // the copies already issued (tiles k .. k + ST - 1) still land in this CTA's shared
        // memory: wait for them, bounded, before the CTA exits
        for (long long q = k; q < mine && q < k + ST; q++)
            ring_wait(&full[q % ST], (unsigned)((q / ST) & 1), kRingDrainNs);
    }
}

}  // namespace gp5

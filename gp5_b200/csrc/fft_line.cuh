// fft_line.cuh - line FFT engines for the axis passes.
//
// Both engines run the Stockham autosort formulation of the mixed-radix Cooley-Tukey DFT
// (each pass: gather R inputs at stride n/R, twiddle, DFT-R, scatter in autosorted order),
// so results come out in natural order without a bit-reversal pass:
//
//   pass with radix R after radices of product Ns:
//     butterfly b in [0, n/R): inputs  x[b + r n/R]              (r in [0,R))
//                              twiddle x_r *= W_{Ns R}^{r (b mod Ns)}
//                              outputs y[(b/Ns) Ns R + (b mod Ns) + r Ns]
//
// * RegEngine<N>: N a power of two in [16, 1024].  Each of T = N/E threads of a line owns E
//   elements at positions tid + T*m for the whole transform; passes run in registers and
//   exchange through shared memory only between passes (one exchange for N <= 256).
// * The shared-memory engine (smem_fft) handles any length whose prime factors are <= 61,
//   with ping-pong buffers; it serves the non-power-of-two grids of the reference's tests.
//
// Sign convention (FFTW, src/fourierTransform.cpp:155-162): DIR = -1 forward e^{-2 pi i jk/n},
// DIR = +1 backward e^{+2 pi i jk/n}, both unnormalised.  Twiddles come from a per-length
// table tw[j] = e^{-2 pi i j/n} computed on the host in long double; the backward
// transform uses its conjugate.
#pragma once

#include "common.cuh"

namespace gp5 {

// ------------------------------------------------------------------------------------------
// small DFT kernels (compile-time radix), DIR = -1 forward / +1 backward
// ------------------------------------------------------------------------------------------
// cos(pi/8), sin(pi/8), sqrt(1/2), and the radix-3/5 constants, from their closed forms.
#define GP5_C8 0.92387953251128675612818318939678829
#define GP5_S8 0.38268343236508977172845998403039887
#define GP5_R2 0.70710678118654752440084436210484904
#define GP5_S3 0.86602540378443864676372317075293618   /* sqrt(3)/2 */
#define GP5_C51 0.30901699437494742410229341718281906  /* cos(2 pi/5) */
#define GP5_C52 -0.80901699437494742410229341718281906 /* cos(4 pi/5) */
#define GP5_S51 0.95105651629515357211643933337938214  /* sin(2 pi/5) */
#define GP5_S52 0.58778525229247312916870595463907277  /* sin(4 pi/5) */

template <int DIR, typename V> __device__ __forceinline__ void dft2(V &a, V &b) {
    V t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR, typename V> __device__ __forceinline__ void dft4(V &x0, V &x1, V &x2, V &x3) {
    V a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = mul_i<DIR>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

// W_16^m (sign DIR) applied to v, m compile-time in [0, 16)
template <int DIR, int M, typename V> __device__ __forceinline__ V tw16(V v) {
    using R = decltype(v.x);
    constexpr int m = M & 15;
    if constexpr (m == 0) return v;
    else if constexpr (m == 4) return mul_i<DIR>(v);
    else if constexpr (m == 8) { V r; r.x = -v.x; r.y = -v.y; return r; }
    else if constexpr (m == 12) return mul_i<-DIR>(v);
    else {
        // cos(2 pi m/16), sin(2 pi m/16) from the first-octant constants
        constexpr double cs[16] = {1, GP5_C8, GP5_R2, GP5_S8, 0, -GP5_S8, -GP5_R2, -GP5_C8,
                                   -1, -GP5_C8, -GP5_R2, -GP5_S8, 0, GP5_S8, GP5_R2, GP5_C8};
        constexpr double sn[16] = {0, GP5_S8, GP5_R2, GP5_C8, 1, GP5_C8, GP5_R2, GP5_S8,
                                   0, -GP5_S8, -GP5_R2, -GP5_C8, -1, -GP5_C8, -GP5_R2, -GP5_S8};
        V w;
        w.x = (R)cs[m];
        w.y = (R)(DIR * sn[m]);
        return cmul(v, w);
    }
}

template <int DIR, typename V> __device__ __forceinline__ void dft8(V (&x)[8]) {
    // radix-2 over two radix-4 halves
    dft4<DIR>(x[0], x[2], x[4], x[6]);
    dft4<DIR>(x[1], x[3], x[5], x[7]);
    // x[0],x[2],x[4],x[6] hold E0..E3 ; x[1],x[3],x[5],x[7] hold O0..O3
    V o1 = tw16<DIR, 2>(x[3]), o2 = tw16<DIR, 4>(x[5]), o3 = tw16<DIR, 6>(x[7]);
    V e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1];
    x[0] = cadd(e0, o0); x[4] = csub(e0, o0);
    x[1] = cadd(e1, o1); x[5] = csub(e1, o1);
    x[2] = cadd(e2, o2); x[6] = csub(e2, o2);
    x[3] = cadd(e3, o3); x[7] = csub(e3, o3);
}

template <int DIR, typename V> __device__ __forceinline__ void dft16(V (&x)[16]) {
    // n = 4 n1 + n2, k = k1 + 4 k2
    dft4<DIR>(x[0], x[4], x[8], x[12]);
    dft4<DIR>(x[1], x[5], x[9], x[13]);
    dft4<DIR>(x[2], x[6], x[10], x[14]);
    dft4<DIR>(x[3], x[7], x[11], x[15]);
    // A[n2][k1] sits in x[n2 + 4 k1]; twiddle by W16^{n2 k1}
    x[5] = tw16<DIR, 1>(x[5]);  x[9] = tw16<DIR, 2>(x[9]);   x[13] = tw16<DIR, 3>(x[13]);
    x[6] = tw16<DIR, 2>(x[6]);  x[10] = tw16<DIR, 4>(x[10]); x[14] = tw16<DIR, 6>(x[14]);
    x[7] = tw16<DIR, 3>(x[7]);  x[11] = tw16<DIR, 6>(x[11]); x[15] = tw16<DIR, 9>(x[15]);
    dft4<DIR>(x[0], x[1], x[2], x[3]);
    dft4<DIR>(x[4], x[5], x[6], x[7]);
    dft4<DIR>(x[8], x[9], x[10], x[11]);
    dft4<DIR>(x[12], x[13], x[14], x[15]);
    // X[k1 + 4 k2] now in x[4 k1 + k2]: transpose the 4x4 index
    V t;
    t = x[1]; x[1] = x[4]; x[4] = t;
    t = x[2]; x[2] = x[8]; x[8] = t;
    t = x[3]; x[3] = x[12]; x[12] = t;
    t = x[6]; x[6] = x[9]; x[9] = t;
    t = x[7]; x[7] = x[13]; x[13] = t;
    t = x[11]; x[11] = x[14]; x[14] = t;
}

template <int DIR, typename V> __device__ __forceinline__ void dft3(V &x0, V &x1, V &x2) {
    using R = decltype(x0.x);
    V t1 = cadd(x1, x2), t2 = csub(x1, x2);
    V m;
    m.x = x0.x - (R)0.5 * t1.x;
    m.y = x0.y - (R)0.5 * t1.y;
    V s = mul_i<DIR>(cscale(t2, (R)GP5_S3));
    x0 = cadd(x0, t1);
    x1 = cadd(m, s);
    x2 = csub(m, s);
}

template <int DIR, typename V> __device__ __forceinline__ void dft5(V (&x)[5]) {
    using R = decltype(x[0].x);
    V a1 = cadd(x[1], x[4]), b1 = csub(x[1], x[4]);
    V a2 = cadd(x[2], x[3]), b2 = csub(x[2], x[3]);
    V x0 = x[0];
    V p1, p2;
    p1.x = x0.x + (R)GP5_C51 * a1.x + (R)GP5_C52 * a2.x;
    p1.y = x0.y + (R)GP5_C51 * a1.y + (R)GP5_C52 * a2.y;
    p2.x = x0.x + (R)GP5_C52 * a1.x + (R)GP5_C51 * a2.x;
    p2.y = x0.y + (R)GP5_C52 * a1.y + (R)GP5_C51 * a2.y;
    V q1, q2;
    q1.x = (R)GP5_S51 * b1.x + (R)GP5_S52 * b2.x;
    q1.y = (R)GP5_S51 * b1.y + (R)GP5_S52 * b2.y;
    q2.x = (R)GP5_S52 * b1.x - (R)GP5_S51 * b2.x;
    q2.y = (R)GP5_S52 * b1.y - (R)GP5_S51 * b2.y;
    q1 = mul_i<DIR>(q1);
    q2 = mul_i<DIR>(q2);
    x[0] = cadd(x0, cadd(a1, a2));
    x[1] = cadd(p1, q1);
    x[4] = csub(p1, q1);
    x[2] = cadd(p2, q2);
    x[3] = csub(p2, q2);
}

// compile-time radix dispatch on a register array
template <int R, int DIR, typename V> __device__ __forceinline__ void dft_r(V (&x)[R]) {
    if constexpr (R == 2) dft2<DIR>(x[0], x[1]);
    else if constexpr (R == 4) dft4<DIR>(x[0], x[1], x[2], x[3]);
    else if constexpr (R == 8) dft8<DIR>(x);
    else if constexpr (R == 16) dft16<DIR>(x);
    else if constexpr (R == 3) dft3<DIR>(x[0], x[1], x[2]);
    else if constexpr (R == 5) dft5<DIR>(x);
    else static_assert(R == 2, "unsupported compile-time radix");
}

// twiddle W_n^j from the forward table, conjugated for the backward direction
template <int DIR, typename V> __device__ __forceinline__ V twiddle(const V *__restrict__ tw, int j) {
    V w = __ldg(tw + j);
    if (DIR > 0) w.y = -w.y;
    return w;
}

// ------------------------------------------------------------------------------------------
// register engine: N = 2^p, radix schedule fixed at compile time.  Two schedules per length:
// S = 0 and S = 1 differ in the elements a thread owns (E) and so in the threads per line
// (N / E), the passes and the registers a thread needs; the plan's autotuner picks one per
// pass.  The two round differently (other butterflies, other twiddle products), so a plan
// keeps its choice for every plan of the same grid and precision (see autotune_plan).
// ------------------------------------------------------------------------------------------
template <int N, int S = 0> struct RegCfg;
template <> struct RegCfg<16, 0> { static constexpr int E = 4, NP = 2; static constexpr int rad(int p) { return 4; } };
template <> struct RegCfg<32, 0> { static constexpr int E = 8, NP = 2; static constexpr int rad(int p) { return p == 0 ? 8 : 4; } };
template <> struct RegCfg<64, 0> { static constexpr int E = 8, NP = 2; static constexpr int rad(int p) { return 8; } };
template <> struct RegCfg<128, 0> { static constexpr int E = 16, NP = 2; static constexpr int rad(int p) { return p == 0 ? 16 : 8; } };
template <> struct RegCfg<256, 0> { static constexpr int E = 16, NP = 2; static constexpr int rad(int p) { return 16; } };
template <> struct RegCfg<512, 0> { static constexpr int E = 8, NP = 3; static constexpr int rad(int p) { return 8; } };
template <> struct RegCfg<1024, 0> { static constexpr int E = 16, NP = 3; static constexpr int rad(int p) { return p == 2 ? 4 : 16; } };
// S = 1: half the elements per thread (twice the threads per line, fewer registers), except
// 512 (twice the elements: radix-16 passes)
template <> struct RegCfg<16, 1> : RegCfg<16, 0> {};
template <> struct RegCfg<32, 1> { static constexpr int E = 4, NP = 3; static constexpr int rad(int p) { return p == 2 ? 2 : 4; } };
template <> struct RegCfg<64, 1> { static constexpr int E = 4, NP = 3; static constexpr int rad(int p) { return 4; } };
template <> struct RegCfg<128, 1> { static constexpr int E = 8, NP = 3; static constexpr int rad(int p) { return p == 2 ? 2 : 8; } };
template <> struct RegCfg<256, 1> { static constexpr int E = 8, NP = 3; static constexpr int rad(int p) { return p == 2 ? 4 : 8; } };
template <> struct RegCfg<512, 1> { static constexpr int E = 16, NP = 3; static constexpr int rad(int p) { return p == 2 ? 2 : 16; } };
template <> struct RegCfg<1024, 1> : RegCfg<1024, 0> {};

template <int N, int S = 0> struct RegCfgAll : RegCfg<N, S> {
    static constexpr int T = N / RegCfg<N, S>::E;
    static constexpr int ns(int p) { return p == 0 ? 1 : ns(p - 1) * RegCfg<N, S>::rad(p - 1); }
};

// Shared-memory index maps for the exchange between passes.
//  * strided-axis tiles: element (line, pos) at pos*LINES + line (lanes run over lines)
//  * x-axis tiles: element (line, pos) at line*LD + pos + pos/P, one pad slot every P elements
//    (P = 16, or the first pass's radix for S = 1) so that the stride-P scatter of the first
//    pass spreads over the banks
struct LayStrided {
    int lines;
    __device__ __forceinline__ int operator()(int line, int pos) const { return pos * lines + line; }
};
template <int N, int S = 0> struct LayContig {
    static constexpr int P = S == 0 ? 16 : RegCfg<N, S>::rad(0);
    static constexpr int LD = N + N / P + 1;
    __device__ __forceinline__ int operator()(int line, int pos) const { return line * LD + pos + pos / P; }
};

// One Stockham pass P of the register engine on the E registers of one line-thread.
template <int N, int S, int P, int DIR, typename V, class Lay>
__device__ __forceinline__ void reg_pass(V (&v)[RegCfg<N, S>::E], int tid, int line,
                                         const V *__restrict__ tw, V *sm, const Lay &lay) {
    using C = RegCfgAll<N, S>;
    constexpr int E = C::E, T = C::T, R = C::rad(P), Ns = C::ns(P);
    constexpr bool last = (P == C::NP - 1);
#pragma unroll
    for (int t = 0; t < E / R; t++) {
        const int b = tid + t * T;
        V x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = v[t + r * (E / R)];
        if constexpr (Ns > 1) {
            const int bm = b % Ns;
            constexpr int step = N / (Ns * R);
            if constexpr (R == 16) {
                // w^r for r = 1..15 from four table entries (w, w^2, w^4, w^8); every power is
                // a product of at most four exactly rounded table values (<= 3 extra roundings)
                const V w1 = twiddle<DIR>(tw, bm * step), w2 = twiddle<DIR>(tw, 2 * bm * step);
                const V w4 = twiddle<DIR>(tw, 4 * bm * step), w8 = twiddle<DIR>(tw, 8 * bm * step);
                const V w3 = cmul(w2, w1), w12 = cmul(w8, w4);
                x[1] = cmul(x[1], w1);
                x[2] = cmul(x[2], w2);
                x[3] = cmul(x[3], w3);
                x[4] = cmul(x[4], w4);
                x[5] = cmul(x[5], cmul(w4, w1));
                x[6] = cmul(x[6], cmul(w4, w2));
                x[7] = cmul(x[7], cmul(w4, w3));
                x[8] = cmul(x[8], w8);
                x[9] = cmul(x[9], cmul(w8, w1));
                x[10] = cmul(x[10], cmul(w8, w2));
                x[11] = cmul(x[11], cmul(w8, w3));
                x[12] = cmul(x[12], w12);
                x[13] = cmul(x[13], cmul(w12, w1));
                x[14] = cmul(x[14], cmul(w12, w2));
                x[15] = cmul(x[15], cmul(w12, w3));
            } else {
#pragma unroll
                for (int r = 1; r < R; r++) x[r] = cmul(x[r], twiddle<DIR>(tw, r * bm * step));
            }
        }
        dft_r<R, DIR>(x);
        if constexpr (last) {
#pragma unroll
            for (int r = 0; r < R; r++) v[t + r * (E / R)] = x[r];
        } else {
            const int base = (b / Ns) * Ns * R + (b % Ns);
#pragma unroll
            for (int r = 0; r < R; r++) sm[lay(line, base + r * Ns)] = x[r];
        }
    }
    if constexpr (!last) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = sm[lay(line, tid + T * m)];
        __syncthreads();
    }
}

template <int N, int S, int P, int DIR, typename V, class Lay>
__device__ __forceinline__ void reg_fft_from(V (&v)[RegCfg<N, S>::E], int tid, int line,
                                             const V *__restrict__ tw, V *sm, const Lay &lay) {
    if constexpr (P < RegCfg<N, S>::NP) {
        reg_pass<N, S, P, DIR>(v, tid, line, tw, sm, lay);
        reg_fft_from<N, S, P + 1, DIR>(v, tid, line, tw, sm, lay);
    }
}

// Full length-N transform of the line held in v (positions tid + T*m in, and out), schedule S.
template <int N, int S, int DIR, typename V, class Lay>
__device__ __forceinline__ void reg_fft(V (&v)[RegCfg<N, S>::E], int tid, int line,
                                        const V *__restrict__ tw, V *sm, const Lay &lay) {
    reg_fft_from<N, S, 0, DIR>(v, tid, line, tw, sm, lay);
}

// ------------------------------------------------------------------------------------------
// shared-memory engine: any length with prime factors <= 61
// ------------------------------------------------------------------------------------------
constexpr int kMaxRadix = 64;
constexpr int kMaxPasses = 16;

struct LineSchedule {
    int n;
    int np;
    int rad[kMaxPasses];
};

template <int DIR, typename V>
__device__ __forceinline__ void dft_generic(V *x, int R, int n, const V *__restrict__ tw) {
    // direct O(R^2) DFT with W_R^a = W_n^{a n/R}
    V y[kMaxRadix];
    const int step = n / R;
    for (int k = 0; k < R; k++) {
        V s = x[0];
        int a = 0;
        for (int r = 1; r < R; r++) {
            a += k;
            if (a >= R) a -= R;
            s = cadd(s, cmul(x[r], twiddle<DIR>(tw, a * step)));
        }
        y[k] = s;
    }
    for (int k = 0; k < R; k++) x[k] = y[k];
}

// One pass over all lines of a tile: src -> dst (both shared memory).  Work items are
// (line, butterfly) pairs, lines fastest so that neighbouring threads touch neighbouring
// words in the strided layout.
template <int DIR, typename V, class Lay>
__device__ void smem_pass(const V *src, V *dst, int lines, int n, int R, int Ns,
                          const V *__restrict__ tw, const Lay &lay) {
    const int nb = n / R;
    const int total = lines * nb;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int line = q % lines, b = q / lines;
        const int bm = b % Ns;
        const int tstep = n / (Ns * R);
        V x[kMaxRadix];
        for (int r = 0; r < R; r++) {
            V e = src[lay(line, b + r * nb)];
            if (Ns > 1 && r > 0) e = cmul(e, twiddle<DIR>(tw, r * bm * tstep));
            x[r] = e;
        }
        switch (R) {
            case 2: dft2<DIR>(x[0], x[1]); break;
            case 3: dft3<DIR>(x[0], x[1], x[2]); break;
            case 4: dft4<DIR>(x[0], x[1], x[2], x[3]); break;
            case 5: dft5<DIR>(*reinterpret_cast<V(*)[5]>(x)); break;
            case 8: dft8<DIR>(*reinterpret_cast<V(*)[8]>(x)); break;
            default: dft_generic<DIR>(x, R, n, tw); break;
        }
        const int base = (b / Ns) * Ns * R + bm;
        for (int r = 0; r < R; r++) dst[lay(line, base + r * Ns)] = x[r];
    }
}

// Runs the schedule; data starts in buf[0], returns the buffer holding the result.
template <int DIR, typename V, class Lay>
__device__ V *smem_fft(V *buf0, V *buf1, int lines, const LineSchedule &s,
                       const V *__restrict__ tw, const Lay &lay) {
    V *src = buf0, *dst = buf1;
    int Ns = 1;
    for (int p = 0; p < s.np; p++) {
        smem_pass<DIR>(src, dst, lines, s.n, s.rad[p], Ns, tw, lay);
        __syncthreads();
        Ns *= s.rad[p];
        V *t = src; src = dst; dst = t;
    }
    return src;
}

}  // namespace gp5

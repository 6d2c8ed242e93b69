// ops.cuh - the point-wise arithmetic of the GP hot path, written as hooks that the axis
// passes call on every element they load, transform or store.
//
// Reference arithmetic restated here (lucaparisi91/GP5):
//   kinetic       operators.cpp:7-36 (K^2 = KX*KX + KY*KY + KZ*KZ; IFFT(-K^2 FFT)/N^3) with
//                 functional.cpp:24 / :118 (-1/2, 1/m): one multiplier K^2/(2 m N^3) in k-space
//   positions     geometry.cpp:184 (x = left + dx (i + 1/2)); momenta geometry.cpp:127-148
//   potential     functional.cpp:46-53; harmonic V = (wx wx x x + wy wy y y + wz wz z z) 0.5,
//                 externalPotential.cpp:26
//   interaction   GP 1 comp functional.cpp:54-68; 2 comp :71-89; LHY :112-119 (n^{3/2}
//                 evaluated as n*sqrt(n)); unlocked LHY :125-150
//   RK4 stages    stepper.cpp:46-71;  Euler stepper.cpp:30-44
//   normalize     geometry.cpp:190-229 (applied lazily as a device-side scale)
//   phase constr. constraint.cpp:6-9
//
// Every launch may carry several independent solves of one grid ("solve" index of a tile).
// Their parameters (box, couplings, time step, targets) come from a SolveParams array and
// their scalars (pending scales, sums) from a DevScalars array, both indexed by solve.
// Positions and K^2 are formed with explicitly rounded operations (no contraction), so they
// equal the host-side (and the reference's) values bit for bit.
#pragma once

#include <cuda_bf16.h>

#include "passes.cuh"

namespace gp5 {

constexpr int kNRed = 8;

// ---- per-solve device data ---------------------------------------------------------------
struct DevScalars {
    double sigma[2];     // pending scale of the state (1 when clean)
    double alpha[2][2];  // [stage & 1][component]: scale of the stage's transform input
    double sums[8];      // last reduction result (raw sums, not yet times dV)
    double mu;           // chemical potential for the residual pass
    double factor;       // scale factor for normalize
    unsigned status;     // DevStatus bits
    unsigned pad;
};

struct SolveParams {
    double dk[3];           // Fourier steps 2 pi / L_d
    double left[3], dx[3];  // cell-centred x_d = left_d + dx_d (i + 1/2)
    double dV;
    double kin[2];          // kinetic multiplier 1/(2 m_c N^3) (or -1/N^3 for the Laplacian)
    double c3, c4;          // LHY: H = -1/2 lap + (c3 n + c4 n^{3/2})
    double g00, g01, g11;   // GP couplings
    double la, lb, le;      // unlocked LHY alpha, beta, eta
    double om2[2][3];       // harmonic trap: w_d * w_d per component
    double Nt[2];           // normalisation targets
    double tre, tim;        // complex time step
    int active;             // 0: this solve is finished; its tiles return at once
    int pad_;
};

// Per-CTA copy (shared memory) of the solve's parameters and of the scalars the kernel reads;
// filled once at kernel start so that element loops read them without aliasing global stores.
struct SolveCtx {
    SolveParams S;
    double sigma[2];
    double alpha[2][2];
};

// The context is fetched in two halves so that its global loads overlap the tile's loads:
// ctx_fetch issues them into one register per thread (threads 0..30: SolveParams words,
// threads 32..37: sigma and alpha), ctx_store writes them to shared memory (then sync).
constexpr int kCtxWords = (int)(sizeof(SolveParams) / 8);
static_assert(kCtxWords <= 32, "SolveParams must fit one warp's fetch");

__device__ __forceinline__ unsigned long long ctx_fetch(const SolveParams *sp, const DevScalars *ds, int solve) {
    const int t = threadIdx.x;
    if (sp && t < kCtxWords) return __ldg(reinterpret_cast<const unsigned long long *>(sp + solve) + t);
    if (ds && t >= 32 && t < 38) {
        const DevScalars &d = ds[solve];
        const double v = (t < 34) ? d.sigma[t - 32] : d.alpha[(t - 34) >> 1][(t - 34) & 1];
        return (unsigned long long)__double_as_longlong(v);
    }
    return 0ull;
}

__device__ __forceinline__ void ctx_store(SolveCtx &X, const SolveParams *sp, const DevScalars *ds,
                                          unsigned long long w) {
    const int t = threadIdx.x;
    if (sp && t < kCtxWords) reinterpret_cast<unsigned long long *>(&X.S)[t] = w;
    if (ds && t >= 32 && t < 38) {
        const double v = __longlong_as_double((long long)w);
        if (t < 34) X.sigma[t - 32] = v;
        else X.alpha[(t - 34) >> 1][(t - 34) & 1] = v;
    }
}

__device__ __forceinline__ void load_ctx(SolveCtx &X, const SolveParams *sp, const DevScalars *ds, int solve) {
    ctx_store(X, sp, ds, ctx_fetch(sp, ds, solve));
}

__device__ __forceinline__ double position(const SolveParams &S, int d, int i) {
    return __dadd_rn(S.left[d], __dmul_rn(S.dx[d], (double)i + 0.5));
}
// k = dk * m with m = i below the Nyquist split, i - n above (even n: Nyquist -> -n/2)
__device__ __forceinline__ double momentum(const SolveParams &S, int d, int i, int n) {
    const int half = (n % 2 == 0) ? n / 2 : (n - 1) / 2 + 1;
    return __dmul_rn(S.dk[d], (double)(i < half ? i : i - n));
}

// ---- hook interface ----------------------------------------------------------------------
//   params(), scalars()      per-solve arrays copied into the CTA's SolveCtx X (may be null)
//   load(x, g, e, acc, X)    value entering the transform (x = first stream at element g)
//   mid(v, e, X)             k-space multiply between a forward and an inverse transform
//   pre(g) -> Pre            operand loads of the epilogue (issued BATCH elements at a time)
//   post(g, e, v, pre, acc, X)  epilogue: consume the transformed value and store
//   streams(p)               arrays the pass reads (first: the one the prologue loads)
//   finalize(sums, solve)    last block of a solve, with the FP64 sums of NRED accumulators
struct NoPre {};

template <typename Real> struct OpCopy {
    static constexpr int NRED = 0, BATCH = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *src;
    V *dst;
    const SolveParams *sp;  // may be null: every solve active
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &, const SolveCtx &) const { return v; }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *, const SolveCtx &) const {
        dst[g] = v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const { p[0] = src; return 1; }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

// z pass of an H application: forward z, times K^2 kin_c, inverse z.
template <typename Real> struct OpKinetic {
    static constexpr int NRED = 0, BATCH = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *src;
    V *dst;
    const SolveParams *sp;
    int nx, ny, nz;
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const double kx = momentum(S, 0, e.i, nx), ky = momentum(S, 1, e.j, ny), kz = momentum(S, 2, e.k, nz);
        const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
        return cscale(v, (Real)(k2 * S.kin[e.c]));
    }
    // z lines: kx^2 + ky^2 is fixed along the line, so it is formed once and each element adds
    // its own kz^2; kidx is kz's signed index.  complex128: the same operations in the same
    // order as mid (bit-identical).  complex64: the per-element part runs in FP32 (one
    // rounding of kx^2 + ky^2 per line; the factor's error stays below the transform's).
    static constexpr bool MID_Z = true;
    struct MidLine {
        Real kxy2, dkz, kin;
    };
    __device__ __forceinline__ MidLine mid_line(const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const double kx = momentum(S, 0, e.i, nx), ky = momentum(S, 1, e.j, ny);
        return MidLine{(Real)__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), (Real)S.dk[2], (Real)S.kin[e.c]};
    }
    __device__ __forceinline__ V mid_z(V v, int kidx, const MidLine &L) const {
        if constexpr (sizeof(Real) == 8) {
            const double kz = __dmul_rn(L.dkz, (double)kidx);
            const double k2 = __dadd_rn(L.kxy2, __dmul_rn(kz, kz));
            return cscale(v, (Real)(k2 * L.kin));
        } else {
            const float kz = L.dkz * (float)kidx;
            return cscale(v, (L.kxy2 + kz * kz) * L.kin);
        }
    }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *, const SolveCtx &) const {
        dst[g] = v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const { p[0] = src; return 1; }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

// ---- stage input (prologue of the first forward pass) -----------------------------------
// u~ = sigma_c psi - c kprev (c = tau * cfac); optional sum |u~|^2 per component ->
// alpha_c = sqrt(N_c / (dV S)) in alpha[slot].
// One axis's term of the kinetic operator, (1/2m)(-d^2/dx_d^2) u, in its 1D spectral form
// IFFT_d(k_d^2 / (2 m N_d) FFT_d u): the sum of the three axes' terms is the 3D form
// IFFT(K^2/(2 m N) FFT u) because K^2 = kx^2 + ky^2 + kz^2 and the axis transforms commute.
// The y and z passes of the per-axis stepper scheme (Launch::step_axes) run it from the stage
// input u into T (ACC = false) or added to T (ACC = true); the x term is formed inside the
// stage boundary (OpStageAxes).  The factor 1/(2 m N_d) is kin * (N / N_d) with kin = 1/(2 m N).
template <typename Real, int AXIS, bool ACC> struct OpDeriv {
    static constexpr int NRED = 0, BATCH = ACC ? 4 : 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    struct Pre {
        V t;
    };
    const V *src;
    V *dst;
    const SolveParams *sp;
    int nx, ny, nz;
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ double axis_factor(const SolveParams &S, int c) const {
        const double other = AXIS == 0 ? (double)ny * nz : (AXIS == 1 ? (double)nx * nz : (double)nx * ny);
        return __dmul_rn(S.kin[c], other);
    }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const int pos = AXIS == 0 ? e.i : (AXIS == 1 ? e.j : e.k);
        const double k = momentum(S, AXIS, pos, AXIS == 0 ? nx : (AXIS == 1 ? ny : nz));
        return cscale(v, (Real)(__dmul_rn(k, k) * axis_factor(S, e.c)));
    }
    // z lines: the per-line part is the factor; each element forms its own kz^2
    static constexpr bool MID_Z = true;
    struct MidLine {
        Real dkz;
        double fac;
    };
    __device__ __forceinline__ MidLine mid_line(const LineRef &e, const SolveCtx &X) const {
        return MidLine{(Real)X.S.dk[2], axis_factor(X.S, e.c)};
    }
    __device__ __forceinline__ V mid_z(V v, int kidx, const MidLine &L) const {
        if constexpr (sizeof(Real) == 8) {
            const double kz = __dmul_rn(L.dkz, (double)kidx);
            return cscale(v, (Real)(__dmul_rn(kz, kz) * L.fac));
        } else {
            const float kz = L.dkz * (float)kidx;
            return cscale(v, kz * kz * (float)L.fac);
        }
    }
    __device__ __forceinline__ Pre pre(long long g) const {
        Pre p;
        if (ACC) p.t = dst[g];
        return p;
    }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &in, double *,
                                         const SolveCtx &) const {
        dst[g] = ACC ? cadd(in.t, v) : v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        p[0] = src;
        if (ACC) { p[1] = dst; return 2; }
        return 1;
    }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

template <typename Real, bool RED> struct OpStageIn {
    static constexpr int NRED = RED ? 2 : 0, BATCH = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *psi;
    const V *kprev;  // null for the first stage
    V *dst;
    DevScalars *ds;
    const SolveParams *sp;
    int use_sigma;
    double cfac;
    int slot;
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return ds; }
    __device__ __forceinline__ V load(V p, long long g, const LineRef &e, double *acc, const SolveCtx &X) const {
        if (use_sigma) p = cscale(p, (Real)X.sigma[e.c]);
        if (kprev) {
            const SolveParams &S = X.S;
            V c;
            c.x = (Real)(S.tre * cfac);
            c.y = (Real)(S.tim * cfac);
            p = csub(p, cmul(c, kprev[g]));
        }
        if (RED) {
            const double n = (double)p.x * (double)p.x + (double)p.y * (double)p.y;
            if (e.c == 0) acc[0] += n;
            else acc[1] += n;
        }
        return p;
    }
    __device__ __forceinline__ V mid(V v, const LineRef &, const SolveCtx &) const { return v; }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *, const SolveCtx &) const {
        dst[g] = v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        p[0] = psi;
        if (kprev) { p[1] = kprev; return 2; }
        return 1;
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const {
        if (RED) {
            const SolveParams &S = sp[solve];
            DevScalars &d = ds[solve];
            d.alpha[slot][0] = sqrt(S.Nt[0] / (S.dV * s[0]));
            d.alpha[slot][1] = (S.Nt[1] > 0) ? sqrt(S.Nt[1] / (S.dV * s[1])) : 1.0;
            if (!isfinite(s[0]) || !isfinite(s[1]) || !isfinite(d.alpha[slot][0])) d.status |= DS_NONFINITE;
        }
    }
};

// ---- the stage epilogue -------------------------------------------------------------------
enum EpiMode : int {
    EPI_H = 0,      // dst = H src
    EPI_OBS = 1,    // dst = H src, with the observable sums
    EPI_EULER = 2,  // psi <- psi - tau H psi
    EPI_RK1 = 3,
    EPI_RK2 = 4,
    EPI_RK3 = 5,
    EPI_RK4 = 6,
};
enum FuncKind : int { FK_GP = 0, FK_LHY = 1, FK_LHY_UNLOCKED = 2 };

template <typename Real> struct EpiParams {
    using V = cpx<Real>;
    long long nsites;  // sites per solve (component offset)
    int mode;
    // state (element indices include the solve offset)
    const V *psi;  // stage base psi0 (read); EPI_H/OBS: the source field
    V *psi_out;    // EULER / RK4 result (may alias psi)
    const V *kprev;
    V *kout;       // k_s (RK1 -> Ka, RK2 -> Kb, RK3 -> Kb) or H src (H/OBS)
    V *kacc;       // Ka: RK accumulator (RK2/RK3/RK4)
    const V *tsrc; // kinetic buffer for the non-fused (2 component) epilogue
    DevScalars *ds;          // [solve]
    const SolveParams *sp;   // [solve]
    int use_sigma, use_alpha;
    int slot;       // alpha slot of this stage (stage & 1)
    int u1_raw;     // first stage / Euler: the transform input was the raw state (its pending
                    // scale sigma is folded into alpha by the previous step)
    double cfac;    // stage coefficient c = tau * cfac of u~ = sigma psi - c kprev
    double dfac;    // d = tau * dfac: tau (Euler) or tau/6 (RK4)
    int turn;       // also form the next stage's transform input (stage boundary kernel)
    int stream_aux; // psi / k (and compensation) loads and stores with evict-first cache hints
    double cnfac;   // next stage: u~' = sigma psi - (tau cnfac) k_s (RK1..RK3); psi1 for RK4/Euler
    // functional
    int fkind;
    int has_g;
    int pot;        // 0 none, 1 harmonic, 2 array
    int nx, ny, nz;
    const Real *varr;
    // constraint
    const V *phase_exp;  // e^{i phi} or null
    // output renormalisation
    int renorm_out;
    // compensated state (complex64 real-time runs): the part of psi below FP32 resolution,
    // BF16 pairs; null = off.  psi1 = psi + (lo - d sum) is formed by a two-sum per lane
    __nv_bfloat162 *comp;
    // complex64: the new state of the last stage (and Euler) is rounded stochastically
    // (gp5cu_stepper_set_stochastic_rounding); ignored where comp is set
    int sround;
};

template <typename Real>
__device__ __forceinline__ Real potential_at(const EpiParams<Real> &P, const SolveParams &S, long long s, int i,
                                             int j, int k, int c) {
    if (P.pot == 1) {
        const double x = position(S, 0, i), y = position(S, 1, j), z = position(S, 2, k);
        const double vx = __dmul_rn(__dmul_rn(S.om2[c][0], x), x);
        const double vy = __dmul_rn(__dmul_rn(S.om2[c][1], y), y);
        const double vz = __dmul_rn(__dmul_rn(S.om2[c][2], z), z);
        return (Real)__dmul_rn(__dadd_rn(__dadd_rn(vx, vy), vz), 0.5);
    }
    return __ldg(P.varr + s + (long long)c * P.nsites);
}

// H applied at one site, components in registers.  u = alpha*u~, kin = alpha*t.
template <typename Real, int NC>
__device__ __forceinline__ void apply_functional(const EpiParams<Real> &P, const SolveParams &S, long long s,
                                                 int i, int j, int k, const cpx<Real> (&u)[NC],
                                                 const cpx<Real> (&kin)[NC], cpx<Real> (&h)[NC], Real (&Vv)[NC],
                                                 Real (&nn)[NC]) {
    using V = cpx<Real>;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        nn[c] = u[c].x * u[c].x + u[c].y * u[c].y;
        Vv[c] = P.pot ? potential_at(P, S, s, i, j, k, c) : (Real)0;
    }
    if (P.fkind == FK_GP) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            V r = kin[c];
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            if (P.has_g) {
                Real f;
                if constexpr (NC == 1) f = (Real)S.g00 * nn[0];
                else f = (c == 0) ? ((Real)S.g00 * nn[0] + (Real)S.g01 * nn[NC - 1])
                                  : ((Real)S.g11 * nn[NC - 1] + (Real)S.g01 * nn[0]);
                r = cadd(r, cscale(u[c], f));
            }
            h[c] = r;
        }
    } else if (NC == 1 || P.fkind == FK_LHY) {
        const Real c3 = (Real)S.c3, c4 = (Real)S.c4;
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const Real f = c3 * nn[c] + c4 * (nn[c] * sqrt(nn[c]));
            V r = cadd(kin[c], cscale(u[c], f));
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            h[c] = r;
        }
    } else if constexpr (NC == 2) {  // unlocked LHY, two components
        const Real la = (Real)S.la, lb = (Real)S.lb, le = (Real)S.le;
        const Real n1 = nn[0], n2 = nn[NC - 1];
        const Real m = n1 + lb * n2;
        const Real p = m * sqrt(m);
        const Real f0 = n1 + le * n2 + la * p;
        const Real f1 = le * lb * n1 + lb * n2 + la * lb * lb * p;
#pragma unroll
        for (int c = 0; c < NC; c++) {
            V r = cadd(kin[c], cscale(u[c], c == 0 ? f0 : f1));
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            h[c] = r;
        }
    }
}

template <typename D, int NC, class EP>
__device__ __forceinline__ double interaction_energy(const EP &P, const SolveParams &S, const D (&nn)[NC]) {
    if (P.fkind == FK_GP) {
        if (!P.has_g) return 0.0;
        if (NC == 1) return 0.5 * S.g00 * (double)nn[0] * (double)nn[0];
        const double a = nn[0], b = nn[NC - 1];
        return 0.5 * S.g00 * a * a + 0.5 * S.g11 * b * b + S.g01 * a * b;
    } else if (P.fkind == FK_LHY) {
        const double n = nn[0];
        return 0.5 * S.c3 * n * n + 0.4 * S.c4 * n * n * sqrt(n);
    }
    const double a = nn[0], b = nn[NC - 1];
    const double m = a + S.lb * b;
    return 0.5 * a * a + 0.5 * S.lb * b * b + S.le * a * b + 0.4 * S.la * m * m * sqrt(m);
}

// Operands of one site's epilogue, loaded before any store of the batch.
template <typename Real> struct EpiIn {
    cpx<Real> psi, kprev, kacc, lo;
};

// store of a psi / k element: evict-first when P.stream_aux
template <typename Real>
__device__ __forceinline__ void aux_store(const EpiParams<Real> &P, cpx<Real> *dst, cpx<Real> v) {
    if (P.stream_aux) __stcs(dst, v);
    else *dst = v;
}

template <typename Real>
__device__ __forceinline__ EpiIn<Real> epi_load(const EpiParams<Real> &P, long long g) {
    EpiIn<Real> in;
    if (P.stream_aux) {
        in.psi = __ldcs(P.psi + g);
        in.kprev = P.mode >= EPI_RK2 ? __ldcs(P.kprev + g) : mk<Real>(0, 0);
        in.kacc = (P.mode == EPI_RK3 || P.mode == EPI_RK4) ? __ldcs(P.kacc + g) : mk<Real>(0, 0);
    } else {
        in.psi = P.psi[g];
        in.kprev = P.mode >= EPI_RK2 ? P.kprev[g] : mk<Real>(0, 0);
        in.kacc = (P.mode == EPI_RK3 || P.mode == EPI_RK4) ? P.kacc[g] : mk<Real>(0, 0);
    }
    if (P.comp && (P.mode == EPI_RK4 || P.mode == EPI_EULER)) {
        const float2 f = __bfloat1622float2(P.stream_aux ? __ldcs(P.comp + g) : P.comp[g]);
        in.lo = mk<Real>((Real)f.x, (Real)f.y);
    } else {
        in.lo = mk<Real>(0, 0);
    }
    return in;
}

// Stochastic rounding of the complex64 state update.  sround_mix is the "lowbias32" integer
// hash (C. Wellons, 2018); sround_hash seeds it with the element index and bits of the element's
// state and increment, so the draw differs between elements and steps, and is reproducible.
__device__ __forceinline__ unsigned sround_mix(unsigned h) {
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ unsigned sround_hash(unsigned g, unsigned a, unsigned b) {
    return sround_mix(g * 0x9e3779b1u ^ a ^ ((b << 7) | (b >> 25)));
}
// r = round-to-nearest(x), lo = x - r exactly; returns r or the float next to r on lo's side,
// the latter with probability |lo| / (its distance from r), drawn from the top 24 bits of h:
// the expectation is x.
__device__ __forceinline__ float sround(float r, float lo, unsigned h) {
    if (lo == 0.f || r == 0.f || !isfinite(r)) return r;
    const int b = __float_as_int(r);
    const float rn = __int_as_float(((lo > 0.f) == (r > 0.f)) ? b + 1 : b - 1);
    const float u = (float)(h >> 8) * 5.9604644775390625e-8f;  // [0, 1) in steps of 2^-24
    return u * fabsf(rn - r) < fabsf(lo) ? rn : r;
}

// Stage constants of the epilogue in the plan precision: c0 = tau cfac (u~_s = sigma psi0 -
// c0 k_{s-1}), cn = tau cnfac (u~_{s+1}), d = tau dfac (psi1 = p - d sum).  The stage boundary
// forms them once per tile (its element loop would otherwise repeat the FP64 products, since
// the compiler cannot keep the shared-memory context in registers across the loop's shared
// stores); the other callers form them per site.
template <typename Real> struct StageK {
    cpx<Real> c0, cn, d;
};
template <typename Real>
__device__ __forceinline__ StageK<Real> stage_k(const EpiParams<Real> &P, const SolveParams &S) {
    StageK<Real> K;
    K.c0.x = (Real)(S.tre * P.cfac);
    K.c0.y = (Real)(S.tim * P.cfac);
    K.cn.x = (Real)(S.tre * P.cnfac);
    K.cn.y = (Real)(S.tim * P.cnfac);
    K.d.x = (Real)(S.tre * P.dfac);
    K.d.y = (Real)(S.tim * P.dfac);
    return K;
}

// The epilogue of one site: t[c] = kinetic of u~_c (already times K^2/(2 m N^3)).
// With P.turn the epilogue also returns, in next[c], the input of the following transform:
// u~_{s+1} = sigma psi - cn k_s after stages 1-3, or the new state psi1 after the last stage
// (and Euler); with RED it accumulates |next|^2 for the following normalisation.
template <typename Real, int NC, bool RED, bool TURN = false>
__device__ __forceinline__ void epilogue_site(const EpiParams<Real> &P, const SolveCtx &X, long long s, int i,
                                              int j, int k, const cpx<Real> (&t)[NC], const EpiIn<Real> (&in)[NC],
                                              double *acc, cpx<Real> (&next)[NC], const StageK<Real> &K) {
    using V = cpx<Real>;
    const SolveParams &S = X.S;
    V p[NC], u[NC], kin[NC], h[NC];
    Real Vv[NC], nn[NC];
    const int mode = P.mode;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const V raw = in[c].psi;
        V x = raw;
        if (P.use_sigma) x = cscale(x, (Real)X.sigma[c]);
        p[c] = x;
        V ut = P.u1_raw ? raw : x;
        if (mode >= EPI_RK2) ut = csub(x, cmul(K.c0, in[c].kprev));
        if (P.use_alpha) {
            const Real a = (Real)X.alpha[P.slot][c];
            u[c] = cscale(ut, a);
            kin[c] = cscale(t[c], a);
        } else {
            u[c] = ut;
            kin[c] = t[c];
        }
    }
    apply_functional<Real, NC>(P, S, s, i, j, k, u, kin, h, Vv, nn);

    if (!TURN && (mode == EPI_H || mode == EPI_OBS)) {
#pragma unroll
        for (int c = 0; c < NC; c++) P.kout[s + (long long)c * P.nsites] = h[c];
        // (compiled only where the caller provides all eight sums: the stage boundary has two)
        if constexpr (RED && !TURN) if (mode == EPI_OBS) {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                const double ur = u[c].x, ui = u[c].y;
                acc[0] += ur * ur + ui * ui;
                acc[1] += ur * (double)kin[c].x + ui * (double)kin[c].y;
                acc[2] += (double)Vv[c] * (ur * ur + ui * ui);
                acc[4] += ur * (double)h[c].x + ui * (double)h[c].y;
            }
            if constexpr (sizeof(Real) == 8) {
                acc[3] += interaction_energy<Real, NC>(P, S, nn);
            } else {
                // complex64: the densities of the energy sum are formed in FP64
                double nd[NC];
#pragma unroll
                for (int c = 0; c < NC; c++) nd[c] = (double)u[c].x * u[c].x + (double)u[c].y * u[c].y;
                acc[3] += interaction_energy<double, NC>(P, S, nd);
            }
        }
        return;
    }
    if (mode == EPI_RK1 || mode == EPI_RK2 || mode == EPI_RK3) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const long long g = s + (long long)c * P.nsites;
            if (mode == EPI_RK1) {
                aux_store(P, P.kout + g, h[c]);
            } else if (mode == EPI_RK2) {
                aux_store(P, P.kout + g, h[c]);
                aux_store(P, P.kacc + g, cadd(in[c].kprev, cscale(h[c], (Real)2)));
            } else {
                aux_store(P, P.kacc + g, cadd(in[c].kacc, cscale(h[c], (Real)2)));
                aux_store(P, P.kout + g, h[c]);
            }
            if (TURN) {
                const V nx = csub(p[c], cmul(K.cn, h[c]));
                next[c] = nx;
                if (RED) acc[c] += (double)nx.x * (double)nx.x + (double)nx.y * (double)nx.y;
            }
        }
        return;
    }
    // EULER / RK4: psi1 = p - d * (sum)
    const V d = K.d;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const long long g = s + (long long)c * P.nsites;
        V sum = h[c];
        if (mode == EPI_RK4) sum = cadd(in[c].kacc, h[c]);
        V r;
        if (P.comp) {
            // two-sum per lane: r + lo' = p + (lo - d sum) exactly when |p| >= |lo - d sum|
            const V delta = csub(in[c].lo, cmul(d, sum));
            r = cadd(p[c], delta);
            V lo;
            lo.x = (p[c].x - r.x) + delta.x;
            lo.y = (p[c].y - r.y) + delta.y;
            const __nv_bfloat162 lo2 = __floats2bfloat162_rn((float)lo.x, (float)lo.y);
            if (P.stream_aux) __stcs(P.comp + g, lo2);
            else P.comp[g] = lo2;
        } else if (sizeof(Real) == 4 && P.sround) {
            // unbiased (stochastic) rounding of p - d sum: the exact error lo of the rounded sum
            // decides, with probability |lo| / spacing, whether the neighbouring float replaces r
            const V delta = csub(mk<Real>(0, 0), cmul(d, sum));
            r = cadd(p[c], delta);
            const float lox = ((float)p[c].x - (float)r.x) + (float)delta.x;
            const float loy = ((float)p[c].y - (float)r.y) + (float)delta.y;
            // seeded by the element's index within its solve, so that a batched solve rounds as it
            // does alone
            const unsigned site = (unsigned)(i + P.nx * (j + P.ny * k)) + (unsigned)c * (unsigned)P.nsites;
            const unsigned h = sround_hash(site, __float_as_uint((float)p[c].x), __float_as_uint((float)delta.y));
            r.x = (Real)sround((float)r.x, lox, h);
            r.y = (Real)sround((float)r.y, loy, sround_mix(h ^ __float_as_uint((float)p[c].y)));
        } else {
            r = csub(p[c], cmul(d, sum));
        }
        if (P.phase_exp) {
            const Real a = sqrt(r.x * r.x + r.y * r.y);
            r = cscale(P.phase_exp[g], a);
        }
        aux_store(P, P.psi_out + g, r);
        if (TURN) next[c] = r;
        if (RED && P.renorm_out) acc[c] += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    }
}

template <typename Real> struct EpiFinalize {
    // OBS: keep the raw sums; mu for the residual.  RK4/EULER with renorm: new sigma.
    static __device__ __forceinline__ void run(const EpiParams<Real> &P, const double *s, int solve) {
        DevScalars *ds = P.ds + solve;
        const SolveParams &S = P.sp[solve];
        if (P.mode == EPI_OBS) {
            for (int r = 0; r < 8; r++) ds->sums[r] = s[r];
            ds->mu = s[4] / s[0];
            if (!isfinite(s[0]) || !isfinite(s[4])) ds->status |= DS_NONFINITE;
        } else if ((P.mode == EPI_EULER || P.mode == EPI_RK4) && P.renorm_out) {
            ds->sigma[0] = sqrt(S.Nt[0] / (S.dV * s[0]));
            ds->sigma[1] = (S.Nt[1] > 0) ? sqrt(S.Nt[1] / (S.dV * s[1])) : 1.0;
            if (P.turn) {
                // the next step transforms the raw state: its first stage scales by sigma
                ds->alpha[1][0] = ds->sigma[0];
                ds->alpha[1][1] = ds->sigma[1];
            }
            if (!isfinite(s[0]) || !isfinite(ds->sigma[0])) ds->status |= DS_NONFINITE;
        } else if (P.turn && P.renorm_out) {
            // normalisation of the next stage's input u~_{s+1} (slot of stage s+1)
            const int ns = P.slot ^ 1;
            ds->alpha[ns][0] = sqrt(S.Nt[0] / (S.dV * s[0]));
            ds->alpha[ns][1] = (S.Nt[1] > 0) ? sqrt(S.Nt[1] / (S.dV * s[1])) : 1.0;
            if (!isfinite(s[0]) || !isfinite(ds->alpha[ns][0])) ds->status |= DS_NONFINITE;
        }
    }
};

// Fused epilogue (one component): the inverse x pass hands every element to the site logic.
// TURN (stage boundary, mode inverse -> turn -> forward): turn() runs the epilogue of stage s
// and returns the next stage's transform input; post() stores the forward transform into src.
// BATCH = 4: the epilogue issues the psi / k loads of four elements together (the boundary
// waits on memory; 4 measured 8% faster than 2 at 256^3, 8 spills).
template <typename Real, bool RED, bool TURN = false> struct OpStageOut {
    // the stage boundary only reduces |next|^2 per component (two sums); the observables
    // epilogue needs all eight
    static constexpr int NRED = RED ? (TURN ? 2 : kNRed) : 0, BATCH = 4;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = EpiIn<Real>;
    const V *src;  // inverse-pass input buffer (the boundary kernel writes it back in place)
    EpiParams<Real> P;
    __device__ __forceinline__ const SolveParams *params() const { return P.sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return P.ds; }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &, const SolveCtx &) const { return v; }
    __device__ __forceinline__ Pre pre(long long g) const { return epi_load(P, g); }
    __device__ __forceinline__ StageK<Real> consts(const SolveCtx &X) const { return stage_k(P, X.S); }
    __device__ __forceinline__ V turn(long long g, const LineRef &e, V v, const Pre &in, double *acc,
                                      const SolveCtx &X, const StageK<Real> &K) const {
        const V t[1] = {v};
        const Pre ins[1] = {in};
        V nx[1] = {v};
        epilogue_site<Real, 1, RED, true>(P, X, g, e.i, e.j, e.k, t, ins, acc, nx, K);
        return nx[0];
    }
    __device__ __forceinline__ void post(long long g, const LineRef &e, V v, const Pre &in, double *acc,
                                         const SolveCtx &X) const {
        if (TURN) {
            const_cast<V *>(src)[g] = v;
        } else {
            const V t[1] = {v};
            const Pre ins[1] = {in};
            V nx[1];
            epilogue_site<Real, 1, RED>(P, X, g, e.i, e.j, e.k, t, ins, acc, nx, stage_k(P, X.S));
        }
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        int n = 0;
        p[n++] = src;
        p[n++] = P.psi;
        if (P.mode >= EPI_RK2) p[n++] = P.kprev;
        if (P.mode == EPI_RK3 || P.mode == EPI_RK4) p[n++] = P.kacc;
        return n;
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const { EpiFinalize<Real>::run(P, s, solve); }
};

#ifndef GP5_AXES_BATCH
#define GP5_AXES_BATCH 2
#endif
// Stage boundary of the per-axis scheme (one component, x lines): forms the stage input
// u~_s = sigma psi0 - c_s k_{s-1} (or the raw state in the first stage) from psi and k_{s-1},
// its x term of the kinetic operator IFFT_x(kx^2/(2 m Nx) FFT_x u~), adds the y and z terms the
// strided passes left in T, and runs the stage epilogue: k_s, the RK bookkeeping, and the next
// stage's input u~_{s+1} stored in real space to unext (the last stage stores psi1 instead,
// unext null).  The operands of u~ are read twice (before the transform and in the epilogue);
// the second read finds the tile's lines in L2.
template <typename Real, bool RED> struct OpStageAxes {
    static constexpr int NRED = RED ? kNRed : 0, BATCH = GP5_AXES_BATCH;
    static constexpr bool HEAVY_EPILOGUE = true;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    struct Pre {
        EpiIn<Real> in;
        V t;
    };
    EpiParams<Real> P;
    const V *tsum;  // y and z kinetic terms of u~_s
    V *unext;       // u~_{s+1} (real space), or null after the last stage
    int nx, ny, nz;
    __device__ __forceinline__ const SolveParams *params() const { return P.sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return P.ds; }
    // u~_s from the psi element (src0) and k_{s-1}: the expressions of epilogue_site
    __device__ __forceinline__ V load(V raw, long long g, const LineRef &e, double *, const SolveCtx &X) const {
        if (P.u1_raw) return raw;
        V x = raw;
        if (P.use_sigma) x = cscale(x, (Real)X.sigma[e.c]);
        if (P.mode >= EPI_RK2) {
            V c0;
            c0.x = (Real)(X.S.tre * P.cfac);
            c0.y = (Real)(X.S.tim * P.cfac);
            return csub(x, cmul(c0, P.kprev[g]));  // a normal load: the epilogue reads it again
        }
        return x;
    }
    __device__ __forceinline__ V mid(V v, const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const double k = momentum(S, 0, e.i, nx);
        return cscale(v, (Real)(__dmul_rn(k, k) * __dmul_rn(S.kin[e.c], (double)ny * nz)));
    }
    __device__ __forceinline__ Pre pre(long long g) const {
        Pre p;
        p.in = epi_load(P, g);
        p.t = tsum[g];
        return p;
    }
    __device__ __forceinline__ void post(long long g, const LineRef &e, V v, const Pre &in, double *acc,
                                         const SolveCtx &X) const {
        const V t[1] = {cadd(v, in.t)};
        const EpiIn<Real> ins[1] = {in.in};
        V nx_[1];
        epilogue_site<Real, 1, RED, true>(P, X, g, e.i, e.j, e.k, t, ins, acc, nx_, stage_k(P, X.S));
        if (unext) unext[g] = nx_[0];
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        int n = 0;
        p[n++] = P.psi;
        if (P.mode >= EPI_RK2) p[n++] = P.kprev;
        p[n++] = tsum;
        if (P.mode == EPI_RK3 || P.mode == EPI_RK4) p[n++] = P.kacc;
        return n;
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const { EpiFinalize<Real>::run(P, s, solve); }
};

// ---- point-wise ops (site(solve, s, acc) for s in [0, nsites) of one solve) --------------
// Non-fused epilogue over sites (two components): t from the kinetic buffer.
template <typename Real, int NC, bool RED> struct OpSiteEpilogue {
    static constexpr int NRED = RED ? kNRed : 0;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    EpiParams<Real> P;
    long long stride;  // elements between solves
    __device__ __forceinline__ const SolveParams *params() const { return P.sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return P.ds; }
    __device__ __forceinline__ void site(int solve, long long s, double *acc, const SolveCtx &X) const {
        const long long g0 = (long long)solve * stride + s;
        V t[NC];
        EpiIn<Real> in[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            t[c] = P.tsrc[g0 + (long long)c * P.nsites];
            in[c] = epi_load(P, g0 + (long long)c * P.nsites);
        }
        const int i = (int)(s % P.nx);
        const long long r = s / P.nx;
        const int j = (int)(r % P.ny), k = (int)(r / P.ny);
        V nx[NC];
        epilogue_site<Real, NC, RED>(P, X, g0, i, j, k, t, in, acc, nx, stage_k(P, X.S));
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const { EpiFinalize<Real>::run(P, s, solve); }
};

// sum |psi_c|^2 over one component (or all when comp < 0); result in ds->sums[0], factor for
// normalize = sqrt(N / (dV S)).
template <typename Real> struct OpNorm {
    static constexpr int NRED = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    const V *f;
    long long nsites, stride;
    int comp, ncomp;
    DevScalars *ds;
    double Ntarget, dV;
    __device__ __forceinline__ const SolveParams *params() const { return nullptr; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ void site(int solve, long long s, double *acc, const SolveCtx &) const {
        const V *fs = f + (long long)solve * stride;
        if (comp >= 0) {
            const V v = fs[s + (long long)comp * nsites];
            acc[0] += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
        } else {
            for (int c = 0; c < ncomp; c++) {
                const V v = fs[s + (long long)c * nsites];
                acc[0] += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
            }
        }
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const {
        DevScalars &d = ds[solve];
        d.sums[0] = s[0];
        d.factor = Ntarget > 0 ? sqrt(Ntarget / (dV * s[0])) : 1.0;
        if (!isfinite(s[0])) d.status |= DS_NONFINITE;
    }
};

// psi_c *= factor (device scalar); comp < 0 scales every component by sigma[c].
template <typename Real> struct OpScale {
    static constexpr int NRED = 0;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    V *f;
    long long nsites, stride;
    int comp, ncomp;
    DevScalars *ds;
    int from_sigma;
    __device__ __forceinline__ const SolveParams *params() const { return nullptr; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ void site(int solve, long long s, double *, const SolveCtx &) const {
        V *fs = f + (long long)solve * stride;
        const DevScalars &d = ds[solve];
        if (!from_sigma) {
            const Real a = (Real)d.factor;
            const long long g = s + (long long)comp * nsites;
            fs[g] = cscale(fs[g], a);
        } else {
            for (int c = 0; c < ncomp; c++) {
                const long long g = s + (long long)c * nsites;
                fs[g] = cscale(fs[g], (Real)d.sigma[c]);
            }
        }
    }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

// residual: sum |H psi - mu psi|^2
template <typename Real> struct OpResidual {
    static constexpr int NRED = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    const V *psi, *hpsi;
    long long nsites, stride;
    int ncomp;
    DevScalars *ds;
    const SolveParams *sp;  // may be null
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ void site(int solve, long long s, double *acc, const SolveCtx &) const {
        const double mu = __ldg(&ds[solve].mu);
        for (int c = 0; c < ncomp; c++) {
            const long long g = (long long)solve * stride + s + (long long)c * nsites;
            const V a = psi[g], h = hpsi[g];
            const double rx = (double)h.x - mu * (double)a.x, ry = (double)h.y - mu * (double)a.y;
            acc[0] += rx * rx + ry * ry;
        }
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const { ds[solve].sums[5] = s[0]; }
};

// ---- preconditioned ground-state iteration ---------------------------------------------------
// One iteration of every solve (single component):
//   r = H psi - mu psi,  d = (alpha - 1/2m lap)^{-1} r,  psi <- (psi - theta d) normalised to N,
// with mu = <psi|H psi>/<psi|psi> of the current state (ds[solve].mu, written by the observables
// epilogue of the H application) and alpha = max(|mu|, kPrecondAlphaMin, kPrecondVShare Vmax)
// per solve, Vmax the harmonic potential at the farthest cell centre (the preconditioner does
// not see V: theta (V - mu) / alpha must stay below 2 where V is large).  The inverse
// of the kinetic operator shifted by alpha is applied in k-space, between a forward and an
// inverse transform, so every Fourier mode of the residual moves at a rate of order one: the
// iteration needs tens of passes where imaginary time needs thousands of steps, and its fixed
// point (r = 0 at norm N) is the state imaginary-time evolution converges to.
constexpr double kPrecondAlphaMin = 0.05, kPrecondVShare = 0.5;

// x forward pass: the transform input is the residual H psi - mu psi
template <typename Real> struct OpPrecondIn {
    static constexpr int NRED = 0, BATCH = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *hpsi, *psi;
    V *dst;
    const DevScalars *ds;
    const SolveParams *sp;
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ V load(V h, long long g, const LineRef &e, double *, const SolveCtx &) const {
        const Real mu = (Real)__ldg(&ds[e.solve].mu);
        return csub(h, cscale(psi[g], mu));
    }
    __device__ __forceinline__ V mid(V v, const LineRef &, const SolveCtx &) const { return v; }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *, const SolveCtx &) const {
        dst[g] = v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        p[0] = hpsi;
        p[1] = psi;
        return 2;
    }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

// z pass: forward z, times 1 / (ns (alpha + kin ns K^2)), inverse z.  kin = 1/(2 m ns) is the
// plan's kinetic multiplier, so kin ns K^2 = K^2 / 2m, and the 1/ns is the normalisation of
// the unnormalised inverse transform.  The factor is formed in FP64 in both precisions.
template <typename Real> struct OpPrecond {
    static constexpr int NRED = 0, BATCH = 1;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *src;
    V *dst;
    const SolveParams *sp;
    const DevScalars *ds;
    int nx, ny, nz;
    double ns;  // sites per solve
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ double alpha(int solve, const SolveParams &S) const {
        const int n[3] = {nx, ny, nz};
        double vmax = 0.0;
        for (int d = 0; d < 3; d++) {
            const double lo = S.left[d] + 0.5 * S.dx[d], hi = S.left[d] + (n[d] - 0.5) * S.dx[d];
            vmax += S.om2[0][d] * fmax(lo * lo, hi * hi);
        }
        return fmax(fmax(fabs(__ldg(&ds[solve].mu)), kPrecondAlphaMin), kPrecondVShare * 0.5 * vmax);
    }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const double kx = momentum(S, 0, e.i, nx), ky = momentum(S, 1, e.j, ny), kz = momentum(S, 2, e.k, nz);
        const double k2 = (kx * kx + ky * ky) + kz * kz;
        return cscale(v, (Real)(1.0 / (ns * alpha(e.solve, S) + S.kin[e.c] * ns * ns * k2)));
    }
    static constexpr bool MID_Z = true;
    struct MidLine {
        double kxy2, dkz, a, b;
    };
    __device__ __forceinline__ MidLine mid_line(const LineRef &e, const SolveCtx &X) const {
        const SolveParams &S = X.S;
        const double kx = momentum(S, 0, e.i, nx), ky = momentum(S, 1, e.j, ny);
        return MidLine{kx * kx + ky * ky, S.dk[2], ns * alpha(e.solve, S), S.kin[e.c] * ns * ns};
    }
    __device__ __forceinline__ V mid_z(V v, int kidx, const MidLine &L) const {
        const double kz = L.dkz * (double)kidx;
        return cscale(v, (Real)(1.0 / (L.a + L.b * (L.kxy2 + kz * kz))));
    }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *, const SolveCtx &) const {
        dst[g] = v;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const { p[0] = src; return 1; }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

// x inverse pass: psi <- psi - theta d, with sum |psi|^2 per solve -> the normalisation factor
// sqrt(N / (dV S)) in ds[solve].factor (applied by an OpScale pass)
template <typename Real> struct OpPrecondOut {
    static constexpr int NRED = 1, BATCH = 4;
    using Ctx = SolveCtx;
    using V = cpx<Real>;
    struct Pre {
        V p;
    };
    const V *src;  // transform buffer
    V *psi;
    DevScalars *ds;
    const SolveParams *sp;  // targets N and cell volumes
    double theta;
    __device__ __forceinline__ const SolveParams *params() const { return sp; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ V load(V x, long long, const LineRef &, double *, const SolveCtx &) const { return x; }
    __device__ __forceinline__ V mid(V v, const LineRef &, const SolveCtx &) const { return v; }
    __device__ __forceinline__ Pre pre(long long g) const { return Pre{psi[g]}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &q, double *acc,
                                         const SolveCtx &) const {
        const V r = csub(q.p, cscale(v, (Real)theta));
        psi[g] = r;
        acc[0] += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        p[0] = src;
        p[1] = psi;
        return 2;
    }
    __device__ __forceinline__ void finalize(const double *s, int solve) const {
        const SolveParams &S = sp[solve];
        DevScalars &d = ds[solve];
        d.factor = sqrt(S.Nt[0] / (S.dV * s[0]));
        if (!isfinite(s[0]) || !isfinite(d.factor)) d.status |= DS_NONFINITE;
    }
};

// complex128 <-> plan precision conversion over nsites elements (one solve)
template <typename Real> struct OpConvert {
    static constexpr int NRED = 0;
    using Ctx = SolveCtx;
    const double2 *in128;
    cpx<Real> *out;
    const cpx<Real> *in;
    double2 *out128;
    __device__ __forceinline__ const SolveParams *params() const { return nullptr; }
    __device__ __forceinline__ const DevScalars *scalars() const { return nullptr; }
    __device__ __forceinline__ void site(int, long long s, double *, const SolveCtx &) const {
        if (in128) {
            const double2 v = in128[s];
            out[s] = mk<Real>((Real)v.x, (Real)v.y);
        } else {
            const cpx<Real> v = in[s];
            out128[s] = make_double2((double)v.x, (double)v.y);
        }
    }
    __device__ __forceinline__ void finalize(const double *, int) const {}
};

}  // namespace gp5

// ops.cuh - the point-wise arithmetic of the GP hot path, written as hooks that the axis
// passes call on every element they load, transform or store.
//
// Reference arithmetic restated here (lucaparisi91/GP5):
//   kinetic       operators.cpp:28-36 (IFFT(-K^2 FFT)/N^3) with functional.cpp:24 / :118
//                 (-1/2, 1/m): one multiplier (1/2 K^2 / m / N^3) in k-space
//   potential     functional.cpp:46-53; harmonic V = (wx^2 x^2 + wy^2 y^2 + wz^2 z^2)/2,
//                 externalPotential.cpp:26
//   interaction   GP 1 comp functional.cpp:54-68; 2 comp :71-89; LHY :112-119 (n^{3/2}
//                 evaluated as n*sqrt(n)); unlocked LHY :125-150
//   RK4 stages    stepper.cpp:46-71;  Euler stepper.cpp:30-44
//   normalize     geometry.cpp:190-229 (applied lazily as a device-side scale)
//   phase constr. constraint.cpp:6-9
#pragma once

#include "passes.cuh"

namespace gp5 {

constexpr int kNRed = 8;

// ---- device scalars shared by the kernels of one stepper / plan -------------------------
struct DevScalars {
    double sigma[2];   // pending scale of the state (1 when clean)
    double alpha[2][2];  // [stage & 1][component]: scale of the stage's transform input
    double sums[8];    // last reduction result (raw sums, not yet times dV)
    double mu;         // chemical potential for the residual pass
    double factor;     // scale factor for normalize
    unsigned status;   // DevStatus bits
    unsigned pad;
};

// ---- plain copy / kinetic-multiply ops --------------------------------------------------
// Hook interface of the axis passes:
//   load(g, e, acc)          value entering the transform at element g (prologue)
//   mid(v, e)                k-space multiply between a forward and an inverse transform
//   pre(g) -> Pre            operand loads of the epilogue (issued BATCH elements at a time)
//   post(g, e, v, pre, acc)  epilogue: consume the transformed value and store
//   streams(p)               arrays the pass reads, for the L2 prefetch of the next tile
//   finalize(sums)           last block, with the FP64 sums of the NRED accumulators
struct NoPre {};

template <typename Real> struct OpCopy {
    static constexpr int NRED = 0, BATCH = 1;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *src;
    V *dst;
    __device__ __forceinline__ V load(long long g, const LineRef &, double *) const { return src[g]; }
    __device__ __forceinline__ V mid(V v, const LineRef &) const { return v; }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *) const { dst[g] = v; }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const { p[0] = src; return 1; }
    __device__ __forceinline__ void finalize(const double *) const {}
};

// z pass of an H application: forward z, times (K^2 * coef_c), inverse z.
template <typename Real> struct OpKinetic {
    static constexpr int NRED = 0, BATCH = 1;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *src;
    V *dst;
    const double *kx2, *ky2, *kz2;  // k_d^2 tables
    double coef0, coef1;            // per component: 1/(2 m N^3) for H, -1/N^3 for the Laplacian
    int nz;                         // k_z is formed arithmetically (same value as the table):
    double dkz;                     // k = dkz * m, m = k < nz/2 (even) or k <= (nz-1)/2 (odd), else k - nz
    __device__ __forceinline__ V load(long long g, const LineRef &, double *) const { return src[g]; }
    __device__ __forceinline__ V mid(V v, const LineRef &e) const {
        const int half = (nz % 2 == 0) ? nz / 2 : (nz - 1) / 2 + 1;
        const double kz = e.k < half ? dkz * e.k : (-nz + e.k) * dkz;
        const double k2 = (__ldg(kx2 + e.i) + __ldg(ky2 + e.j)) + kz * kz;
        const Real f = (Real)(k2 * (e.c ? coef1 : coef0));
        return cscale(v, f);
    }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *) const { dst[g] = v; }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const { p[0] = src; return 1; }
    __device__ __forceinline__ void finalize(const double *) const {}
};

// ---- stage input (prologue of the first forward pass) -----------------------------------
// u~ = sigma_c psi - c kprev ; optional sum |u~|^2 per component -> alpha_c = sqrt(N_c/(dV S)).
template <typename Real, bool RED> struct OpStageIn {
    static constexpr int NRED = RED ? 2 : 0, BATCH = 1;
    using V = cpx<Real>;
    using Pre = NoPre;
    const V *psi;
    const V *kprev;  // null for the first stage
    V *dst;
    DevScalars *ds;
    int use_sigma;
    Real cre, cim;
    double Nt0, Nt1, dV;
    int slot;  // alpha slot (stage & 1) written by finalize
    __device__ __forceinline__ V load(long long g, const LineRef &e, double *acc) const {
        V p = psi[g];
        if (use_sigma) p = cscale(p, (Real)__ldg(&ds->sigma[e.c]));
        if (kprev) {
            V kk = kprev[g];
            V c;
            c.x = cre;
            c.y = cim;
            p = csub(p, cmul(c, kk));
        }
        if (RED) {
            const double n = (double)p.x * (double)p.x + (double)p.y * (double)p.y;
            if (e.c == 0) acc[0] += n;
            else acc[1] += n;
        }
        return p;
    }
    __device__ __forceinline__ V mid(V v, const LineRef &) const { return v; }
    __device__ __forceinline__ Pre pre(long long) const { return Pre{}; }
    __device__ __forceinline__ void post(long long g, const LineRef &, V v, const Pre &, double *) const { dst[g] = v; }
    __device__ __forceinline__ int streams(const void *(&p)[4]) const {
        p[0] = psi;
        if (kprev) { p[1] = kprev; return 2; }
        return 1;
    }
    __device__ __forceinline__ void finalize(const double *s) const {
        if (RED) {
            ds->alpha[slot][0] = sqrt(Nt0 / (dV * s[0]));
            ds->alpha[slot][1] = (Nt1 > 0) ? sqrt(Nt1 / (dV * s[1])) : 1.0;
            if (!isfinite(s[0]) || !isfinite(s[1]) || !isfinite(ds->alpha[slot][0])) ds->status |= DS_NONFINITE;
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
    long long nsites;
    int mode;
    // state
    const V *psi;  // stage base psi0 (read); EPI_H/OBS: the source field
    V *psi_out;    // EULER / RK4 result (may alias psi)
    const V *kprev;
    V *kout;       // k_s (RK1 -> Ka, RK2 -> Kb, RK3 -> Kb) or H src (H/OBS)
    V *kacc;       // Ka: RK accumulator (RK2/RK3/RK4)
    const V *tsrc; // kinetic buffer for the non-fused (2 component) epilogue
    DevScalars *ds;
    int use_sigma, use_alpha;
    int slot;       // alpha slot of this stage (stage & 1)
    int u1_raw;     // first stage / Euler: the transform input was the raw state (its pending
                    // scale sigma is folded into alpha by the previous step)
    Real cre, cim;  // stage coefficient of u~ = sigma psi - c kprev
    Real dre, dim;  // tau (Euler) or tau/6 (RK4)
    int turn;       // also form the next stage's transform input (stage boundary kernel)
    Real cnre, cnim;  // next stage: u~' = sigma psi - cn k_s (RK1..RK3); psi1 for RK4/Euler
    // functional
    int fkind;
    int has_g;
    Real g00, g01, g11;
    Real c3, c4;
    Real la, lb, le;  // unlocked alpha, beta, eta
    int pot;          // 0 none, 1 harmonic, 2 array
    const double *hx, *hy, *hz;  // harmonic: w_d^2 x_d^2 tables [ncomp][n_d]
    int nx, ny, nz;
    const Real *varr;
    // constraint
    const V *phase_exp;  // e^{i phi} or null
    // output renormalisation
    int renorm_out;
    double Nt0, Nt1, dV;
};

template <typename Real>
__device__ __forceinline__ Real potential_at(const EpiParams<Real> &P, long long s, int i, int j, int k, int c) {
    if (P.pot == 1) {
        const double v = ((__ldg(P.hx + c * P.nx + i) + __ldg(P.hy + c * P.ny + j)) + __ldg(P.hz + c * P.nz + k)) * 0.5;
        return (Real)v;
    }
    return __ldg(P.varr + s + (long long)c * P.nsites);
}

// H applied at one site, components in registers.  u = alpha*u~, kin = alpha*t.
template <typename Real, int NC>
__device__ __forceinline__ void apply_functional(const EpiParams<Real> &P, long long s, int i, int j, int k,
                                                 const cpx<Real> (&u)[NC], const cpx<Real> (&kin)[NC],
                                                 cpx<Real> (&h)[NC], Real (&Vv)[NC], Real (&nn)[NC]) {
    using V = cpx<Real>;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        nn[c] = u[c].x * u[c].x + u[c].y * u[c].y;
        Vv[c] = P.pot ? potential_at(P, s, i, j, k, c) : (Real)0;
    }
    if (P.fkind == FK_GP) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            V r = kin[c];
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            if (P.has_g) {
                Real f;
                if (NC == 1) f = P.g00 * nn[0];
                else f = (c == 0) ? (P.g00 * nn[0] + P.g01 * nn[NC - 1]) : (P.g11 * nn[NC - 1] + P.g01 * nn[0]);
                r = cadd(r, cscale(u[c], f));
            }
            h[c] = r;
        }
    } else if (P.fkind == FK_LHY) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const Real f = P.c3 * nn[c] + P.c4 * (nn[c] * sqrt(nn[c]));
            V r = cadd(kin[c], cscale(u[c], f));
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            h[c] = r;
        }
    } else {  // unlocked LHY, two components
        const Real n1 = nn[0], n2 = nn[NC - 1];
        const Real m = n1 + P.lb * n2;
        const Real p = m * sqrt(m);
        const Real f0 = n1 + P.le * n2 + P.la * p;
        const Real f1 = P.le * P.lb * n1 + P.lb * n2 + P.la * P.lb * P.lb * p;
#pragma unroll
        for (int c = 0; c < NC; c++) {
            V r = cadd(kin[c], cscale(u[c], c == 0 ? f0 : f1));
            if (P.pot) r = cadd(r, cscale(u[c], Vv[c]));
            h[c] = r;
        }
    }
}

template <typename Real, int NC>
__device__ __forceinline__ double interaction_energy(const EpiParams<Real> &P, const Real (&nn)[NC]) {
    if (P.fkind == FK_GP) {
        if (!P.has_g) return 0.0;
        if (NC == 1) return 0.5 * (double)P.g00 * (double)nn[0] * (double)nn[0];
        const double a = nn[0], b = nn[NC - 1];
        return 0.5 * (double)P.g00 * a * a + 0.5 * (double)P.g11 * b * b + (double)P.g01 * a * b;
    } else if (P.fkind == FK_LHY) {
        const double n = nn[0];
        return 0.5 * (double)P.c3 * n * n + 0.4 * (double)P.c4 * n * n * sqrt(n);
    }
    const double a = nn[0], b = nn[NC - 1];
    const double m = a + (double)P.lb * b;
    return 0.5 * a * a + 0.5 * (double)P.lb * b * b + (double)P.le * a * b + 0.4 * (double)P.la * m * m * sqrt(m);
}

// The epilogue of one site: t[c] = kinetic of u~_c (already times 1/(2 m N^3) K^2).
// Operands of one site's epilogue, loaded before any store of the batch.
template <typename Real> struct EpiIn {
    cpx<Real> psi, kprev, kacc;
};

template <typename Real>
__device__ __forceinline__ EpiIn<Real> epi_load(const EpiParams<Real> &P, long long g) {
    EpiIn<Real> in;
    in.psi = P.psi[g];
    in.kprev = P.mode >= EPI_RK2 ? P.kprev[g] : mk<Real>(0, 0);
    in.kacc = (P.mode == EPI_RK3 || P.mode == EPI_RK4) ? P.kacc[g] : mk<Real>(0, 0);
    return in;
}

// With P.turn the epilogue also returns, in next[c], the input of the following transform:
// u~_{s+1} = sigma psi - cn k_s after stages 1-3, or the new state psi1 after the last stage
// (and Euler); with RED it accumulates |next|^2 for the following normalisation.
template <typename Real, int NC, bool RED>
__device__ __forceinline__ void epilogue_site(const EpiParams<Real> &P, long long s, int i, int j, int k,
                                              const cpx<Real> (&t)[NC], const EpiIn<Real> (&in)[NC],
                                              double *acc, cpx<Real> (&next)[NC]) {
    using V = cpx<Real>;
    V p[NC], u[NC], kin[NC], h[NC];
    Real Vv[NC], nn[NC];
    const int mode = P.mode;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const V raw = in[c].psi;
        V x = raw;
        if (P.use_sigma) x = cscale(x, (Real)__ldg(&P.ds->sigma[c]));
        p[c] = x;
        V ut = P.u1_raw ? raw : x;
        if (mode >= EPI_RK2) {
            V c0;
            c0.x = P.cre;
            c0.y = P.cim;
            ut = csub(x, cmul(c0, in[c].kprev));
        }
        if (P.use_alpha) {
            const Real a = (Real)__ldg(&P.ds->alpha[P.slot][c]);
            u[c] = cscale(ut, a);
            kin[c] = cscale(t[c], a);
        } else {
            u[c] = ut;
            kin[c] = t[c];
        }
    }
    apply_functional<Real, NC>(P, s, i, j, k, u, kin, h, Vv, nn);

    if (mode == EPI_H || mode == EPI_OBS) {
#pragma unroll
        for (int c = 0; c < NC; c++) P.kout[s + (long long)c * P.nsites] = h[c];
        if (RED && mode == EPI_OBS) {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                const double ur = u[c].x, ui = u[c].y;
                acc[0] += ur * ur + ui * ui;
                acc[1] += ur * (double)kin[c].x + ui * (double)kin[c].y;
                acc[2] += (double)Vv[c] * (ur * ur + ui * ui);
                acc[4] += ur * (double)h[c].x + ui * (double)h[c].y;
            }
            acc[3] += interaction_energy<Real, NC>(P, nn);
        }
        return;
    }
    if (mode == EPI_RK1 || mode == EPI_RK2 || mode == EPI_RK3) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const long long g = s + (long long)c * P.nsites;
            if (mode == EPI_RK1) {
                P.kout[g] = h[c];
            } else if (mode == EPI_RK2) {
                P.kout[g] = h[c];
                P.kacc[g] = cadd(in[c].kprev, cscale(h[c], (Real)2));
            } else {
                P.kacc[g] = cadd(in[c].kacc, cscale(h[c], (Real)2));
                P.kout[g] = h[c];
            }
            if (P.turn) {
                V cn;
                cn.x = P.cnre;
                cn.y = P.cnim;
                const V nx = csub(p[c], cmul(cn, h[c]));
                next[c] = nx;
                if (RED) acc[c] += (double)nx.x * (double)nx.x + (double)nx.y * (double)nx.y;
            }
        }
        return;
    }
    // EULER / RK4: psi1 = p - d * (sum)
    V d;
    d.x = P.dre;
    d.y = P.dim;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const long long g = s + (long long)c * P.nsites;
        V sum = h[c];
        if (mode == EPI_RK4) sum = cadd(in[c].kacc, h[c]);
        V r = csub(p[c], cmul(d, sum));
        if (P.phase_exp) {
            const Real a = sqrt(r.x * r.x + r.y * r.y);
            r = cscale(P.phase_exp[g], a);
        }
        P.psi_out[g] = r;
        if (P.turn) next[c] = r;
        if (RED && P.renorm_out) acc[c] += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    }
}

template <typename Real> struct EpiFinalize {
    // OBS: keep the raw sums; mu for the residual.  RK4/EULER with renorm: new sigma.
    static __device__ __forceinline__ void run(const EpiParams<Real> &P, const double *s) {
        DevScalars *ds = P.ds;
        if (P.mode == EPI_OBS) {
            for (int r = 0; r < 8; r++) ds->sums[r] = s[r];
            ds->mu = s[4] / s[0];
            if (!isfinite(s[0]) || !isfinite(s[4])) ds->status |= DS_NONFINITE;
        } else if ((P.mode == EPI_EULER || P.mode == EPI_RK4) && P.renorm_out) {
            ds->sigma[0] = sqrt(P.Nt0 / (P.dV * s[0]));
            ds->sigma[1] = (P.Nt1 > 0) ? sqrt(P.Nt1 / (P.dV * s[1])) : 1.0;
            if (P.turn) {
                // the next step transforms the raw state: its first stage scales by sigma
                ds->alpha[1][0] = ds->sigma[0];
                ds->alpha[1][1] = ds->sigma[1];
            }
            if (!isfinite(s[0]) || !isfinite(ds->sigma[0])) ds->status |= DS_NONFINITE;
        } else if (P.turn && P.renorm_out) {
            // normalisation of the next stage's input u~_{s+1} (slot of stage s+1)
            const int ns = P.slot ^ 1;
            ds->alpha[ns][0] = sqrt(P.Nt0 / (P.dV * s[0]));
            ds->alpha[ns][1] = (P.Nt1 > 0) ? sqrt(P.Nt1 / (P.dV * s[1])) : 1.0;
            if (!isfinite(s[0]) || !isfinite(ds->alpha[ns][0])) ds->status |= DS_NONFINITE;
        }
    }
};

// Fused epilogue (one component): the inverse x pass hands every element to the site logic.
// TURN (stage boundary, mode inverse -> turn -> forward): turn() runs the epilogue of stage s
// and returns the next stage's transform input; post() stores the forward transform into src.
template <typename Real, bool RED, bool TURN = false> struct OpStageOut {
    static constexpr int NRED = RED ? kNRed : 0, BATCH = 2;
    using V = cpx<Real>;
    using Pre = EpiIn<Real>;
    const V *src;  // inverse-pass input buffer (the boundary kernel writes it back in place)
    EpiParams<Real> P;
    __device__ __forceinline__ V load(long long g, const LineRef &, double *) const { return src[g]; }
    __device__ __forceinline__ V mid(V v, const LineRef &) const { return v; }
    __device__ __forceinline__ Pre pre(long long g) const { return epi_load(P, g); }
    __device__ __forceinline__ V turn(long long g, const LineRef &e, V v, const Pre &in, double *acc) const {
        const V t[1] = {v};
        const Pre ins[1] = {in};
        V nx[1] = {v};
        epilogue_site<Real, 1, RED>(P, g, e.i, e.j, e.k, t, ins, acc, nx);
        return nx[0];
    }
    __device__ __forceinline__ void post(long long g, const LineRef &e, V v, const Pre &in, double *acc) const {
        if (TURN) {
            const_cast<V *>(src)[g] = v;
        } else {
            const V t[1] = {v};
            const Pre ins[1] = {in};
            V nx[1];
            epilogue_site<Real, 1, RED>(P, g, e.i, e.j, e.k, t, ins, acc, nx);
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
    __device__ __forceinline__ void finalize(const double *s) const { EpiFinalize<Real>::run(P, s); }
};

// Non-fused epilogue over sites (two components): t from the kinetic buffer.
template <typename Real, int NC, bool RED> struct OpSiteEpilogue {
    static constexpr int NRED = RED ? kNRed : 0;
    using V = cpx<Real>;
    EpiParams<Real> P;
    __device__ __forceinline__ void site(long long s, double *acc) const {
        V t[NC];
        EpiIn<Real> in[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            t[c] = P.tsrc[s + (long long)c * P.nsites];
            in[c] = epi_load(P, s + (long long)c * P.nsites);
        }
        const int i = (int)(s % P.nx);
        const long long r = s / P.nx;
        const int j = (int)(r % P.ny), k = (int)(r / P.ny);
        V nx[NC];
        epilogue_site<Real, NC, RED>(P, s, i, j, k, t, in, acc, nx);
    }
    __device__ __forceinline__ void finalize(const double *s) const { EpiFinalize<Real>::run(P, s); }
};

// ---- point-wise ops ------------------------------------------------------------------------
// sum |psi_c|^2 over one component (or all when comp < 0); result in ds->sums[0], factor for
// normalize = sqrt(N / (dV S)).
template <typename Real> struct OpNorm {
    static constexpr int NRED = 1;
    using V = cpx<Real>;
    const V *f;
    long long nsites;
    int comp, ncomp;
    DevScalars *ds;
    double Ntarget, dV;
    __device__ __forceinline__ void site(long long s, double *acc) const {
        if (comp >= 0) {
            const V v = f[s + (long long)comp * nsites];
            acc[0] += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
        } else {
            for (int c = 0; c < ncomp; c++) {
                const V v = f[s + (long long)c * nsites];
                acc[0] += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
            }
        }
    }
    __device__ __forceinline__ void finalize(const double *s) const {
        ds->sums[0] = s[0];
        ds->factor = Ntarget > 0 ? sqrt(Ntarget / (dV * s[0])) : 1.0;
        if (!isfinite(s[0])) ds->status |= DS_NONFINITE;
    }
};

// psi_c *= factor (device scalar); comp < 0 scales every component by sigma[c].
template <typename Real> struct OpScale {
    static constexpr int NRED = 0;
    using V = cpx<Real>;
    V *f;
    long long nsites;
    int comp, ncomp;
    DevScalars *ds;
    int from_sigma;
    __device__ __forceinline__ void site(long long s, double *) const {
        if (!from_sigma) {
            const Real a = (Real)ds->factor;
            const long long g = s + (long long)comp * nsites;
            f[g] = cscale(f[g], a);
        } else {
            for (int c = 0; c < ncomp; c++) {
                const long long g = s + (long long)c * nsites;
                f[g] = cscale(f[g], (Real)ds->sigma[c]);
            }
        }
    }
    __device__ __forceinline__ void finalize(const double *) const {}
};

// max |psi|^2 over every site and component (exact, order-independent)
template <typename Real> struct OpMaxDensity {
    static constexpr int NRED = 0;
    using V = cpx<Real>;
    const V *f;
    long long nsites;
    int ncomp;
    unsigned long long *out;  // double bits of a non-negative value: integer order == value order
    __device__ __forceinline__ void site(long long s, double *) const {
        double m = 0.0;
        for (int c = 0; c < ncomp; c++) {
            const V v = f[s + (long long)c * nsites];
            const double n = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
            m = n > m ? n : m;
        }
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
    __device__ __forceinline__ void finalize(const double *) const {}
};

// residual: sum |H psi - mu psi|^2
template <typename Real> struct OpResidual {
    static constexpr int NRED = 1;
    using V = cpx<Real>;
    const V *psi, *hpsi;
    long long nsites;
    int ncomp;
    DevScalars *ds;
    __device__ __forceinline__ void site(long long s, double *acc) const {
        const double mu = __ldg(&ds->mu);
        for (int c = 0; c < ncomp; c++) {
            const long long g = s + (long long)c * nsites;
            const V a = psi[g], h = hpsi[g];
            const double rx = (double)h.x - mu * (double)a.x, ry = (double)h.y - mu * (double)a.y;
            acc[0] += rx * rx + ry * ry;
        }
    }
    __device__ __forceinline__ void finalize(const double *s) const { ds->sums[5] = s[0]; }
};

// complex128 <-> plan precision conversion
template <typename Real> struct OpConvert {
    static constexpr int NRED = 0;
    const double2 *in128;
    cpx<Real> *out;
    const cpx<Real> *in;
    double2 *out128;
    __device__ __forceinline__ void site(long long s, double *) const {
        if (in128) {
            const double2 v = in128[s];
            out[s] = mk<Real>((Real)v.x, (Real)v.y);
        } else {
            const cpx<Real> v = in[s];
            out128[s] = make_double2((double)v.x, (double)v.y);
        }
    }
    __device__ __forceinline__ void finalize(const double *) const {}
};

}  // namespace gp5

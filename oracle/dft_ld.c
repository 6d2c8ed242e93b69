/*
 * Long-double direct DFT: the pin for every FFT in this project (test infrastructure only;
 * only tests/ and the smoke check load it).
 *
 * Restates the transform the reference asks FFTW for in src/fourierTransform.cpp:146-174
 * (fftw_plan_many_dft over dims {Nz,Ny,Nx} of ColMajor data, one component at a time,
 * FFTW_FORWARD = e^{-2 pi i jk/n}, FFTW_BACKWARD = e^{+2 pi i jk/n}, unnormalised), as
 * three separable O(n^2) passes in 80-bit long double.  Twiddles use the exact integer
 * phase (j*k mod n) so that the argument of sinl/cosl never grows.
 *
 * Data: interleaved (re, im) doubles, index = i + nx*(j + ny*(k + nz*c)).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef long double ld;

static void dft_axis(ld *re, ld *im, int nx, int ny, int nz, int axis, int dir) {
    int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    long stride = axis == 0 ? 1 : (axis == 1 ? nx : (long)nx * ny);
    ld *cr = (ld *)malloc(sizeof(ld) * n), *ci = (ld *)malloc(sizeof(ld) * n);
    ld *tr = (ld *)malloc(sizeof(ld) * n), *ti = (ld *)malloc(sizeof(ld) * n);
    const ld twopi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < n; m++) {
        ld a = twopi * (ld)m / (ld)n;
        cr[m] = cosl(a);
        ci[m] = (ld)dir * sinl(a);
    }
    long total = (long)nx * ny * nz;
    for (long base = 0; base < total; base++) {
        /* base enumerates the first element of each line: its axis coordinate must be 0 */
        long i = base % nx, j = (base / nx) % ny, k = base / ((long)nx * ny);
        long coord = axis == 0 ? i : (axis == 1 ? j : k);
        if (coord != 0) continue;
        for (int q = 0; q < n; q++) {
            ld sr = 0, si = 0;
            for (int p = 0; p < n; p++) {
                int m = (int)(((long)p * q) % n);
                ld xr = re[base + p * stride], xi = im[base + p * stride];
                sr += xr * cr[m] - xi * ci[m];
                si += xr * ci[m] + xi * cr[m];
            }
            tr[q] = sr;
            ti[q] = si;
        }
        for (int q = 0; q < n; q++) {
            re[base + q * stride] = tr[q];
            im[base + q * stride] = ti[q];
        }
    }
    free(cr); free(ci); free(tr); free(ti);
}

/* dir = -1 forward, +1 backward; ncomp components transformed independently */
void dft3_ld(int nx, int ny, int nz, int ncomp, const double *in, double *out, int dir) {
    long n = (long)nx * ny * nz;
    ld *re = (ld *)malloc(sizeof(ld) * n), *im = (ld *)malloc(sizeof(ld) * n);
    for (int c = 0; c < ncomp; c++) {
        const double *src = in + 2 * n * c;
        for (long s = 0; s < n; s++) { re[s] = src[2 * s]; im[s] = src[2 * s + 1]; }
        dft_axis(re, im, nx, ny, nz, 0, dir);
        dft_axis(re, im, nx, ny, nz, 1, dir);
        dft_axis(re, im, nx, ny, nz, 2, dir);
        double *dst = out + 2 * n * c;
        for (long s = 0; s < n; s++) { dst[2 * s] = (double)re[s]; dst[2 * s + 1] = (double)im[s]; }
    }
    free(re); free(im);
}

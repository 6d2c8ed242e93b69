/* cluster.c - CPU restatement of gp::decompose::decompose (src/cluster.cpp:17-83), the
 * reference's droplet labelling.  Test infrastructure only: the GPU kernels of
 * gp5_b200/csrc/gp5cu_cluster.cu are checked against it.
 *
 * Scan (i outermost, then j, then k, src/cluster.cpp:26-39): an unvisited site starts a depth-
 * first traversal that gives every site with density > cutoff reachable through the 26
 * neighbours (periodic, src/cluster.cpp:12-15,70-80) the current color and marks each visited
 * site at or below the cutoff with -1 (src/cluster.cpp:53-62); the color advances when the
 * starting site got it (src/cluster.cpp:34-37).  The reference recurses; this restatement keeps
 * the same visiting rule with an explicit stack, which changes the order of visits inside one
 * traversal but not the labels; a site is queued once (marked -2 until it is visited).
 *
 * psi: interleaved complex128, ColMajor (x fastest, component slowest); out: int32 in the same
 * layout, only component `comp` is written (the caller zero-fills). */
#include <stdlib.h>

static long long idx(int i, int j, int k, int nx, int ny) { return i + (long long)nx * (j + (long long)ny * k); }
static int pbc(int i, int L) { return i < 0 ? i + L : (i >= L ? i - L : i); }

int decompose(int nx, int ny, int nz, int comp, const double *psi, double cutoff, int *out) {
    const long long n = (long long)nx * ny * nz;
    const double *p = psi + 2 * n * comp;
    int *lab = out + n * comp;
    for (long long s = 0; s < n; s++) lab[s] = 0;
    long long *stack = (long long *)malloc(sizeof(long long) * (size_t)(n + 1));
    if (!stack) return -1;
    int color = 1;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const long long s0 = idx(i, j, k, nx, ny);
                if (lab[s0] != 0) continue;
                long long top = 0;
                stack[top++] = s0;
                lab[s0] = -2;
                while (top > 0) {
                    const long long s = stack[--top];
                    const double re = p[2 * s], im = p[2 * s + 1];
                    const double d = re * re + im * im;
                    if (!(d > cutoff)) {
                        lab[s] = -1;
                        continue;
                    }
                    lab[s] = color;
                    const int si = (int)(s % nx), sj = (int)((s / nx) % ny), sk = (int)(s / ((long long)nx * ny));
                    for (int a = -1; a <= 1; a++)
                        for (int b = -1; b <= 1; b++)
                            for (int c = -1; c <= 1; c++) {
                                const long long t = idx(pbc(si + a, nx), pbc(sj + b, ny), pbc(sk + c, nz), nx, ny);
                                if (lab[t] == 0) {
                                    lab[t] = -2;
                                    stack[top++] = t;
                                }
                            }
                }
                if (lab[s0] != -1) color += 1;
            }
    free(stack);
    return color - 1;
}

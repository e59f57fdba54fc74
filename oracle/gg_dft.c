/*
 * gg_dft.c -- the specified 3D real DFT (TEST INFRASTRUCTURE, see gg_dft.h).
 *
 * Every output is one sequential fma chain over m = 0..n-1, so the loop nest may
 * be reordered freely (and vectorised across independent outputs) without
 * changing a single bit.  The loops below put the independent outputs innermost
 * so that the compiler can vectorise them.
 */
#include "gg_dft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void ggdft_twiddles(int n, double* c, double* s) {
    for (int j = 0; j < n; j++) {
        double a = 6.283185307179586476925286766559 * (double)j / (double)n;
        c[j] = cos(a);
        s[j] = sin(a);
    }
}

/* Complex line transform along an axis: for every output k and every one of the
 * `cnt` independent lines (contiguous in the innermost index), accumulate over m.
 * src/dst are split planes: re[m * cnt + l], im[m * cnt + l]. */
static void line_dft(int n, int cnt, const double* c, const double* s, int inverse,
                     const double* sre, const double* sim, double* dre, double* dim) {
    for (int k = 0; k < n; k++) {
        double* ore = dre + (size_t)k * cnt;
        double* oim = dim + (size_t)k * cnt;
        for (int l = 0; l < cnt; l++) { ore[l] = 0.0; oim[l] = 0.0; }
        int t = 0;
        for (int m = 0; m < n; m++) {
            const double cc = c[t], ss = s[t];
            const double* ir = sre + (size_t)m * cnt;
            const double* ii = sim + (size_t)m * cnt;
            if (!inverse) {
                for (int l = 0; l < cnt; l++) {
                    double re = ore[l], im = oim[l];
                    re = fma(ir[l], cc, re);
                    re = fma(ii[l], ss, re);
                    im = fma(ii[l], cc, im);
                    im = fma(-ir[l], ss, im);
                    ore[l] = re; oim[l] = im;
                }
            } else {
                for (int l = 0; l < cnt; l++) {
                    double re = ore[l], im = oim[l];
                    re = fma(ir[l], cc, re);
                    re = fma(-ii[l], ss, re);
                    im = fma(ii[l], cc, im);
                    im = fma(ir[l], ss, im);
                    ore[l] = re; oim[l] = im;
                }
            }
            t += k; if (t >= n) t -= n;
        }
    }
}

void ggdft_forward_r2c_3d(int n, const double* in, double* out) {
    const int h = n / 2 + 1;
    const size_t plane = (size_t)n * h;          /* one z-plane of the half spectrum */
    double* c = (double*)malloc(sizeof(double) * 2 * n);
    double* s = c + n;
    ggdft_twiddles(n, c, s);
    double* are = (double*)malloc(sizeof(double) * plane * n);
    double* aim = (double*)malloc(sizeof(double) * plane * n);
    double* bre = (double*)malloc(sizeof(double) * plane * n);
    double* bim = (double*)malloc(sizeof(double) * plane * n);
    double* xt = (double*)malloc(sizeof(double) * n * n);
    /* x axis (r2c): per z-plane, transpose to [x][y] so that the n lines of the
     * plane are contiguous; result a[z][kx][y]. */
    for (int z = 0; z < n; z++) {
        const double* src = in + (size_t)z * n * n;
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++) xt[(size_t)x * n + y] = src[(size_t)y * n + x];
        double* ore = are + (size_t)z * plane;
        double* oim = aim + (size_t)z * plane;
        for (int k = 0; k < h; k++) {
            double* r = ore + (size_t)k * n;
            double* i = oim + (size_t)k * n;
            for (int y = 0; y < n; y++) { r[y] = 0.0; i[y] = 0.0; }
            int t = 0;
            for (int m = 0; m < n; m++) {
                const double cc = c[t], ss = s[t];
                const double* xv = xt + (size_t)m * n;
                for (int y = 0; y < n; y++) {
                    r[y] = fma(xv[y], cc, r[y]);
                    i[y] = fma(-xv[y], ss, i[y]);
                }
                t += k; if (t >= n) t -= n;
            }
        }
    }
    /* y axis: per z-plane, lines indexed by kx (a[z][kx][y] -> need [y][kx]).
     * Transpose each plane to [y][kx], transform along y with kx innermost. */
    for (int z = 0; z < n; z++) {
        double* pr = are + (size_t)z * plane;
        double* pi = aim + (size_t)z * plane;
        double* tr = bre + (size_t)z * plane;
        double* ti = bim + (size_t)z * plane;
        for (int k = 0; k < h; k++)
            for (int y = 0; y < n; y++) {
                tr[(size_t)y * h + k] = pr[(size_t)k * n + y];
                ti[(size_t)y * h + k] = pi[(size_t)k * n + y];
            }
        line_dft(n, h, c, s, 0, tr, ti, pr, pi);   /* pr/pi now [ky][kx] */
    }
    /* z axis: lines indexed by (ky,kx), contiguous plane of size n*h. */
    line_dft(n, (int)plane, c, s, 0, are, aim, bre, bim);
    for (size_t q = 0; q < plane * n; q++) { out[2 * q] = bre[q]; out[2 * q + 1] = bim[q]; }
    free(xt); free(bim); free(bre); free(aim); free(are); free(c);
}

void ggdft_backward_c2r_3d(int n, const double* in, double* out) {
    const int h = n / 2 + 1;
    const size_t plane = (size_t)n * h;
    double* c = (double*)malloc(sizeof(double) * 2 * n);
    double* s = c + n;
    ggdft_twiddles(n, c, s);
    double* are = (double*)malloc(sizeof(double) * plane * n);
    double* aim = (double*)malloc(sizeof(double) * plane * n);
    double* bre = (double*)malloc(sizeof(double) * plane * n);
    double* bim = (double*)malloc(sizeof(double) * plane * n);
    for (size_t q = 0; q < plane * n; q++) { are[q] = in[2 * q]; aim[q] = in[2 * q + 1]; }
    /* z axis */
    line_dft(n, (int)plane, c, s, 1, are, aim, bre, bim);
    /* y axis: plane [ky][kx] -> lines over ky, kx innermost; result [y][kx] */
    for (int z = 0; z < n; z++)
        line_dft(n, h, c, s, 1, bre + (size_t)z * plane, bim + (size_t)z * plane,
                 are + (size_t)z * plane, aim + (size_t)z * plane);
    /* x axis (c2r): per z-plane, X[y][kx]; transpose to [kx][y], accumulate with y innermost. */
    double* xr = bre; double* xi = bim;          /* reuse as [kx][y] per plane */
    double* acc = (double*)malloc(sizeof(double) * n);
    for (int z = 0; z < n; z++) {
        const double* pr = are + (size_t)z * plane;
        const double* pi = aim + (size_t)z * plane;
        for (int y = 0; y < n; y++)
            for (int k = 0; k < h; k++) {
                xr[(size_t)k * n + y] = pr[(size_t)y * h + k];
                xi[(size_t)k * n + y] = pi[(size_t)y * h + k];
            }
        double* dst = out + (size_t)z * n * n;
        for (int m = 0; m < n; m++) {
            for (int y = 0; y < n; y++) acc[y] = xr[y];
            int t = 0;
            for (int k = 1; k < h; k++) {
                t += m; if (t >= n) t -= n;          /* t = (k*m) mod n */
                const double cc = c[t], ss = s[t];
                const double* rr = xr + (size_t)k * n;
                const double* ii = xi + (size_t)k * n;
                if (2 * k == n) {
                    for (int y = 0; y < n; y++) acc[y] = fma(rr[y], cc, acc[y]);
                } else {
                    for (int y = 0; y < n; y++) {
                        double a = fma(2.0 * rr[y], cc, acc[y]);
                        acc[y] = fma(-2.0 * ii[y], ss, a);
                    }
                }
            }
            for (int y = 0; y < n; y++) dst[(size_t)y * n + m] = acc[y];
        }
    }
    free(acc); free(bim); free(bre); free(aim); free(are); free(c);
}

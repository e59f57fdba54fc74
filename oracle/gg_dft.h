/*
 * gg_dft.h -- the specified 3D real DFT used by the oracle (TEST INFRASTRUCTURE).
 *
 * The reference convolves each grain box with a Gaussian through Intel MKL DFTI
 * (box.cpp:685-795: DftiComputeForward -> multiply by G -> DftiComputeBackward,
 * unnormalised, dims {n,n,n}, input strides {0,n,n*n,1}, output strides
 * {0,n/2+1,(n/2+1)*n,1}).  MKL is a closed binary that is not available here, so
 * the oracle replaces it with this DFT, whose arithmetic is fixed down to the
 * order of every fused multiply-add.  The FP64 GPU path implements the very same
 * sequence, which makes the two bit-identical.
 *
 * Layout: a cubic box of side n, real values flat [z][y][x] (x fastest).  The
 * half spectrum is flat [kz][ky][kx], kx in [0, n/2], complex interleaved
 * (re, im) -- exactly MKL's CCE output for the strides above.
 *
 * Twiddles: c[j] = cos(2*pi*j/n), s[j] = sin(2*pi*j/n), j in [0, n), from libm,
 * angle evaluated as (6.283185307179586 * j) / n.
 *
 * Forward (r2c), axes in the order x, y, z.  For every output the sum runs over
 * m = 0..n-1 in increasing order, starting from +0.0, index t = (k*m) mod n:
 *   x (real in):    re = fma(r, c[t], re);             im = fma(-r, s[t], im)
 *   y, z (complex): re = fma(zr, c[t], re); re = fma(zi, s[t], re);
 *                   im = fma(zi, c[t], im); im = fma(-zr, s[t], im)
 * Backward (c2r), axes in the order z, y, x:
 *   z, y (complex): re = fma(zr, c[t], re); re = fma(-zi, s[t], re);
 *                   im = fma(zi, c[t], im); im = fma(zr, s[t], im)
 *   x (c2r): acc = X[0].re; then for k = 1..n/2:
 *            if 2k == n:  acc = fma(X[k].re, c[t], acc)
 *            else:        acc = fma(2*X[k].re, c[t], acc); acc = fma(-2*X[k].im, s[t], acc)
 *            (imaginary parts of X[0] and X[n/2] are ignored, as a c2r transform does)
 */
#ifndef GG_DFT_H
#define GG_DFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* c[j] = cos(2 pi j / n), s[j] = sin(2 pi j / n) for j in [0, n). */
void ggdft_twiddles(int n, double* c, double* s);

/* Unnormalised forward r2c transform of an n^3 box; out holds 2*n*n*(n/2+1) doubles. */
void ggdft_forward_r2c_3d(int n, const double* in, double* out);

/* Unnormalised backward c2r transform; in holds 2*n*n*(n/2+1) doubles, out n^3. */
void ggdft_backward_c2r_3d(int n, const double* in, double* out);

#ifdef __cplusplus
}
#endif
#endif

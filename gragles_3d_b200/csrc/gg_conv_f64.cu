// gg_conv_f64.cu -- FP64 Gaussian convolution of every grain box (the plain path).
//
// Stands in for LSbox::executeConvolution / convolutionGeneratorMKL
// (box.cpp:414-427, 685-795): out = IDFT3(DFT3(in) * G) with
// G = exp(-sqrt(2/pi) * S * 4 dt N^2 / n^2 * pi^2) / n^3, S = i2^2 + j2^2 + k2^2.
//
// The reference's MKL transform is replaced by a DFT whose arithmetic is fixed to
// the order of every fused multiply-add (see the oracle's gg_dft.h): each output
// is one fma chain over m = 0..n-1 with twiddle index (k*m) mod n taken from a
// host-built libm table, and G comes from a host-built table per box side.  These
// kernels run exactly those chains, so the FP64 path is bit-identical to the
// oracle.  The transform is split in three batched passes over all boxes:
//   A  per (grain, z-plane): x r2c, then y                    -> spectrum scratch
//   B  per (grain, ky-row):  z forward, multiply by G, z inverse (in place)
//   C  per (grain, z-plane): y inverse, then x c2r            -> output arena
// Lanes map to independent lines and each thread carries Q frequencies, so every
// twiddle read is a warp-wide broadcast from shared memory.
#include "gg_common.cuh"
#include "gg_conv.cuh"

namespace gg {

namespace {

constexpr int kQ = 4;

__device__ __forceinline__ int odd_pitch(int v) { return v | 1; }

// Complex DFT along nl lines of length n held in shared memory; outputs k in [0, nk).
// src(l, m) = src[l*sl + m*sm], dst(l, k) = dst[l*dl + k*dk].
template <bool INV>
__device__ void cdft_lines(const double2* __restrict__ src, int sl, int sm, double2* __restrict__ dst, int dl,
                           int dk, int n, int nl, int nk, const double2* __restrict__ tw) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int lchunks = (nl + 31) >> 5, kgroups = (nk + kQ - 1) / kQ;
    for (int item = warp; item < lchunks * kgroups; item += nw) {
        const int lc = item % lchunks, kg = item / lchunks;
        const int l = lc * 32 + lane;
        const bool active = l < nl;
        const int k0 = kg * kQ;
        double re[kQ], im[kQ];
        int t[kQ], kk[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            re[q] = 0.0; im[q] = 0.0; t[q] = 0;
            kk[q] = min(k0 + q, nk - 1);
        }
        const double2* s = src + (active ? l : 0) * sl;
        for (int m = 0; m < n; m++) {
            const double2 z = s[m * sm];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                const double2 w = tw[t[q]];
                if (!INV) {
                    re[q] = fma(z.x, w.x, re[q]);
                    re[q] = fma(z.y, w.y, re[q]);
                    im[q] = fma(z.y, w.x, im[q]);
                    im[q] = fma(-z.x, w.y, im[q]);
                } else {
                    re[q] = fma(z.x, w.x, re[q]);
                    re[q] = fma(-z.y, w.y, re[q]);
                    im[q] = fma(z.y, w.x, im[q]);
                    im[q] = fma(z.x, w.y, im[q]);
                }
                t[q] += kk[q];
                if (t[q] >= n) t[q] -= n;
            }
        }
        if (active) {
#pragma unroll
            for (int q = 0; q < kQ; q++)
                if (k0 + q < nk) dst[l * dl + (k0 + q) * dk] = make_double2(re[q], im[q]);
        }
    }
}

// Real-input DFT (x axis, r2c) along nl lines: src(l, m) = src[l*sl + m], outputs k < nk.
__device__ void r2c_lines(const double* __restrict__ src, int sl, double2* __restrict__ dst, int dl, int dk, int n,
                          int nl, int nk, const double2* __restrict__ tw) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int lchunks = (nl + 31) >> 5, kgroups = (nk + kQ - 1) / kQ;
    for (int item = warp; item < lchunks * kgroups; item += nw) {
        const int lc = item % lchunks, kg = item / lchunks;
        const int l = lc * 32 + lane;
        const bool active = l < nl;
        const int k0 = kg * kQ;
        double re[kQ], im[kQ];
        int t[kQ], kk[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            re[q] = 0.0; im[q] = 0.0; t[q] = 0;
            kk[q] = min(k0 + q, nk - 1);
        }
        const double* s = src + (active ? l : 0) * sl;
        for (int m = 0; m < n; m++) {
            const double x = s[m];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                const double2 w = tw[t[q]];
                re[q] = fma(x, w.x, re[q]);
                im[q] = fma(-x, w.y, im[q]);
                t[q] += kk[q];
                if (t[q] >= n) t[q] -= n;
            }
        }
        if (active) {
#pragma unroll
            for (int q = 0; q < kQ; q++)
                if (k0 + q < nk) dst[l * dl + (k0 + q) * dk] = make_double2(re[q], im[q]);
        }
    }
}

// Half-spectrum to real (x axis, c2r): X(l, k) = src[l*sl + k], k < n/2+1; out(l, m) = dst[l*dl + m].
__device__ void c2r_lines(const double2* __restrict__ src, int sl, double* __restrict__ dst, int dl, int n, int nl,
                          const double2* __restrict__ tw) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int h = n / 2 + 1;
    const int lchunks = (nl + 31) >> 5, mgroups = (n + kQ - 1) / kQ;
    for (int item = warp; item < lchunks * mgroups; item += nw) {
        const int lc = item % lchunks, mg = item / lchunks;
        const int l = lc * 32 + lane;
        const bool active = l < nl;
        const int m0 = mg * kQ;
        const double2* s = src + (active ? l : 0) * sl;
        double acc[kQ];
        int t[kQ], mm[kQ];
        const double x0 = s[0].x;
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            acc[q] = x0; t[q] = 0;
            mm[q] = min(m0 + q, n - 1);
        }
        for (int k = 1; k < h; k++) {
            const double2 X = s[k];
            const bool nyq = (2 * k == n);
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                t[q] += mm[q];
                if (t[q] >= n) t[q] -= n;
                const double2 w = tw[t[q]];
                if (nyq) {
                    acc[q] = fma(X.x, w.x, acc[q]);
                } else {
                    const double a = fma(2.0 * X.x, w.x, acc[q]);
                    acc[q] = fma(-2.0 * X.y, w.y, a);
                }
            }
        }
        if (active) {
#pragma unroll
            for (int q = 0; q < kQ; q++)
                if (m0 + q < n) dst[l * dl + m0 + q] = acc[q];
        }
    }
}

__device__ __forceinline__ void load_twiddles(double2* tw_s, const double2* __restrict__ tw, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) tw_s[j] = tw[j];
}

// Pass A: x r2c then y forward, one z-plane per tile.
__global__ void __launch_bounds__(256) conv_pass_a(ConvArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int z = t - a.toff[g];
        const Box b = load_box(a.in_box + 6 * g);
        const int n = b.nx(), h = n / 2 + 1;
        const int P = odd_pitch(n), Hp = odd_pitch(h);
        double2* tw_s = reinterpret_cast<double2*>(smem_raw);
        double* xp = reinterpret_cast<double*>(tw_s + n);
        double2* A = reinterpret_cast<double2*>(xp + ((n * P + 1) & ~1));
        load_twiddles(tw_s, a.tw + a.tw_off[n], n);
        const double* src = a.in + a.in_off[g] + (long long)z * n * n;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int y = q / n, x = q - y * n;
            xp[y * P + x] = src[q];
        }
        __syncthreads();
        r2c_lines(xp, P, A, Hp, 1, n, n, h, tw_s);
        __syncthreads();
        double2* dst = a.spec + a.spec_off[g] + (long long)z * n * h;
        cdft_lines<false>(A, 1, Hp, dst, 1, h, n, h, n, tw_s);
        __syncthreads();
    }
}

// Pass B: z forward, Gaussian multiply, z inverse, one ky-row of the spectrum per tile.
__global__ void __launch_bounds__(256) conv_pass_b(ConvArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int ky = t - a.toff[g];
        const Box b = load_box(a.in_box + 6 * g);
        const int n = b.nx(), h = n / 2 + 1;
        const int Hp = odd_pitch(h);
        double2* tw_s = reinterpret_cast<double2*>(smem_raw);
        double2* S = tw_s + n;
        double2* T = S + n * Hp;
        load_twiddles(tw_s, a.tw + a.tw_off[n], n);
        double2* spec = a.spec + a.spec_off[g];
        for (int q = threadIdx.x; q < n * h; q += blockDim.x) {
            const int z = q / h, kx = q - z * h;
            S[z * Hp + kx] = spec[((long long)z * n + ky) * h + kx];
        }
        __syncthreads();
        cdft_lines<false>(S, 1, Hp, T, 1, Hp, n, h, n, tw_s);
        __syncthreads();
        const double* G = a.gtab + a.g_off[n];
        const int i2 = min(ky, n - ky);
        for (int q = threadIdx.x; q < n * h; q += blockDim.x) {
            const int kz = q / h, kx = q - kz * h;
            const int j2 = min(kx, n - kx), k2 = min(kz, n - kz);
            const double gv = __ldg(G + (i2 * i2 + j2 * j2 + k2 * k2));
            double2 v = T[kz * Hp + kx];
            v.x = v.x * gv;
            v.y = v.y * gv;
            T[kz * Hp + kx] = v;
        }
        __syncthreads();
        cdft_lines<true>(T, 1, Hp, spec + (long long)ky * h, 1, n * h, n, h, n, tw_s);
        __syncthreads();
    }
}

// Pass C: y inverse then x c2r, one z-plane per tile, written to the output arena.
__global__ void __launch_bounds__(256) conv_pass_c(ConvArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int z = t - a.toff[g];
        const Box b = load_box(a.in_box + 6 * g);
        const int n = b.nx(), h = n / 2 + 1;
        const int P = odd_pitch(n), Hp = odd_pitch(h);
        double2* tw_s = reinterpret_cast<double2*>(smem_raw);
        double2* Pk = tw_s + n;        // [ky][kx]
        double2* Ay = Pk + n * Hp;     // [y][kx]
        double* xo = reinterpret_cast<double*>(Ay + n * Hp);  // [y][x], pitch P
        load_twiddles(tw_s, a.tw + a.tw_off[n], n);
        const double2* spec = a.spec + a.spec_off[g] + (long long)z * n * h;
        for (int q = threadIdx.x; q < n * h; q += blockDim.x) {
            const int ky = q / h, kx = q - ky * h;
            Pk[ky * Hp + kx] = spec[q];
        }
        __syncthreads();
        cdft_lines<true>(Pk, 1, Hp, Ay, 1, Hp, n, h, n, tw_s);
        __syncthreads();
        c2r_lines(Ay, Hp, xo, P, n, n, tw_s);
        __syncthreads();
        double* dst = a.out + a.out_off[g] + (long long)z * n * n;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int y = q / n, x = q - y * n;
            dst[q] = xo[y * P + x];
        }
        __syncthreads();
    }
}

}  // namespace

size_t conv_f64_smem_bytes(int nmax) {
    const int n = nmax, h = n / 2 + 1, P = n | 1, Hp = h | 1;
    size_t a = 16 * n + 8 * (size_t)((n * P + 1) & ~1) + 16 * (size_t)n * Hp;
    size_t b = 16 * n + 2 * 16 * (size_t)n * Hp;
    size_t c = 16 * n + 2 * 16 * (size_t)n * Hp + 8 * (size_t)n * P;
    size_t m = a > b ? a : b;
    return m > c ? m : c;
}

int conv_f64_max_side(size_t smem_limit) {
    int n = 8;
    while (n < 4096 && conv_f64_smem_bytes(n + 1) <= smem_limit) n++;
    return n;
}

void launch_conv_f64(const ConvArgs& a, int grid, size_t smem, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(conv_pass_a);
        allow_max_dynamic_smem(conv_pass_b);
        allow_max_dynamic_smem(conv_pass_c);
    });
    conv_pass_a<<<grid, 256, smem, s>>>(a);
    conv_pass_b<<<grid, 256, smem, s>>>(a);
    conv_pass_c<<<grid, 256, smem, s>>>(a);
}

}  // namespace gg

// gg_conv_tc.cu -- mixed-precision per-axis circulant convolution (FP32 storage).
//
// See gg_conv_tc.cuh.  Two batched passes over all boxes:
//   xy: one CTA per (grain, z-plane): x then y contraction of the plane with C_n
//   z:  one CTA per (grain, y-row):   z contraction of the [z][x] slab, in place
// Each thread holds a 4-row block of outputs so every C_n read feeds four FMAs.
#include <cmath>

#include "gg_common.cuh"
#include "gg_conv_tc.cuh"

namespace gg {

void circulant_matrix(int n, int N, double time_step, std::vector<float>& out) {
    // per-axis factor of box.cpp:760-761: exp(-sqrt(2/pi) 4 dt N^2 pi^2 / n^2 * f^2), f = min(k, n-k)
    const double pi = 3.14159265358979323846;
    const double dt = time_step / double(N * N);
    const double c = std::sqrt(2 / pi) * 4.0 * dt * double(N * N) / double(n * n) * pi * pi;
    std::vector<long double> col(n);
    for (int d = 0; d < n; d++) {
        long double acc = 0;
        for (int f = 0; f < n; f++) {
            const int ff = f < n - f ? f : n - f;
            acc += std::exp(-(long double)c * ff * ff) * std::cos(2.0L * (long double)pi * f * d / n);
        }
        col[d] = acc / n;
    }
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) out.push_back((float)col[(p - q + n) % n]);
}

namespace {

constexpr int kThreads = 256;
constexpr int kR = 4;

// dst[r][k] = sum_m C[k][m] * src[r][m] for rows r < nr, outputs k < n.
// src/dst row pitch sp/dp, C row pitch cp.  Lanes cover k, each thread kR rows.
__device__ void rows_times_ct(const float* __restrict__ src, int sp, float* __restrict__ dst, int dp,
                              const float* __restrict__ C, int cp, int n, int nr) {
    const int nkc = (n + 31) >> 5, nrg = (nr + kR - 1) / kR;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int item = warp; item < nkc * nrg; item += nw) {
        const int kc = item % nkc, rg = item / nkc;
        const int k = kc * 32 + lane;
        const int kk = k < n ? k : n - 1;
        const int r0 = rg * kR;
        float acc[kR];
#pragma unroll
        for (int r = 0; r < kR; r++) acc[r] = 0.f;
        const float* crow = C + kk * cp;
        for (int m = 0; m < n; m++) {
            const float cv = crow[m];
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int rr = min(r0 + r, nr - 1);
                acc[r] = fmaf(cv, src[rr * sp + m], acc[r]);
            }
        }
        if (k < n) {
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (r0 + r < nr) dst[(r0 + r) * dp + k] = acc[r];
        }
    }
}

// dst[k][c] = sum_m C[k][m] * src[m][c] for columns c < nc, outputs k < n (lanes cover c).
__device__ void ct_times_cols(const float* __restrict__ src, int sp, float* __restrict__ dst, int dp,
                              const float* __restrict__ C, int cp, int n, int nc) {
    const int ncc = (nc + 31) >> 5, nkg = (n + kR - 1) / kR;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int item = warp; item < ncc * nkg; item += nw) {
        const int cc = item % ncc, kg = item / ncc;
        const int c = cc * 32 + lane;
        const int c2 = c < nc ? c : nc - 1;
        const int k0 = kg * kR;
        float acc[kR];
#pragma unroll
        for (int r = 0; r < kR; r++) acc[r] = 0.f;
        for (int m = 0; m < n; m++) {
            const float v = src[m * sp + c2];
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int kk = min(k0 + r, n - 1);
                acc[r] = fmaf(C[kk * cp + m], v, acc[r]);
            }
        }
        if (c < nc) {
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (k0 + r < n) dst[(k0 + r) * dp + c] = acc[r];
        }
    }
}

__global__ void __launch_bounds__(kThreads) conv_xy_kernel(ConvTCArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int z = t - a.toff[g];
        const Box b = load_box(a.box + 6 * g);
        const int n = b.nx(), cp = n | 1;
        float* C = reinterpret_cast<float*>(smem_raw);
        float* P = C + n * cp;
        float* Q = P + n * cp;
        const float* Cg = a.circ + a.circ_off[n];
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) C[(q / n) * cp + q % n] = Cg[q];
        const float* src = a.in + a.in_off[g] + (long long)z * n * n;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) P[(q / n) * cp + q % n] = src[q];
        __syncthreads();
        rows_times_ct(P, cp, Q, cp, C, cp, n, n);    // x: Q[y][x'] = sum_x C[x'][x] P[y][x]
        __syncthreads();
        ct_times_cols(Q, cp, P, cp, C, cp, n, n);    // y: P[y'][x] = sum_y C[y'][y] Q[y][x]
        __syncthreads();
        float* dst = a.out + a.out_off[g] + (long long)z * n * n;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) dst[q] = P[(q / n) * cp + q % n];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) conv_z_kernel(ConvTCArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int y = t - a.toff[g];
        const Box b = load_box(a.box + 6 * g);
        const int n = b.nx(), cp = n | 1;
        float* C = reinterpret_cast<float*>(smem_raw);
        float* S = C + n * cp;
        float* T = S + n * cp;
        const float* Cg = a.circ + a.circ_off[n];
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) C[(q / n) * cp + q % n] = Cg[q];
        float* io = a.out + a.out_off[g] + (long long)y * n;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int zz = q / n, x = q % n;
            S[zz * cp + x] = io[(long long)zz * n * n + x];
        }
        __syncthreads();
        ct_times_cols(S, cp, T, cp, C, cp, n, n);    // z: T[z'][x] = sum_z C[z'][z] S[z][x]
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int zz = q / n, x = q % n;
            io[(long long)zz * n * n + x] = T[zz * cp + x];
        }
        __syncthreads();
    }
}

}  // namespace

void launch_conv_tc(const ConvTCArgs& a, int num_sms, int side_max, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(conv_xy_kernel);
        allow_max_dynamic_smem(conv_z_kernel);
    });
    const int n = side_max;
    const size_t smem = 3 * (size_t)n * (n | 1) * sizeof(float);
    const int grid = num_sms * 8;
    conv_xy_kernel<<<grid, kThreads, smem, s>>>(a);
    conv_z_kernel<<<grid, kThreads, smem, s>>>(a);
}

}  // namespace gg

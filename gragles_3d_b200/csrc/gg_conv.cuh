// gg_conv.cuh -- launch interface of the convolution passes.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace gg {

struct ConvArgs {
    int G;
    const int* toff;          // tile offsets (G + 2): n tiles per convolved grain
    const double* in;         // input arena
    const int* in_box;
    const long long* in_off;
    double* out;              // output arena (same boxes as the input)
    const long long* out_off;
    double2* spec;            // half-spectrum scratch
    const long long* spec_off;
    const double2* tw;        // (cos, sin) twiddles for every side n, at tw_off[n]
    const long long* tw_off;
    const double* gtab;       // Gaussian multiplier by S = i2^2+j2^2+k2^2, at g_off[n]
    const long long* g_off;
};

size_t conv_f64_smem_bytes(int nmax);
int conv_f64_max_side(size_t smem_limit);
void launch_conv_f64(const ConvArgs& a, int grid, size_t smem, cudaStream_t s);

}  // namespace gg

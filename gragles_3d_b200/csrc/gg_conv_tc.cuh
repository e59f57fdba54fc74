// gg_conv_tc.cuh -- mixed-precision (FP32-storage) Gaussian convolution.
//
// The reference's multiplier G (box.cpp:760-761) is exp(-c (i2^2 + j2^2 + k2^2)) / n^3,
// a product of one factor per axis, so IDFT3(DFT3(in) G) equals three applications
// of one real symmetric circulant matrix C_n = F^-1 diag(g) F / n along x, y and z.
// The mixed path runs those three contractions as dense per-axis GEMMs.
#pragma once

#include <cuda_runtime.h>
#include <vector>

namespace gg {

struct ConvTCArgs {
    int G;
    const int* toff;          // one tile per convolved grain
    const float* in;
    const int* box;
    const long long* in_off;
    float* out;
    const long long* out_off;
    const float* circ;        // C_n row-major (n x n) for every side n at circ_off[n]
    const long long* circ_off;
    int* err;
};

// Append C_n (row-major, FP32) for box side n, domain size N and TimeStepSize.
void circulant_matrix(int n, int N, double time_step, std::vector<float>& out);

// toff holds n tiles per grain (z-planes, then y-rows).
void launch_conv_tc(const ConvTCArgs& a, int num_sms, int side_max, cudaStream_t s);

}  // namespace gg

// gg_conv_tc.cuh -- mixed-precision (FP32-storage) Gaussian convolution.
//
// The reference's multiplier G (box.cpp:760-761) is exp(-c (i2^2 + j2^2 + k2^2)) / n^3,
// a product of one factor per axis, so IDFT3(DFT3(in) G) equals three applications
// of one real symmetric circulant matrix C_n = F^-1 diag(g) F / n along x, y and z.
// The mixed path runs those three contractions as dense per-axis GEMMs.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
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

// ---- tcgen05 tensor-core path (gg_conv_umma.cu) ----
constexpr int kUmmaMaxSide = 64;  // largest box side of the tensor-core kernel (TMEM, shared memory)
constexpr int kUmmaRows = 128;    // box rows per MMA tile

// One rotating pass: dst[c'][a][b] = sum_c C_n[c'][c] src[a][b][c] for every box.
struct UmmaPassArgs {
    int G;
    const int* toff;          // ceil(n^2 / 128) row tiles per grain
    const int* box;           // 6 ints per grain, cubic
    const float* src;
    const long long* src_off;
    float* dst;
    const long long* dst_off;
    const uint16_t* bmat;     // 2^8 C_n split into FP16 hi and lo, MMA operand layout, per side
    const long long* boff;
    int side_max;             // largest side in the launch (sizes the shared memory)
    int* err;
};

// The three passes: in -> out -> scratch -> out (scratch shares out's offsets).
struct UmmaConvArgs {
    int G;
    const int* toff;
    const int* box;
    const float* in;
    const long long* in_off;
    float* out;
    const long long* out_off;
    float* scratch;
    const uint16_t* bmat;
    const long long* boff;
    int* err;
};

int umma_side_limit();
// True when the tensor-core kernel takes boxes up to side_max (else the SIMT kernels).
bool umma_supported(int side_max);
// C_n of every side 1..nmax as the MMA's B operand (hi block, then lo block).
void umma_tables(int N, double time_step, int nmax, std::vector<uint16_t>& bmat, std::vector<long long>& boff);
void launch_conv_umma(const UmmaConvArgs& a, int num_sms, int side_max, cudaStream_t s);

}  // namespace gg

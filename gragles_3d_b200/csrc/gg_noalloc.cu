// gg_noalloc.cu -- FP64 box convolution that allocates no device memory.
//
// gg_convolve_boxes_f64 allocates its half-spectrum scratch and its tables with
// cudaMalloc on every call.  Some callers cannot allocate device memory: a host
// program that hands all of the GPU's memory to its own pool allocator when it starts
// (so a cudaMalloc from a library would fail or take memory the pool counts on), or
// one that forbids allocation after start-up so that its memory footprint stays
// fixed.  gg_convolve_boxes_f64_noalloc computes exactly the same result with every
// buffer it needs -- the half-spectrum scratch, the DFT twiddles, the Gaussian table
// and the per-box metadata -- in file-scope __device__ arrays of fixed size (32 MiB of
// scratch plus under 2 MiB of tables, held by every GPU that loads the library until
// the process exits).  The caller still owns and passes the input and output boxes.
//
// Limits: at most kMaxBoxes boxes per call, sides up to kMaxSide, and
// sum over boxes of n*n*(n/2+1) <= kScratchComplex; larger requests are refused with
// GG_ERR_UNSUPPORTED before anything runs.  The first call on each device looks up
// the arrays' device addresses (cudaGetSymbolAddress) and uploads the twiddles.
//
// The call is synchronous: it copies the per-box metadata with cudaMemcpy from static
// host staging, launches on the legacy default stream and ends with
// cudaDeviceSynchronize, so it waits for all work on the device.  Because every call
// uses the same device arrays, calls from the threads of one process are serialised
// by a mutex held from the metadata upload until the device has finished; the arrays
// keep the last call's contents, and every buffer a call reads is rewritten by that
// call first.  (Other processes have their own contexts and so their own copies of
// the arrays.)
#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/gg_b200.h"
#include "gg_common.cuh"
#include "gg_conv.cuh"

namespace {

constexpr int kMaxBoxes = 256;
constexpr int kMaxSide = 96;
constexpr long long kScratchComplex = 1LL << 21;  // 2 Mi complex doubles = 32 MiB
constexpr int kMaxDevices = 64;

constexpr long long twiddle_count() {
    long long s = 0;
    for (int n = 1; n <= kMaxSide; n++) s += n;
    return s;
}
constexpr long long gauss_count() {
    long long s = 0;
    for (int n = 1; n <= kMaxSide; n++) s += 3LL * (n / 2) * (n / 2) + 1;
    return s;
}
constexpr long long kTw = twiddle_count();
constexpr long long kGauss = gauss_count();

// the scratch and everything else the kernels read, in fixed device storage
static __device__ __align__(256) double2 g_scratch[kScratchComplex];
static __device__ __align__(256) double2 g_tw[kTw];
static __device__ __align__(256) double g_gauss[kGauss];
static __device__ __align__(256) long long g_tw_off[kMaxSide + 2];
static __device__ __align__(256) long long g_g_off[kMaxSide + 2];
static __device__ __align__(256) int g_box[6 * (kMaxBoxes + 1)];
static __device__ __align__(256) long long g_off[kMaxBoxes + 1];
static __device__ __align__(256) long long g_spec_off[kMaxBoxes + 1];
static __device__ __align__(256) int g_toff[kMaxBoxes + 2];

struct DeviceState {
    bool ready = false;
    double2* scratch = nullptr;
    double2* tw = nullptr;
    double* gauss = nullptr;
    long long *tw_off = nullptr, *g_off = nullptr, *off = nullptr, *spec_off = nullptr;
    int *box = nullptr, *toff = nullptr;
    int gauss_N = -1;
    double gauss_ts = 0.0;
};

std::mutex g_mu;
DeviceState g_dev[kMaxDevices];

// host staging in static storage (no heap use on the call path)
double2 h_tw[kTw];
double h_gauss[kGauss];
long long h_tw_off[kMaxSide + 2], h_g_off[kMaxSide + 2];
int h_box[6 * (kMaxBoxes + 1)];
long long h_off[kMaxBoxes + 1], h_spec_off[kMaxBoxes + 1];
int h_toff[kMaxBoxes + 2];

// Once per device, with that device current: the arrays' device addresses and the
// twiddles (cos, sin)(2 pi j / n), angle (6.283185307179586 * j) / n.
int setup(DeviceState& d) {
    if (d.ready) return GG_OK;
    if (cudaGetSymbolAddress((void**)&d.scratch, g_scratch) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.tw, g_tw) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.gauss, g_gauss) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.tw_off, g_tw_off) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.g_off, g_g_off) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.box, g_box) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.off, g_off) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.spec_off, g_spec_off) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.toff, g_toff) != cudaSuccess)
        return GG_ERR_CUDA;
    long long k = 0, q = 0;
    for (int n = 1; n <= kMaxSide; n++) {
        h_tw_off[n] = k;
        for (int j = 0; j < n; j++, k++) {
            const double a = 6.283185307179586476925286766559 * (double)j / (double)n;
            h_tw[k] = make_double2(std::cos(a), std::sin(a));
        }
        h_g_off[n] = q;
        q += 3LL * (n / 2) * (n / 2) + 1;
    }
    if (cudaMemcpy(d.tw, h_tw, sizeof(h_tw), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d.tw_off, h_tw_off, sizeof(h_tw_off), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d.g_off, h_g_off, sizeof(h_g_off), cudaMemcpyHostToDevice) != cudaSuccess)
        return GG_ERR_CUDA;
    d.ready = true;
    return GG_OK;
}

// The Gaussian multiplier of box.cpp:760-761 for every side n <= kMaxSide and every
// S = i2^2 + j2^2 + k2^2, for this domain size and TimeStepSize.
int upload_gauss(DeviceState& d, int N, double time_step) {
    if (d.gauss_N == N && d.gauss_ts == time_step) return GG_OK;
    const double pi = 3.14159265358979323846;
    const double dt = time_step / double(N * N);
    const double nsq = N * N;
    long long q = 0;
    for (int n = 1; n <= kMaxSide; n++) {
        const double local_nsq = n * n;
        const int smax = 3 * (n / 2) * (n / 2);
        for (int S = 0; S <= smax; S++, q++)
            h_gauss[q] = std::exp(-std::sqrt(2 / pi) * S * 4.0 * dt * nsq / local_nsq * pi * pi) / (local_nsq * n);
    }
    if (cudaMemcpy(d.gauss, h_gauss, sizeof(h_gauss), cudaMemcpyHostToDevice) != cudaSuccess) return GG_ERR_CUDA;
    d.gauss_N = N;
    d.gauss_ts = time_step;
    return GG_OK;
}

}  // namespace

extern "C" int gg_convolve_boxes_f64_noalloc(const double* d_in, double* d_out, const int32_t* sides,
                                             const int64_t* offs, int32_t n_boxes, int32_t domain_size,
                                             double time_step) {
    if (!d_in || !d_out || !sides || !offs || domain_size < 1 || !(time_step > 0)) return GG_ERR_INVALID;
    if (n_boxes < 1 || n_boxes > kMaxBoxes) return GG_ERR_UNSUPPORTED;
    long long spec_total = 0;
    int nmax = 0;
    for (int b = 0; b < n_boxes; b++) {
        const int n = sides[b];
        if (n < 1 || n > kMaxSide || offs[b] < 0) return GG_ERR_UNSUPPORTED;
        nmax = n > nmax ? n : nmax;
        spec_total += (long long)n * n * (n / 2 + 1);
    }
    if (spec_total > kScratchComplex) return GG_ERR_UNSUPPORTED;
    int dev = 0, optin = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GG_ERR_CUDA;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = gg::conv_f64_smem_bytes(nmax);
    if (smem > (size_t)optin) return GG_ERR_UNSUPPORTED;

    std::lock_guard<std::mutex> lock(g_mu);
    DeviceState& d = g_dev[dev];
    int rc = setup(d);
    if (rc) return rc;
    rc = upload_gauss(d, domain_size, time_step);
    if (rc) return rc;
    // boxes 1..n_boxes at (0, n, 0, n, 0, n); entry 0 unused
    long long sp = 0;
    h_toff[0] = h_toff[1] = 0;
    for (int q = 0; q < 6; q++) h_box[q] = 0;
    h_off[0] = h_spec_off[0] = 0;
    for (int b = 0; b < n_boxes; b++) {
        const int n = sides[b];
        int* bb = h_box + 6 * (b + 1);
        bb[0] = 0; bb[1] = n; bb[2] = 0; bb[3] = n; bb[4] = 0; bb[5] = n;
        h_off[b + 1] = offs[b];
        h_spec_off[b + 1] = sp;
        sp += (long long)n * n * (n / 2 + 1);
        h_toff[b + 2] = h_toff[b + 1] + n;
    }
    if (cudaMemcpy(d.box, h_box, sizeof(int) * 6 * (n_boxes + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d.off, h_off, sizeof(long long) * (n_boxes + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d.spec_off, h_spec_off, sizeof(long long) * (n_boxes + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d.toff, h_toff, sizeof(int) * (n_boxes + 2), cudaMemcpyHostToDevice) != cudaSuccess)
        return GG_ERR_CUDA;
    gg::ConvArgs a{};
    a.G = n_boxes;
    a.toff = d.toff;
    a.in = d_in;
    a.in_box = d.box;
    a.in_off = d.off;
    a.out = d_out;
    a.out_off = d.off;
    a.spec = d.scratch;
    a.spec_off = d.spec_off;
    a.tw = d.tw;
    a.tw_off = d.tw_off;
    a.gtab = d.gauss;
    a.g_off = d.g_off;
    // an error left over from earlier, unrelated work is not this launch's: clear it
    // first (a sticky error has already failed the copies above)
    (void)cudaGetLastError();
    gg::launch_conv_f64(a, (sms > 0 ? sms : 148) * 8, smem, 0);
    if (cudaGetLastError() != cudaSuccess) return GG_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return GG_ERR_CUDA;
    return GG_OK;
}

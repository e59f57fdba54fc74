// gg_init.cu -- the initial distance field of every grain box.
//
// Stands in for LSbox::calculateDistanceFunction (box.cpp:374-397): inside the
// domain the SDF is +h where the voxel belongs to the grain and -h elsewhere, and
// -h on the border layer of width grid_blowup.  The labels are the mode-4 voxel
// container without its border (grainhdl.cpp:534-557).  The redistancing that
// follows is the regular redistancing kernel.
#include "gg_kernels.cuh"

namespace gg {

namespace {

template <typename T>
__global__ void init_sdf_kernel(InitArgs<T> a) {
    const int total = a.toff[a.G + 1];
    const int gb = a.geo.gb, M = a.geo.M, N = a.geo.N;
    const T h = (T)a.geo.h;
    const int lo = gb, hi = M - gb - 1;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const Box b = a.dst.grain_box(g);
        const int k = b.z0 + (t - a.toff[g]);
        T* dst = a.dst.grain_ptr(g) + (long long)(k - b.z0) * b.nx() * b.ny();
        for (int q = threadIdx.x; q < b.nx() * b.ny(); q += blockDim.x) {
            const int i = b.y0 + q / b.nx(), j = b.x0 + q % b.nx();
            T v;
            if (i < lo || i > hi || j < lo || j > hi || k < lo || k > hi) {
                v = -h;
            } else {
                const uint32_t lab = a.labels[((long long)(k - gb) * N + (i - gb)) * N + (j - gb)];
                v = (lab == (uint32_t)g) ? h : -h;
            }
            dst[q] = v;
        }
    }
}

}  // namespace

template <typename T>
void launch_init_sdf(const InitArgs<T>& a, int grid, cudaStream_t s) {
    init_sdf_kernel<T><<<grid, 256, 0, s>>>(a);
}

template void launch_init_sdf<double>(const InitArgs<double>&, int, cudaStream_t);
template void launch_init_sdf<float>(const InitArgs<float>&, int, cudaStream_t);

}  // namespace gg

// gg_init.cu -- the initial distance field of every grain box.
//
// Stands in for LSbox::calculateDistanceFunction (box.cpp:374-397): inside the
// domain the SDF is +h where the voxel belongs to the grain and -h elsewhere, and
// -h on the border layer of width grid_blowup.  The labels are the mode-4 voxel
// container without its border (grainhdl.cpp:534-557).  The redistancing that
// follows is the regular redistancing kernel.
//
// The inverse map is here too: the voxel container of the current network
// (LSbox::copyDataToContainer, box.cpp:3008-3032, as grainhdl::saveNetworkAsVoxelContainer
// calls it, grainhdl.cpp:1074-1095): every voxel of the domain where a grain's current
// SDF is >= 0 gets the grain's ID.  The reference visits the grains in ascending ID order
// (one thread), so the last writer -- the largest such ID -- stays: an atomicMax.
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

template <typename T>
__global__ void container_kernel(ContainerArgs<T> a) {
    const int total = a.toff[a.G + 1];
    const int gb = a.geo.gb, N = a.geo.N;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const Box b = a.src.grain_box(g);
        const int k = b.z0 + (t - a.toff[g]);
        if (k < gb || k >= N + gb) continue;
        const T* src = a.src.grain_ptr(g) + (long long)(k - b.z0) * b.nx() * b.ny();
        for (int q = threadIdx.x; q < b.nx() * b.ny(); q += blockDim.x) {
            const int i = b.y0 + q / b.nx(), j = b.x0 + q % b.nx();
            if (i < gb || j < gb || i >= N + gb || j >= N + gb) continue;
            if (T(0) <= src[q])
                atomicMax(a.labels + ((long long)(k - gb) * N + (i - gb)) * N + (j - gb), (unsigned)g);
        }
    }
}

}  // namespace

template <typename T>
void launch_container(const ContainerArgs<T>& a, int grid, cudaStream_t s) {
    container_kernel<T><<<grid, 256, 0, s>>>(a);
}

template void launch_container<double>(const ContainerArgs<double>&, int, cudaStream_t);
template void launch_container<float>(const ContainerArgs<float>&, int, cudaStream_t);

template <typename T>
void launch_init_sdf(const InitArgs<T>& a, int grid, cudaStream_t s) {
    init_sdf_kernel<T><<<grid, 256, 0, s>>>(a);
}

template void launch_init_sdf<double>(const InitArgs<double>&, int, cudaStream_t);
template void launch_init_sdf<float>(const InitArgs<float>&, int, cudaStream_t);

}  // namespace gg

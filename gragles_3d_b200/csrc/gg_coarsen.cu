// gg_coarsen.cu -- grid coarsening of every grain box on the device.
//
// Stands in for the per-grain work of grainhdl::gridCoarsement (grainhdl.cpp:1446-1498):
// LSbox::resizeGrid (box.cpp:2595-2694) re-samples each grain's output distance field
// from the old grid onto the new, coarser one by trilinear interpolation into its input
// buffer, on a box that is the old box scaled by h_old / h_new and resized to a cube.
// The host (gg_api.cu) decides when to coarsen, updates the geometry and tables, then
// runs recalculateIDLocal (a comparison without the set comparison) and extractContour
// (marching cubes) with the existing stage kernels.
//
//   regrid_box_kernel: one thread per grain, the new box (integer truncation of the
//     scaled corners, exactly as the reference's int assignments).
//   resample_kernel:   a CTA per (grain, new z-slice); every voxel's value is the
//     reference's trilinear expression, term by term and in its order (no contraction),
//     so the FP64 path stays bit-identical; voxels whose stencil leaves the old box get
//     -delta of the new grid.
//   id_resize_kernel:  IDLocal of grains that skip executeComparison (box.cpp:892-893:
//     not existing), flat-resized onto the new box (dimensionalBuffer.h:120-131), since
//     extractContour reads it.
#include "gg_kernels.cuh"

namespace gg {

namespace {

__global__ void regrid_box_kernel(RegridBoxArgs a) {
    for (int g = 1 + blockIdx.x * blockDim.x + threadIdx.x; g <= a.G; g += gridDim.x * blockDim.x) {
        if (!a.present[g]) continue;
        const Box o = load_box(a.old_box + 6 * g);
        const int gb = a.gb;
        // m_newXMin = (getMinX() - grid_blowup) * (h / hn) + 0.5 + grid_blowup, stored in an int
        const int x0 = (int)((o.x0 - gb) * a.ratio + 0.5 + gb), x1 = (int)((o.x1 - gb) * a.ratio + 0.5 + gb);
        const int y0 = (int)((o.y0 - gb) * a.ratio + 0.5 + gb), y1 = (int)((o.y1 - gb) * a.ratio + 0.5 + gb);
        const int z0 = (int)((o.z0 - gb) * a.ratio + 0.5 + gb), z1 = (int)((o.z1 - gb) * a.ratio + 0.5 + gb);
        const Box s{x0, x1, y0, y1, z0, z1};
        store_box(a.scaled + 6 * g, s);
        // m_inputDistance->resize(...) then resizeToCube(ngridpointsNew)
        const Box c = resize_to_cube(s, a.M_new);
        if (c.nx() <= 0 || c.nx() != c.ny() || c.nx() != c.nz() || c.x0 < 0 || c.y0 < 0 || c.z0 < 0 ||
            c.x1 > a.M_new || c.y1 > a.M_new || c.z1 > a.M_new)
            atomicOr(a.err, ERR_BOX);
        store_box(a.new_box + 6 * g, c);
    }
}

// The old output value at absolute (row i, column j, depth k) of the old grid.
template <typename T>
__device__ __forceinline__ double old_at(const T* src, const Box& ob, int i, int j, int k) {
    return (double)src[ob.at(i, j, k)];
}

template <typename T>
__global__ void __launch_bounds__(256) resample_kernel(ResampleArgs<T> a) {
    const int gb = a.gb;
    const double r = a.ratio_inv;  // hn / h
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box nb = a.dst.grain_box(g);
        const Box ob = a.src.grain_box(g);
        const T* src = a.src.grain_ptr(g);
        T* dst = a.dst.grain_ptr(g);
        const int k = nb.z0 + w.local;
        const int nx = nb.nx(), ny = nb.ny();
        for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {
            const int i = nb.y0 + q / nx, j = nb.x0 + q % nx;
            const double pointx = (j - gb) * r;
            const double pointy = (i - gb) * r;
            const double pointz = (k - gb) * r;
            const double xl = floor(pointx), xr = floor(pointx + 1);
            const double yu = floor(pointy), yo = floor(pointy + 1);
            const double zu = floor(pointz), zo = floor(pointz + 1);
            double v;
            if (xr + gb > ob.x1 - 2 || yo + gb > ob.y1 - 2 || zo + gb > ob.z1 - 2 || yu + gb < ob.y0 ||
                xl + gb < ob.x0 || zu + gb < ob.z0) {
                v = -a.delta_new;
            } else {
                const int ixl = (int)(xl + gb), ixr = (int)(xr + gb);
                const int iyu = (int)(yu + gb), iyo = (int)(yo + gb);
                const int izu = (int)(zu + gb), izo = (int)(zo + gb);
                // bilinear interpolation in the plane zu, then zo, then along z (box.cpp:2655-2689)
                double ro = (xr - pointx) * old_at(src, ob, iyo, ixl, izu) + (pointx - xl) * old_at(src, ob, iyo, ixr, izu);
                double ru = (xr - pointx) * old_at(src, ob, iyu, ixl, izu) + (pointx - xl) * old_at(src, ob, iyu, ixr, izu);
                const double zu_val = (yo - pointy) * ru + (pointy - yu) * ro;
                ro = (xr - pointx) * old_at(src, ob, iyo, ixl, izo) + (pointx - xl) * old_at(src, ob, iyo, ixr, izo);
                ru = (xr - pointx) * old_at(src, ob, iyu, ixl, izo) + (pointx - xl) * old_at(src, ob, iyu, ixr, izo);
                const double zo_val = (yo - pointy) * ru + (pointy - yu) * ro;
                v = (zo - pointz) * zu_val + (pointz - zu) * zo_val;
            }
            dst[nb.at(i, j, k)] = (T)v;
        }
    }
}

__global__ void id_resize_kernel(IdResizeArgs a) {
    for (int g = 1 + blockIdx.x; g <= a.G; g += gridDim.x) {
        if (!a.present[g] || a.exists[g]) continue;
        const long long n_new = load_box(a.idbox_new + 6 * g).count();
        const long long n_old = load_box(a.idbox_old + 6 * g).count();
        const uint32_t* src = a.id_old + a.idoff_old[g];
        uint32_t* dst = a.id_new + a.idoff_new[g];
        for (long long f = threadIdx.x; f < n_new; f += blockDim.x) dst[f] = f < n_old ? src[f] : 0u;
    }
}

}  // namespace

void launch_regrid_boxes(const RegridBoxArgs& a, cudaStream_t s) {
    regrid_box_kernel<<<(a.G + 256) / 256, 256, 0, s>>>(a);
}

template <typename T>
void launch_resample(const ResampleArgs<T>& a, int grid, cudaStream_t s) {
    resample_kernel<T><<<grid, 256, 0, s>>>(a);
}

void launch_id_resize(const IdResizeArgs& a, int grid, cudaStream_t s) { id_resize_kernel<<<grid, 256, 0, s>>>(a); }

template void launch_resample<double>(const ResampleArgs<double>&, int, cudaStream_t);
template void launch_resample<float>(const ResampleArgs<float>&, int, cudaStream_t);

}  // namespace gg

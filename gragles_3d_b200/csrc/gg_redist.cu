// gg_redist.cu -- directional-sweep redistancing of every grain.
//
// Stands in for LSbox::executeRedistancing (box.cpp:2322-2586).  The reference
// clears the new (resized) output box to -1, then for every z-slice of the in/out
// intersection except the last runs four sweeps (x forward, x backward, y forward,
// y backward), then sweeps z forward and backward over all columns, and clamps to
// +-delta.  Every sweep is a recurrence along one line and the lines of a sweep are
// independent, so:
//   kernel xy: one CTA per (grain, output z-slice); the slice sits in shared
//              memory and each thread runs one line of a sweep;
//   kernel z:  one CTA per (grain, output y-row); each thread runs the z
//              recurrences of one column (x-adjacent threads read adjacent words).
// Arithmetic is the reference's, statement by statement (no contraction), so the
// FP64 result is bit-identical.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr int kThreadsXY = 128;
constexpr int kThreadsZ = 128;

template <typename T>
struct Intersect {
    int xmin, xmax, ymin, ymax, zmin, zmax;
    __device__ Intersect(const Box& ib, const Box& ob) {
        xmin = ib.x0 < ob.x0 ? ob.x0 : ib.x0;
        ymin = ib.y0 < ob.y0 ? ob.y0 : ib.y0;
        zmin = ib.z0 < ob.z0 ? ob.z0 : ib.z0;
        xmax = ib.x1 < ob.x1 ? ib.x1 : ob.x1;
        ymax = ib.y1 < ob.y1 ? ib.y1 : ob.y1;
        zmax = ib.z1 < ob.z1 ? ib.z1 : ob.z1;
    }
};

// The interpolation step at a sign change between a (here) and b (next), then the
// candidate propagated to next; box.cpp:2370-2391 and the y/z twins.
template <typename T>
__device__ __forceinline__ void step_in(T a, T b, T& out_here, T& out_next, T h) {
    if (a * b <= T(0)) {
        const T i_slope = (b - a) / h;
        const T distToZero = -a / i_slope;
        if (fabs(out_here) > fabs(distToZero)) out_here = -distToZero * isgn(i_slope);
    }
    const T candidate = out_here + (isgn(b) * h);
    if (fabs(candidate) < fabs(out_next)) out_next = candidate;
}
template <typename T>
__device__ __forceinline__ void step_prop(T sgn_src, T out_here, T& out_next, T h) {
    const T candidate = out_here + (isgn(sgn_src) * h);
    if (fabs(candidate) < fabs(out_next)) out_next = candidate;
}

template <typename T>
__global__ void __launch_bounds__(kThreadsXY) redist_xy_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* S = reinterpret_cast<T*>(smem_raw);
    const T h = (T)a.geo.h;
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int k = ob.z0 + (t - a.toff[g]);
        const Intersect<T> I(ib, ob);
        const int nx = ob.nx(), ny = ob.ny();
        T* outg = a.out.grain_ptr(g) + (long long)(k - ob.z0) * nx * ny;
        if (!(k >= I.zmin && k < I.zmax - 1)) {  // no xy sweep reaches this slice
            for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) outg[q] = T(-1);
            continue;
        }
        const int P = nx | 1;
        T* O = S;                  // out slice, [y][x] with pitch P
        T* In = S + ny * P;        // in values on the intersection, same indexing
        const T* ing = a.in.grain_ptr(g);
        for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {
            const int yy = q / nx, xx = q - yy * nx;
            O[yy * P + xx] = T(-1);
            const int i = ob.y0 + yy, j = ob.x0 + xx;
            if (i >= I.ymin && i < I.ymax && j >= I.xmin && j < I.xmax) In[yy * P + xx] = ing[ib.at(i, j, k)];
        }
        __syncthreads();
#define OUT(i, j) O[((i) - ob.y0) * P + ((j) - ob.x0)]
#define IN(i, j) In[((i) - ob.y0) * P + ((j) - ob.x0)]
        // x forward, box.cpp:2367-2401
        for (int i = I.ymin + threadIdx.x; i < ob.y1; i += blockDim.x) {
            for (int j = I.xmin; j < ob.x1 - 1; j++) {
                if (j < I.xmax - 1 && i < I.ymax) step_in(IN(i, j), IN(i, j + 1), OUT(i, j), OUT(i, j + 1), h);
                else step_prop(OUT(i, j + 1), OUT(i, j), OUT(i, j + 1), h);
            }
        }
        __syncthreads();
        // x backward, box.cpp:2403-2435
        for (int i = I.ymin + threadIdx.x; i < ob.y1; i += blockDim.x) {
            for (int j = I.xmax - 1; j > ob.x0; j--) {
                if (j > I.xmin && i < I.ymax) step_prop(IN(i, j - 1), OUT(i, j), OUT(i, j - 1), h);
                else step_prop(OUT(i, j - 1), OUT(i, j), OUT(i, j - 1), h);
            }
        }
        __syncthreads();
        // y forward, box.cpp:2437-2472
        for (int j = I.xmin + threadIdx.x; j < ob.x1; j += blockDim.x) {
            for (int i = I.ymin; i < ob.y1 - 1; i++) {
                if (j < I.xmax && i < I.ymax - 1) step_in(IN(i, j), IN(i + 1, j), OUT(i, j), OUT(i + 1, j), h);
                else step_prop(OUT(i + 1, j), OUT(i, j), OUT(i + 1, j), h);
            }
        }
        __syncthreads();
        // y backward, box.cpp:2474-2496
        for (int j = I.xmin + threadIdx.x; j < ob.x1; j += blockDim.x) {
            for (int i = I.ymax - 1; i > ob.y0; i--) {
                if (j < I.xmax && i > I.ymin) step_prop(IN(i - 1, j), OUT(i, j), OUT(i - 1, j), h);
                else step_prop(OUT(i - 1, j), OUT(i, j), OUT(i - 1, j), h);
            }
        }
        __syncthreads();
#undef OUT
#undef IN
        for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {
            const int yy = q / nx, xx = q - yy * nx;
            outg[q] = O[yy * P + xx];
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreadsZ) redist_z_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* S = reinterpret_cast<T*>(smem_raw);
    const T h = (T)a.geo.h;
    const T delta = (T)a.geo.delta;
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int i = ob.y0 + (t - a.toff[g]);
        const Intersect<T> I(ib, ob);
        const int nx = ob.nx(), nz = ob.nz();
        T* O = S;              // [k][x] of this row
        T* In = S + nz * nx;   // in values, same indexing
        T* outg = a.out.grain_ptr(g);
        const T* ing = a.in.grain_ptr(g);
        for (int q = threadIdx.x; q < nx * nz; q += blockDim.x) {
            const int kk = q / nx, xx = q - kk * nx;
            const int k = ob.z0 + kk, j = ob.x0 + xx;
            O[q] = outg[ob.at(i, j, k)];
            if (i >= I.ymin && i < I.ymax && j >= I.xmin && j < I.xmax && k >= I.zmin && k < I.zmax)
                In[q] = ing[ib.at(i, j, k)];
        }
        __syncthreads();
#define OUT(k, j) O[((k) - ob.z0) * nx + ((j) - ob.x0)]
#define IN(k, j) In[((k) - ob.z0) * nx + ((j) - ob.x0)]
        if (i >= I.ymin) {
            for (int j = I.xmin + threadIdx.x; j < ob.x1; j += blockDim.x) {
                // z forward, box.cpp:2501-2538
                for (int k = I.zmin; k < ob.z1 - 1; k++) {
                    if (k < I.zmax - 1 && i < I.ymax && j < I.xmax) step_in(IN(k, j), IN(k + 1, j), OUT(k, j), OUT(k + 1, j), h);
                    else step_prop(OUT(k + 1, j), OUT(k, j), OUT(k + 1, j), h);
                }
                // z backward, box.cpp:2539-2576
                for (int k = I.zmax - 1; k > ob.z0; k--) {
                    if (k > I.zmin && i < I.ymax && j < I.xmax) step_in(IN(k, j), IN(k - 1, j), OUT(k, j), OUT(k - 1, j), h);
                    else step_prop(OUT(k - 1, j), OUT(k, j), OUT(k - 1, j), h);
                }
            }
        }
        __syncthreads();
#undef OUT
#undef IN
        // clampValues(-delta, delta), dimensionalBufferReal.h:44-57
        for (int q = threadIdx.x; q < nx * nz; q += blockDim.x) {
            const int kk = q / nx, xx = q - kk * nx;
            T v = O[q];
            if (v < -delta) v = -delta;
            else if (v > delta) v = delta;
            outg[ob.at(i, ob.x0 + xx, ob.z0 + kk)] = v;
        }
        __syncthreads();
    }
}

}  // namespace

size_t redist_smem_bytes(int nmax, bool fp64) {
    const size_t e = fp64 ? 8 : 4;
    const size_t xy = 2 * (size_t)nmax * (nmax | 1) * e;
    const size_t z = 2 * (size_t)nmax * nmax * e;
    return xy > z ? xy : z;
}

template <typename T>
void launch_redistance(const RedistArgs<T>& a, int grid, size_t smem_xy, size_t smem_z, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        allow_max_dynamic_smem(redist_xy_kernel<T>);
        allow_max_dynamic_smem(redist_z_kernel<T>);
        configured = true;
    }
    redist_xy_kernel<T><<<grid, kThreadsXY, smem_xy, s>>>(a);
    redist_z_kernel<T><<<grid, kThreadsZ, smem_z, s>>>(a);
}

template void launch_redistance<double>(const RedistArgs<double>&, int, size_t, size_t, cudaStream_t);
template void launch_redistance<float>(const RedistArgs<float>&, int, size_t, size_t, cudaStream_t);

}  // namespace gg

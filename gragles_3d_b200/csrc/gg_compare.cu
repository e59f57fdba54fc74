// gg_compare.cu -- comparison, boundary condition and set-comparison of every grain.
//
// Stands in for LSbox::executeComparison (box.cpp:891-966), boundaryCondition
// (box.cpp:997-1088) and executeSetComparison (box.cpp:814-878), fused in one
// pass over each box.
//
// The reference walks the comparison list in order and keeps, per voxel, the
// first neighbour whose SDF is strictly greater than everything before it
// (starting from -1).  That is the maximum value with ties going to the earliest
// list position, an order-free reduction, so the warps of a tile take
// neighbours in any order: pass 1 folds each neighbour value into a per-voxel
// shared-memory atomicMax, pass 2 (FP64) keeps the smallest list position that
// attains it.  On the FP32 path value and position pack into one 64-bit key and
// one pass suffices.  The winner's value is re-read for the output, so the result
// is bit-identical to the sequential walk.  Voxels no neighbour covers keep their
// IDLocal from the previous layout by the reference's flat-prefix resize
// (dimensionalBuffer.h:120-131).
#include "gg_kernels.cuh"

#include <climits>

namespace gg {

namespace {

constexpr unsigned kNone = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned long long ord64(double v) {
    const long long b = __double_as_longlong(v == 0.0 ? 0.0 : v);  // -0 and +0 compare equal
    return b >= 0 ? ((unsigned long long)b ^ 0x8000000000000000ull) : ~(unsigned long long)b;
}
__device__ __forceinline__ unsigned ord32(float v) {
    const int b = __float_as_int(v == 0.0f ? 0.0f : v);
    return b >= 0 ? ((unsigned)b ^ 0x80000000u) : ~(unsigned)b;
}

// One branch of the reference's boundary distance (box.cpp:1017-1082).  Returns
// false where no branch assigns `dist`, in which case the reference keeps the value
// of the previous voxel in its loop order.
__device__ bool bc_assign(int i, int j, int k, int m, int gb, double& dist) {
    const double distXMax = (j - (m - 1 - gb));
    const double distYMax = (i - (m - 1 - gb));
    const double distZMax = (k - (m - 1 - gb));
    const double distXMin = -(j - gb + 1);
    const double distYMin = -(i - gb + 1);
    const double distZMin = -(k - gb + 1);
    const double distX = fabs(distXMin) < fabs(distXMax) ? distXMin : distXMax;
    const double distY = fabs(distYMin) < fabs(distYMax) ? distYMin : distYMax;
    const double distZ = fabs(distZMin) < fabs(distZMax) ? distZMin : distZMax;
    if (distX > 0 && distY > 0 && distZ > 0) {
        dist = sqrt((double)distX * distX + distY * distY + distZ * distZ);
        return true;
    }
    if (distX < 0 && distY < 0 && distZ < 0) {
        double d = distX < distY ? distY : distX;
        dist = d < distZ ? distZ : d;
        return true;
    }
    if (distX >= 0) {
        if (distY < 0 && distZ < 0) { dist = distX; return true; }
        if (distY < 0 && distZ >= 0) { dist = sqrt((double)distX * distX + distZ * distZ); return true; }
        if (distY >= 0 && distZ < 0) { dist = sqrt((double)distX * distX + distY * distY); return true; }
        return false;
    }
    if (distY >= 0) {
        if (distZ < 0 && distX < 0) { dist = distY; return true; }
        if (distX < 0 && distZ >= 0) { dist = sqrt((double)distY * distY + distZ * distZ); return true; }
        return false;
    }
    if (distZ >= 0) {
        if (distY < 0 && distX < 0) { dist = distZ; return true; }
        return false;
    }
    return false;
}

// The value `dist` holds at voxel (i, j, k) of the boundary loop over box b.
__device__ double bc_dist(const Box& b, int i, int j, int k, int m, int gb) {
    double d;
    if (bc_assign(i, j, k, m, gb, d)) return d;
    int ii = i, jj = j, kk = k;
    for (;;) {
        if (--jj < b.x0) {
            jj = b.x1 - 1;
            if (--ii < b.y0) {
                ii = b.y1 - 1;
                if (--kk < b.z0) return 0.0;  // initial value, box.cpp:1001
            }
        }
        if (bc_assign(ii, jj, kk, m, gb, d)) return d;
    }
}

// Iterate the voxels of intersection `I` with one warp: lanes cover x, several
// rows per pass when the row is short.
template <typename F>
__device__ __forceinline__ void warp_foreach(int ix0, int ix1, int iy0, int iy1, int iz0, int iz1, F&& f) {
    const int lane = threadIdx.x & 31;
    const int wx = ix1 - ix0, wy = iy1 - iy0, rows = wy * (iz1 - iz0);
    const int lpr = wx <= 1 ? 1 : wx <= 2 ? 2 : wx <= 4 ? 4 : wx <= 8 ? 8 : wx <= 16 ? 16 : 32;
    const int rpi = 32 / lpr;
    const int sub = lane & (lpr - 1), rsub = lane / lpr;
    for (int r = rsub; r < rows; r += rpi) {
        const int zz = r / wy;
        const int y = iy0 + (r - zz * wy), z = iz0 + zz;
        for (int x = ix0 + sub; x < ix1; x += lpr) f(x, y, z);
    }
}

template <typename T>
__global__ void __launch_bounds__(512) compare_kernel(CompareArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* key = reinterpret_cast<unsigned long long*>(smem_raw);
    const bool fp64 = sizeof(T) == 8;
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int s = t - a.toff[g];
        const Box A = a.in.grain_box(g);
        const int sz0 = A.z0 + s * a.slab, sz1 = min(A.z1, sz0 + a.slab);
        const int nx = A.nx(), ny = A.ny();
        const int V = nx * ny * (sz1 - sz0);
        unsigned* pos = reinterpret_cast<unsigned*>(key + V);
        const unsigned long long init = fp64 ? ord64(-1.0) : ((unsigned long long)ord32(-1.0f) << 32);
        for (int l = threadIdx.x; l < V; l += blockDim.x) {
            key[l] = init;
            if (fp64) pos[l] = kNone;
        }
        const uint32_t* list = a.cmp + (long long)g * a.list_cap;
        const int K = a.n_cmp[g];
        if (s == 0) {  // m_secondOrderNeighbours = m_comparisonList, box.cpp:895
            uint32_t* son = a.son + (long long)g * a.list_cap;
            for (int q = threadIdx.x; q < K; q += blockDim.x) son[q] = list[q];
            if (threadIdx.x == 0) a.n_son[g] = K;
        }
        __syncthreads();
        const int passes = fp64 ? 2 : 1;
        for (int pass = 0; pass < passes; pass++) {
            for (int p = warp; p < K; p += nw) {
                const int nbid = list[p];
                const Box B = a.in.grain_box(nbid);
                const int ix0 = max(A.x0, B.x0), ix1 = min(A.x1, B.x1);
                const int iy0 = max(A.y0, B.y0), iy1 = min(A.y1, B.y1);
                const int iz0 = max(sz0, B.z0), iz1 = min(sz1, B.z1);
                if (ix0 >= ix1 || iy0 >= iy1 || iz0 >= iz1) continue;
                const T* bin = a.in.grain_ptr(nbid);
                warp_foreach(ix0, ix1, iy0, iy1, iz0, iz1, [&](int x, int y, int z) {
                    const T v = bin[B.at(y, x, z)];
                    if (!(v > T(-1))) return;
                    const int l = ((z - sz0) * ny + (y - A.y0)) * nx + (x - A.x0);
                    if (fp64) {
                        const unsigned long long kv = ord64((double)v);
                        if (pass == 0) atomicMax(key + l, kv);
                        else if (kv == key[l]) atomicMin(pos + l, (unsigned)p);
                    } else {
                        const unsigned long long kv =
                            ((unsigned long long)ord32((float)v) << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned)p);
                        atomicMax(key + l, kv);
                    }
                });
            }
            __syncthreads();
        }
        // epilogue: boundary condition, set comparison, outputs, new bbox
        const bool boundary = !(A.x0 > a.geo.gb && A.x1 < a.geo.M - a.geo.gb && A.y0 > a.geo.gb &&
                                A.y1 < a.geo.M - a.geo.gb && A.z0 > a.geo.gb && A.z1 < a.geo.M - a.geo.gb);
        const Box Bold = load_box(a.idbox_old + 6 * g);
        const long long old_count = Bold.count();
        const uint32_t* idold = a.id_old + a.idoff_old[g];
        uint32_t* idnew = a.id_new + a.idoff_new[g];
        const T* self = a.in.grain_ptr(g);
        T* outp = a.out.grain_ptr(g);
        const double lim = 0.7 * a.geo.delta;
        int bx0 = INT_MAX, bx1 = INT_MIN, by0 = INT_MAX, by1 = INT_MIN, bz0 = INT_MAX, bz1 = INT_MIN;
        const long long base = (long long)(sz0 - A.z0) * nx * ny;
        for (int l = threadIdx.x; l < V; l += blockDim.x) {
            const int x = A.x0 + l % nx;
            const int y = A.y0 + (l / nx) % ny;
            const int z = sz0 + l / (nx * ny);
            const long long f = base + l;
            int p;
            if (fp64) {
                p = pos[l] == kNone ? -1 : (int)pos[l];
            } else {
                const unsigned low = (unsigned)(key[l] & 0xFFFFFFFFull);
                p = low == 0 ? -1 : (int)(0xFFFFFFFFu - low);
            }
            T cmpv;
            uint32_t id;
            if (p >= 0) {
                id = list[p];
                const Box B = a.in.grain_box(id);
                cmpv = a.in.grain_ptr(id)[B.at(y, x, z)];
            } else {
                cmpv = T(-1);
                id = f < old_count ? idold[f] : 0u;
            }
            if (boundary) {
                const double d = bc_dist(A, y, x, z, a.geo.M, a.geo.gb);
                if (d > -a.geo.gb)
                    if (d * a.geo.h > (double)cmpv) {
                        cmpv = (T)(d * a.geo.h);
                        id = 0;
                    }
            }
            const T in = self[f];
            T res;
            if ((double)fabs(in) < lim) res = T(0.5) * (in - cmpv);
            else res = in;
            outp[f] = res;
            idnew[f] = id;
            if (res >= 0) {
                bx0 = min(bx0, x); bx1 = max(bx1, x);
                by0 = min(by0, y); by1 = max(by1, y);
                bz0 = min(bz0, z); bz1 = max(bz1, z);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bx0 = min(bx0, __shfl_xor_sync(0xffffffffu, bx0, o));
            bx1 = max(bx1, __shfl_xor_sync(0xffffffffu, bx1, o));
            by0 = min(by0, __shfl_xor_sync(0xffffffffu, by0, o));
            by1 = max(by1, __shfl_xor_sync(0xffffffffu, by1, o));
            bz0 = min(bz0, __shfl_xor_sync(0xffffffffu, bz0, o));
            bz1 = max(bz1, __shfl_xor_sync(0xffffffffu, bz1, o));
        }
        if ((threadIdx.x & 31) == 0 && bx0 != INT_MAX) {
            int* nb = a.newbox + 6 * g;
            atomicMin(nb + 0, bx0); atomicMax(nb + 1, bx1);
            atomicMin(nb + 2, by0); atomicMax(nb + 3, by1);
            atomicMin(nb + 4, bz0); atomicMax(nb + 5, bz1);
        }
        __syncthreads();
    }
}

__global__ void newbox_init_kernel(int G, const int* present, const int* exists, const int* box, int* newbox) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        if (g == 0 || !present[g] || !exists[g]) continue;
        const Box b = load_box(box + 6 * g);
        // executeSetComparison starts from the inverted out box, box.cpp:815-820
        int* nb = newbox + 6 * g;
        nb[0] = b.x1; nb[1] = b.x0; nb[2] = b.y1; nb[3] = b.y0; nb[4] = b.z1; nb[5] = b.z0;
    }
}

}  // namespace

size_t compare_smem_bytes(int nmax, int slab, bool fp64) {
    const size_t V = (size_t)nmax * nmax * slab;
    return V * 8 + (fp64 ? V * 4 : 0);
}

template <typename T>
void launch_compare(const CompareArgs<T>& a, int grid, size_t smem, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        allow_max_dynamic_smem(compare_kernel<T>);
        configured = true;
    }
    compare_kernel<T><<<grid, 512, smem, s>>>(a);
}

void launch_newbox_init(int G, const int* present, const int* exists, const int* box, int* newbox, cudaStream_t s) {
    newbox_init_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, present, exists, box, newbox);
}

template void launch_compare<double>(const CompareArgs<double>&, int, size_t, cudaStream_t);
template void launch_compare<float>(const CompareArgs<float>&, int, size_t, cudaStream_t);

}  // namespace gg

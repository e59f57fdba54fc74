// gg_compare.cu -- comparison, boundary condition and set-comparison of every grain.
//
// Stands in for LSbox::executeComparison (box.cpp:891-966), boundaryCondition
// (box.cpp:997-1088) and executeSetComparison (box.cpp:814-878), fused in one
// pass over each box.
//
// Work decomposition: a CTA takes one (grain, slab of z-planes) tile and keeps the
// slab's running maximum and its grain ID in shared memory.  The neighbours whose
// boxes reach the slab are staged in shared memory in list order.  Each warp owns
// every nw-th row of the slab and walks the staged neighbours in list order,
// updating only the voxels of its own rows inside the box intersection with the
// reference's strict "greater than" rule -- so every voxel sees the neighbours in
// the reference's order and the result is bit-identical, without atomics, and the
// work is proportional to the voxels the neighbours cover (lanes along x, a
// pointer-stepped loop along z).
// Voxels no neighbour covers keep their IDLocal from the previous layout by the
// reference's flat-prefix resize (dimensionalBuffer.h:120-131).
#include "gg_kernels.cuh"

#include <climits>

namespace gg {

namespace {

constexpr int kThreads = 256;
constexpr int kStageCap = 512;   // staged neighbour boxes per round
constexpr unsigned kNone = 0xFFFFFFFFu;

struct Staged {
    int x0, x1, y0, y1, z0, z1;
    uint32_t id;
    int pad;
    long long off;
};

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

__device__ __forceinline__ int block_excl_scan(int v, int* sums, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < nw ? sums[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < nw) sums[lane] = wi - w;
        if (lane == 31) sums[32] = wi;
    }
    __syncthreads();
    total = sums[32];
    const int r = sums[warp] + incl - v;
    __syncthreads();
    return r;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) compare_kernel(CompareArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sums[33];
    Staged* st = reinterpret_cast<Staged*>(smem_raw);
    T* sval = reinterpret_cast<T*>(st + kStageCap);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int s = t - a.toff[g];
        const Box A = a.in.grain_box(g);
        const int sz0 = A.z0 + s * a.slab, sz1 = min(A.z1, sz0 + a.slab);
        const int nx = A.nx(), ny = A.ny();
        const int P = nx * ny, V = P * (sz1 - sz0);
        uint32_t* sid = reinterpret_cast<uint32_t*>(sval + V);
        for (int l = threadIdx.x; l < V; l += blockDim.x) {
            sval[l] = T(-1);  // clearValues(-1.0), box.cpp:894
            sid[l] = kNone;
        }
        const uint32_t* list = a.cmp + (long long)g * a.list_cap;
        const int K = a.n_cmp[g];
        if (s == 0) {  // m_secondOrderNeighbours = m_comparisonList, box.cpp:895
            uint32_t* son = a.son + (long long)g * a.list_cap;
            for (int q = threadIdx.x; q < K; q += blockDim.x) son[q] = list[q];
            if (threadIdx.x == 0) a.n_son[g] = K;
        }
        for (int c0 = 0; c0 < K; c0 += kStageCap) {
            // stage the neighbours of this round that reach the slab, keeping list order
            int n_staged = 0;
            for (int r0 = c0; r0 < min(K, c0 + kStageCap); r0 += blockDim.x) {
                const int p = r0 + threadIdx.x;
                Staged e;
                bool hit = false;
                if (p < min(K, c0 + kStageCap)) {
                    e.id = list[p];
                    const int* bb = a.in.box + 6 * e.id;
                    e.x0 = bb[0]; e.x1 = bb[1]; e.y0 = bb[2]; e.y1 = bb[3]; e.z0 = bb[4]; e.z1 = bb[5];
                    e.pad = 0;
                    hit = e.x0 < A.x1 && e.x1 > A.x0 && e.y0 < A.y1 && e.y1 > A.y0 && e.z0 < sz1 && e.z1 > sz0;
                    e.off = hit ? a.in.off[e.id] : 0;
                }
                int cnt;
                const int pos = block_excl_scan(hit ? 1 : 0, sums, cnt);
                if (hit) st[n_staged + pos] = e;
                n_staged += cnt;
            }
            __syncthreads();
            // walk them in list order; warp w owns the slab rows y with (y - A.y0) % nw == w,
            // and a short intersection row lets one warp take several owned rows at once
            for (int e = 0; e < n_staged; e++) {
                const Staged B = st[e];
                const int ylo = max(A.y0, B.y0), yhi = min(A.y1, B.y1);
                const int ix0 = max(A.x0, B.x0), ix1 = min(A.x1, B.x1);
                const int iz0 = max(sz0, B.z0), iz1 = min(sz1, B.z1);
                const int wx = ix1 - ix0;
                const int lpr = wx <= 8 ? 8 : wx <= 16 ? 16 : 32;
                const int rpi = 32 / lpr, xo = lane & (lpr - 1), rsub = lane / lpr;
                // first row >= ylo owned by this warp, then this lane's row among the rpi taken together
                int y = ylo + ((warp - (ylo - A.y0)) % nw + nw) % nw + rsub * nw;
                if (ylo + ((warp - (ylo - A.y0)) % nw + nw) % nw >= yhi) continue;
                const int bnx = B.x1 - B.x0;
                const long long bplane = (long long)(B.y1 - B.y0) * bnx;
                const long long bbase = B.off + (long long)(iz0 - B.z0) * bplane - B.x0 - (long long)B.y0 * bnx;
                uint32_t* sidp = sid;
                for (; y < yhi; y += rpi * nw) {
                    for (int x = ix0 + xo; x < ix1; x += lpr) {
                        const T* __restrict__ bp = a.in.data + (bbase + (long long)y * bnx + x);
                        int sp = ((iz0 - sz0) * ny + (y - A.y0)) * nx + (x - A.x0);
#pragma unroll 4
                        for (int z = iz0; z < iz1; z++, bp += bplane, sp += P) {
                            const T v = __ldg(bp);
                            if (v > sval[sp]) {  // box.cpp:938: strict, the first in list order wins
                                sval[sp] = v;
                                sidp[sp] = B.id;
                            }
                        }
                    }
                }
                __syncwarp();
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
        const long long base = (long long)(sz0 - A.z0) * P;
        int bx0 = INT_MAX, bx1 = INT_MIN, by0 = INT_MAX, by1 = INT_MIN, bz0 = INT_MAX, bz1 = INT_MIN;
        for (int l = threadIdx.x; l < V; l += blockDim.x) {
            const int zl = l / P, rem = l - zl * P;
            const int yl = rem / nx;
            const int x = A.x0 + rem - yl * nx, y = A.y0 + yl, z = sz0 + zl;
            const long long f3 = base + l;
            T cmpv = sval[l];
            uint32_t idv = sid[l];
            if (idv == kNone) idv = f3 < old_count ? idold[f3] : 0u;
            if (boundary) {
                const double d = bc_dist(A, y, x, z, a.geo.M, a.geo.gb);
                if (d > -a.geo.gb)
                    if (d * a.geo.h > (double)cmpv) {
                        cmpv = (T)(d * a.geo.h);
                        idv = 0;
                    }
            }
            const T in = self[f3];
            T res;
            if ((double)fabs(in) < lim) res = T(0.5) * (in - cmpv);
            else res = in;
            outp[f3] = res;
            idnew[f3] = idv;
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
        if (lane == 0 && bx0 != INT_MAX) {
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

int compare_slab(int side, bool fp64) {
    const size_t per = fp64 ? 12 : 8;
    const size_t budget = 80 * 1024;
    long long s = (long long)(budget / (per * (size_t)(side > 0 ? side * side : 1)));
    return (int)(s < 1 ? 1 : s > 16 ? 16 : s);
}

size_t compare_smem_bytes(int side, int slab, bool fp64) {
    return sizeof(Staged) * kStageCap + (size_t)side * side * slab * (fp64 ? 12 : 8);
}

template <typename T>
void launch_compare(const CompareArgs<T>& a, int grid, size_t smem, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        allow_max_dynamic_smem(compare_kernel<T>);
        configured = true;
    }
    compare_kernel<T><<<grid, kThreads, smem, s>>>(a);
}

void launch_newbox_init(int G, const int* present, const int* exists, const int* box, int* newbox, cudaStream_t s) {
    newbox_init_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, present, exists, box, newbox);
}

template void launch_compare<double>(const CompareArgs<double>&, int, size_t, cudaStream_t);
template void launch_compare<float>(const CompareArgs<float>&, int, size_t, cudaStream_t);

}  // namespace gg

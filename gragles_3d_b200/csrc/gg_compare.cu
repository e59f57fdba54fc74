// gg_compare.cu -- comparison, boundary condition and set-comparison of every grain.
//
// Stands in for LSbox::executeComparison (box.cpp:891-966), boundaryCondition
// (box.cpp:997-1088) and executeSetComparison (box.cpp:814-878).
//
// The reference, per grain A and voxel v of A's box, walks A's comparison list in
// order and keeps the first neighbour whose value at v is strictly greater than
// everything before it (starting from -1).  That is: the largest value among the
// listed neighbours whose box contains v, ties going to the earliest list
// position.  Each box voxel is read about thirty times that way.  Here the work is
// turned around and done per domain tile instead of per grain:
//
//   1. bin: every tile of kTX x kTY x kTZ domain voxels gets the IDs of the
//      grains whose boxes reach it (count, scan, fill);
//   2. compare: one CTA per tile loads every covering box's values over the tile
//      into shared memory once and looks up, in each covering grain's position
//      table (built once per step from its comparison list), the position of every
//      other covering grain in its list.  Per voxel it keeps the kTop
//      largest values; every (grain, voxel) pair then picks the first candidate
//      that is in that grain's list, resolving equal values by list position --
//      falling back to a full scan of the tile's boxes whenever the kTop
//      candidates cannot decide.  The boundary condition, the set comparison, the
//      outputs and the new bounding box follow in the same pass.
//   3. copy_lists: m_secondOrderNeighbours = m_comparisonList for the next step.
//
// Every value is read once and written once (12 B per voxel on the FP32 path),
// and the result is bit-identical to the sequential walk.  Voxels no listed
// neighbour covers keep their IDLocal from the previous layout by the reference's
// flat-prefix resize (dimensionalBuffer.h:120-131).
#include "gg_kernels.cuh"

#include <math_constants.h>

#include <climits>

namespace gg {

namespace {

constexpr int kThreads = 256;
constexpr int kTV = kTX * kTY * kTZ;   // voxels per tile (64)
constexpr int kTop = 4;                // candidates kept per voxel
constexpr int kParts = kThreads / kTV; // threads scanning the boxes of one voxel
// row stride of the staged values: the kParts lanes of a voxel read kVS apart, which
// puts the 32 lanes of a warp on 32 different banks
constexpr int kVS = kTV + 8;
static_assert(kTV % 32 == 0 && kThreads % kTV == 0, "a warp's lanes share one tile entry per pair sweep");
static_assert(kThreads == kTV * kParts && kTop == 4 && (kParts & (kParts - 1)) == 0, "top-4 merge layout");
constexpr unsigned kNone = 0xFFFFFFFFu;
constexpr unsigned short kNotListed = 0xFFFF;
constexpr int kUCap = 32;              // candidate columns of the position matrix

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

// ---------------------------------------------------------------------------------
// 1. m_secondOrderNeighbours = m_comparisonList (box.cpp:895), for the next list update
// ---------------------------------------------------------------------------------
__global__ void copy_lists_kernel(ListCopyArgs a) {
    const int total = a.toff[a.G + 1];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int K = a.n_cmp[g];
        const uint32_t* list = a.cmp + (long long)g * a.list_cap;
        uint32_t* son = a.son + (long long)g * a.list_cap;
        for (int i = threadIdx.x; i < K; i += blockDim.x) son[i] = list[i];
        if (threadIdx.x == 0) a.n_son[g] = K;
    }
}

// ---------------------------------------------------------------------------------
// 2. binning of grain boxes to domain tiles: one warp per grain, lanes over its tiles
// ---------------------------------------------------------------------------------
template <bool FILL>
__global__ void bin_kernel(TileBins tb, int G, const int* exists, const int* box, int* err) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int g = 1 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); g <= G; g += warps) {
        if (!exists[g]) continue;
        const Box b = load_box(box + 6 * g);
        if (b.nx() <= 0) continue;
        const int tx0 = b.x0 / kTX, nbx = (b.x1 - 1) / kTX - tx0 + 1;
        const int ty0 = b.y0 / kTY, nby = (b.y1 - 1) / kTY - ty0 + 1;
        const int tz0 = b.z0 / kTZ, nbz = (b.z1 - 1) / kTZ - tz0 + 1;
        const int n = nbx * nby * nbz;
        for (int i = lane; i < n; i += 32) {
            const int tx = tx0 + i % nbx, ty = ty0 + (i / nbx) % nby, tz = tz0 + i / (nbx * nby);
            const int t = (tz * tb.nty + ty) * tb.ntx + tx;
            if (!FILL) {
                atomicAdd(tb.count + t, 1);
            } else {
                const long long slot = (long long)tb.off[t] + atomicAdd(tb.cursor + t, 1);
                if (slot >= 0 && slot < tb.capacity) tb.entries[slot] = (uint32_t)g;
                else atomicOr(err, ERR_POOL);
            }
        }
    }
}

// After the device-wide exclusive scan of the tile counts: the largest count and the
// capacity check (off[n_tiles] is the total, count[n_tiles] being 0).
__global__ void bin_check_kernel(TileBins tb, int n_tiles, int* err) {
    int m = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_tiles; t += gridDim.x * blockDim.x) m = max(m, tb.count[t]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(tb.max_count, m);
    if (blockIdx.x == 0 && threadIdx.x == 0 && ((long long)tb.off[n_tiles] > tb.capacity || tb.off[n_tiles] < 0))
        atomicOr(err, ERR_POOL);
}

// Exclusive scan of the tile counts (one CTA), largest count, capacity check.
__global__ void __launch_bounds__(1024) bin_scan_kernel(TileBins tb, int n_tiles, int* err) {
    __shared__ long long sums[33];
    __shared__ int mx[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (n_tiles + blockDim.x - 1) / blockDim.x;
    const int t0 = threadIdx.x * per, t1 = min(n_tiles, t0 + per);
    long long mine = 0;
    int m = 0;
    for (int t = t0; t < t1; t++) {
        mine += tb.count[t];
        m = max(m, tb.count[t]);
    }
    long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 31) sums[warp] = incl;
    if (lane == 0) mx[warp] = m;
    __syncthreads();
    if (warp == 0) {
        const long long w = sums[lane];
        long long wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        sums[lane] = wi - w;
        if (lane == 31) sums[32] = wi;
        int mm = mx[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mm = max(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        if (lane == 0) mx[0] = mm;
    }
    __syncthreads();
    long long run = sums[warp] + incl - mine;
    for (int t = t0; t < t1; t++) {
        tb.off[t] = (int)run;
        run += tb.count[t];
    }
    if (threadIdx.x == 0) {
        tb.off[n_tiles] = (int)sums[32];
        *tb.max_count = mx[0];
        if (sums[32] > tb.capacity) atomicOr(err, ERR_POOL);
    }
}

// ---------------------------------------------------------------------------------
// 3. the per-tile comparison
// ---------------------------------------------------------------------------------
template <typename T>
struct TileSmem {
    // entries (boxes reaching the tile)
    uint32_t* id;
    int* box;           // 6 per entry
    long long* off;
    int* bbox;          // 6 per entry: new bounding box contributions
    long long* outoff;  // per entry: offset of its output box and IDLocal box
    long long* idoff;
    int* tsize;         // per entry: size of its position table
    T* val;             // [entry][voxel]
    unsigned short* pos;// [entry a][entry b]: position of b in a's list, kNotListed, or kUnknown
    T* topv;            // [kTop][voxel]
    unsigned char* topi;
    int* ncand;         // covering entries with value > -1, per voxel
    unsigned* umask;    // 8 words: entries among some voxel's kTop candidates
    unsigned char* ulist;  // those entries, ascending
    unsigned char* ucol;   // per entry: its column of pos (the first kUCap of ulist), 0xFF: none
    int* nu;            // their count
    unsigned char* bnd;    // per entry: its box reaches the boundary grain's zone
    unsigned char* deep;   // per voxel: at least gb from every face of that zone
};

template <typename T>
__device__ TileSmem<T> carve(unsigned char* base, int mcap) {
    TileSmem<T> s;
    unsigned char* p = base;
    s.off = reinterpret_cast<long long*>(p); p += 8 * mcap;
    s.outoff = reinterpret_cast<long long*>(p); p += 8 * mcap;
    s.idoff = reinterpret_cast<long long*>(p); p += 8 * mcap;
    s.val = reinterpret_cast<T*>(p); p += sizeof(T) * (size_t)mcap * kVS;
    s.topv = reinterpret_cast<T*>(p); p += sizeof(T) * kTV * kTop;
    s.id = reinterpret_cast<uint32_t*>(p); p += 4 * mcap;
    s.box = reinterpret_cast<int*>(p); p += 24 * mcap;
    s.bbox = reinterpret_cast<int*>(p); p += 24 * mcap;
    s.tsize = reinterpret_cast<int*>(p); p += 4 * mcap;
    s.ncand = reinterpret_cast<int*>(p); p += 4 * kTV;
    s.umask = reinterpret_cast<unsigned*>(p); p += 4 * 8;
    s.nu = reinterpret_cast<int*>(p); p += 16;
    s.pos = reinterpret_cast<unsigned short*>(p); p += 2 * (size_t)mcap * kUCap;
    s.ulist = p; p += 256;
    s.ucol = p; p += 256;
    s.topi = p; p += kTV * kTop;
    s.deep = p; p += kTV;
    s.bnd = p;
    return s;
}

// |in| < lim, lim in FP64, as (double)fabs(in) < lim: for FP32 values against the FP32
// bound rounded up (a float is below a double exactly when it is below that bound).
__device__ __forceinline__ bool in_band(double in, double lim) { return fabs(in) < lim; }
__device__ __forceinline__ bool in_band(float in, double lim) { return fabsf(in) < __double2float_ru(lim); }

template <typename T>
__device__ __forceinline__ T neg_inf();
template <>
__device__ __forceinline__ double neg_inf<double>() { return -CUDART_INF; }
template <>
__device__ __forceinline__ float neg_inf<float>() { return -CUDART_INF_F; }

// Keep the kTop largest values seen so far in descending order (registers only).
template <typename T>
__device__ __forceinline__ void top_insert(T (&tv)[kTop], int (&ti)[kTop], T w, int e) {
    if (!(w > tv[kTop - 1])) return;
    tv[kTop - 1] = w;
    ti[kTop - 1] = e;
#pragma unroll
    for (int k = kTop - 1; k > 0; k--) {
        if (tv[k] > tv[k - 1]) {
            const T t = tv[k]; tv[k] = tv[k - 1]; tv[k - 1] = t;
            const int u = ti[k]; ti[k] = ti[k - 1]; ti[k - 1] = u;
        }
    }
}

__device__ __forceinline__ unsigned pos_home(uint32_t id, int size) { return (id * 2654435761u) & (unsigned)(size - 1); }

// Position of grain b in grain a's comparison list (a's position table of tsize slots),
// or kNotListed.
template <typename T>
__device__ unsigned short list_position(const CompareArgs<T>& a, uint32_t ga, int tsize, uint32_t gb) {
    const unsigned long long* tab = a.pos_table + (long long)ga * a.pos_cap;
    unsigned h = pos_home(gb, tsize);
    for (int probe = 0; probe < tsize; probe++) {
        const unsigned long long e = __ldg(tab + h);
        const uint32_t k = (uint32_t)(e >> 32);
        if (k == gb) return (unsigned short)(e & 0xFFFFu);
        if (k == kNone) return kNotListed;
        h = (h + 1) & (unsigned)(tsize - 1);
    }
    return kNotListed;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 4) compare_kernel(CompareArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem<T> s = carve<T>(smem_raw, a.mcap);
    const TileBins& tb = a.bins;
    const int n_tiles = tb.ntx * tb.nty * tb.ntz;
    const T NEG = neg_inf<T>();
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const int e0 = tb.off[t], m = tb.off[t + 1] - e0;
        if (m == 0) continue;
        if (m > a.mcap) {
            if (threadIdx.x == 0) atomicOr(a.err, ERR_BOX);
            continue;
        }
        const int tx = t % tb.ntx, ty = (t / tb.ntx) % tb.nty, tz = t / (tb.ntx * tb.nty);
        const int X0 = tx * kTX, Y0 = ty * kTY, Z0 = tz * kTZ;
        // entries
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
            const uint32_t g = tb.entries[e0 + e];
            s.id[e] = g;
            const int* bb = a.in.box + 6 * g;
#pragma unroll
            for (int q = 0; q < 6; q++) s.box[6 * e + q] = bb[q];
            s.off[e] = a.in.off[g];
            s.outoff[e] = a.out.off[g];
            s.idoff[e] = a.idoff_new[g];
            s.tsize[e] = pos_table_size(a.n_cmp[g], a.pos_cap);
            s.bnd[e] = !(bb[0] > a.geo.gb && bb[1] < a.geo.M - a.geo.gb && bb[2] > a.geo.gb &&
                         bb[3] < a.geo.M - a.geo.gb && bb[4] > a.geo.gb && bb[5] < a.geo.M - a.geo.gb);
            s.bbox[6 * e + 0] = INT_MAX; s.bbox[6 * e + 1] = INT_MIN;
            s.bbox[6 * e + 2] = INT_MAX; s.bbox[6 * e + 3] = INT_MIN;
            s.bbox[6 * e + 4] = INT_MAX; s.bbox[6 * e + 5] = INT_MIN;
        }
        if (threadIdx.x < 8) s.umask[threadIdx.x] = 0u;
        __syncthreads();
        // values of every covering box over the tile (-inf outside the box), copied with
        // cp.async so that no thread waits on one load before issuing the next
        {
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int e = warp; e < m; e += nw) {
                const Box B = load_box(s.box + 6 * e);
                const T* src = a.in.data + s.off[e];
#pragma unroll
                for (int vv = 0; vv < kTV; vv += 32) {
                    const int v = vv + lane;
                    const int x = X0 + v % kTX, y = Y0 + (v / kTX) % kTY, z = Z0 + v / (kTX * kTY);
                    if (x >= B.x0 && x < B.x1 && y >= B.y0 && y < B.y1 && z >= B.z0 && z < B.z1)
                        cp_async_elem(s.val + e * kVS + v, src + B.at(y, x, z));
                    else
                        s.val[e * kVS + v] = NEG;
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        // per voxel: the kTop largest values > -1.  The kParts lanes of a voxel are
        // neighbours in one warp; each keeps the top of every kParts-th box, then two
        // shuffle rounds merge their lists (a bitonic merge of two sorted lists of kTop).
        {
            const int lane = threadIdx.x & 31;
            const int part = lane & (kParts - 1), v = (threadIdx.x >> 5) * (32 / kParts) + (lane / kParts);
            T tv[kTop];
            int ti[kTop];
#pragma unroll
            for (int k = 0; k < kTop; k++) { tv[k] = NEG; ti[k] = 0xFF; }
            int nc = 0;
            for (int e = part; e < m; e += kParts) {
                const T w = s.val[e * kVS + v];
                if (!(w > T(-1))) continue;
                nc++;
                top_insert(tv, ti, w, e);
            }
#pragma unroll
            for (int o = 1; o < kParts; o <<= 1) {
                T pv[kTop];
                int pi[kTop];
#pragma unroll
                for (int k = 0; k < kTop; k++) {
                    pv[k] = __shfl_xor_sync(0xffffffffu, tv[k], o);
                    pi[k] = __shfl_xor_sync(0xffffffffu, ti[k], o);
                }
                nc += __shfl_xor_sync(0xffffffffu, nc, o);
                // both lanes merge (lower part's list, higher part's list) alike
                const bool low = (lane & o) == 0;
                T av[kTop], bv[kTop];
                int ai[kTop], bi[kTop];
#pragma unroll
                for (int k = 0; k < kTop; k++) {
                    av[k] = low ? tv[k] : pv[k];
                    ai[k] = low ? ti[k] : pi[k];
                    bv[k] = low ? pv[k] : tv[k];
                    bi[k] = low ? pi[k] : ti[k];
                }
                // the kTop largest of both: max(a[k], b[kTop-1-k]), a bitonic sequence
#pragma unroll
                for (int k = 0; k < kTop; k++) {
                    const bool ta = !(bv[kTop - 1 - k] > av[k]);
                    tv[k] = ta ? av[k] : bv[kTop - 1 - k];
                    ti[k] = ta ? ai[k] : bi[kTop - 1 - k];
                }
                // sorted descending by a bitonic half-cleaner cascade
#pragma unroll
                for (int j = kTop / 2; j > 0; j >>= 1)
#pragma unroll
                    for (int k = 0; k < kTop; k++)
                        if ((k & j) == 0 && tv[k + j] > tv[k]) {
                            const T t = tv[k]; tv[k] = tv[k + j]; tv[k + j] = t;
                            const int u = ti[k]; ti[k] = ti[k + j]; ti[k + j] = u;
                        }
            }
            if (part == 0) {
#pragma unroll
                for (int k = 0; k < kTop; k++) {
                    s.topv[k * kTV + v] = tv[k];
                    s.topi[k * kTV + v] = (unsigned char)ti[k];
                    if (ti[k] != 0xFF) atomicOr(s.umask + (ti[k] >> 5), 1u << (ti[k] & 31));
                }
                s.ncand[v] = nc;
                // A voxel at least gb from every face of the boundary grain's zone gets an
                // all-negative distance <= -gb from bc_assign, which changes nothing.
                const int x = X0 + v % kTX, y = Y0 + (v / kTX) % kTY, z = Z0 + v / (kTX * kTY);
                const int lo_in = 2 * a.geo.gb - 1, hi_in = a.geo.M - 1 - 2 * a.geo.gb;
                s.deep[v] = x >= lo_in && x <= hi_in && y >= lo_in && y <= hi_in && z >= lo_in && z <= hi_in;
            }
        }
        __syncthreads();
        // the columns of pos the pair loop reads: every entry that is among some voxel's
        // kTop candidates.  pos[a][b] = position of b in a's list, from a's position
        // table; kBatch lookups advance together, each round issuing all their next probes
        if (threadIdx.x < 32) {
            int nu = 0;
            for (int b0 = 0; b0 < m; b0 += 32) {
                const int b = b0 + threadIdx.x;
                const bool in_u = b < m && ((s.umask[b >> 5] >> (b & 31)) & 1u);
                const unsigned bal = __ballot_sync(0xffffffffu, in_u);
                const int r = nu + __popc(bal & ((1u << threadIdx.x) - 1));
                if (in_u) s.ulist[r] = (unsigned char)b;
                if (b < m) s.ucol[b] = (in_u && r < kUCap) ? (unsigned char)r : (unsigned char)0xFF;
                nu += __popc(bal);
            }
            if (threadIdx.x == 0) s.nu[0] = nu;
        }
        __syncthreads();
        {
            constexpr int kBatch = 4;
            const int nu = min(s.nu[0], kUCap);  // columns beyond kUCap are looked up when needed
            const int mm = m * nu;
            for (int q0 = 0; q0 < mm; q0 += kBatch * kThreads) {
                unsigned long long e[kBatch];
                const unsigned long long* tab[kBatch];
                unsigned h[kBatch], mask[kBatch];
                uint32_t id[kBatch];
                bool live[kBatch];
                int dst[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    const int q = q0 + u * kThreads + threadIdx.x;
                    const int ea = q / nu, col = q - ea * nu, eb = q < mm ? s.ulist[col] : 0;
                    live[u] = q < mm && ea != eb;
                    dst[u] = ea * kUCap + col;
                    tab[u] = nullptr;
                    h[u] = mask[u] = id[u] = 0;
                    e[u] = 0;
                    if (live[u]) {
                        tab[u] = a.pos_table + (long long)s.id[ea] * a.pos_cap;
                        mask[u] = (unsigned)s.tsize[ea] - 1;
                        id[u] = s.id[eb];
                        h[u] = pos_home(id[u], s.tsize[ea]);
                        e[u] = __ldg(tab[u] + h[u]);
                    }
                }
                for (int round = 0; round < a.pos_cap; round++) {
                    bool more = false;
#pragma unroll
                    for (int u = 0; u < kBatch; u++) {
                        if (!live[u]) continue;
                        const uint32_t k = (uint32_t)(e[u] >> 32);
                        if (k == id[u] || k == kNone) {
                            s.pos[dst[u]] = k == id[u] ? (unsigned short)(e[u] & 0xFFFFu) : kNotListed;
                            live[u] = false;
                        } else {
                            h[u] = (h[u] + 1) & mask[u];
                            more = true;
                        }
                    }
                    if (!more) break;
#pragma unroll
                    for (int u = 0; u < kBatch; u++)
                        if (live[u]) e[u] = __ldg(tab[u] + h[u]);
                }
            }
        }
        __syncthreads();
        // every (grain, voxel) pair of the tile
        const double lim = 0.7 * a.geo.delta;
        for (int q = threadIdx.x; q < m * kTV; q += blockDim.x) {
            const int ea = q / kTV, v = q % kTV;
            const T in = s.val[ea * kVS + v];
            const int x = X0 + v % kTX, y = Y0 + (v / kTX) % kTY, z = Z0 + v / (kTX * kTY);
            bool positive = false;
            // else the voxel is outside this grain's box, or (recalculateIDLocal) the grain
            // does not exist and executeComparison leaves it alone
            if (in != NEG && (a.set_comparison || a.exists[s.id[ea]])) {
            // the first listed neighbour among the largest values, ties to the earliest position
            int best = -1;
            unsigned short bpos = kNotListed;
            T level = NEG;
            bool decided = false;
            int k = 0;
            for (; k < kTop; k++) {
                const int eb = s.topi[k * kTV + v];
                if (eb == 0xFF) break;
                const T w = s.topv[k * kTV + v];
                if (best >= 0 && !(w == level)) { decided = true; break; }
                if (eb == ea) continue;
                const int col = s.ucol[eb];
                const unsigned short p = col != 0xFF ? s.pos[ea * kUCap + col]
                                                     : list_position(a, s.id[ea], s.tsize[ea], s.id[eb]);
                if (p == kNotListed) continue;
                if (best < 0 || p < bpos) { best = eb; bpos = p; level = w; }
            }
            // decided anyway when every covering candidate was among those examined
            if (!decided && s.ncand[v] <= k) decided = true;
            if (!decided) {  // full scan of the tile's boxes at this voxel
                best = -1;
                bpos = kNotListed;
                level = NEG;
                for (int eb = 0; eb < m; eb++) {
                    if (eb == ea) continue;
                    const T w = s.val[eb * kVS + v];
                    if (!(w > T(-1))) continue;
                    if (best >= 0 && w < level) continue;
                    const int col = s.ucol[eb];
                    const unsigned short p = col != 0xFF ? s.pos[ea * kUCap + col]
                                                         : list_position(a, s.id[ea], s.tsize[ea], s.id[eb]);
                    if (p == kNotListed) continue;
                    if (best < 0 || w > level || (w == level && p < bpos)) { best = eb; bpos = p; level = w; }
                }
            }
            const uint32_t ga = s.id[ea];
            const Box A = load_box(s.box + 6 * ea);
            const long long f = A.at(y, x, z);
            T cmpv;
            uint32_t idv;
            if (best >= 0) {
                cmpv = s.val[best * kVS + v];
                idv = s.id[best];
            } else {  // no listed neighbour covers the voxel: value -1, IDLocal kept
                cmpv = T(-1);
                const Box Bold = load_box(a.idbox_old + 6 * ga);
                idv = f < Bold.count() ? a.id_old[a.idoff_old[ga] + f] : 0u;
            }
            if (s.bnd[ea] && !s.deep[v]) {  // the boundary condition near the zone's faces
                const double d = bc_dist(A, y, x, z, a.geo.M, a.geo.gb);
                if (d > -a.geo.gb)
                    if (d * a.geo.h > (double)cmpv) {
                        cmpv = (T)(d * a.geo.h);
                        idv = 0;
                    }
            }
            T res;
            if (!a.set_comparison) res = cmpv;
            else if (in_band(in, lim)) res = T(0.5) * (in - cmpv);
            else res = in;
            a.out.data[s.outoff[ea] + f] = res;
            a.id_new[s.idoff[ea] + f] = idv;
            positive = a.set_comparison && res >= 0;
            }
            // new bounding box (executeSetComparison, box.cpp:858-877), reduced over the warp
            // first: its 32 lanes hold the same entry (kTV and blockDim are multiples of 64)
            if (__ballot_sync(0xffffffffu, positive)) {
                const int x0 = __reduce_min_sync(0xffffffffu, positive ? x : INT_MAX);
                const int x1 = __reduce_max_sync(0xffffffffu, positive ? x : INT_MIN);
                const int y0 = __reduce_min_sync(0xffffffffu, positive ? y : INT_MAX);
                const int y1 = __reduce_max_sync(0xffffffffu, positive ? y : INT_MIN);
                const int z0 = __reduce_min_sync(0xffffffffu, positive ? z : INT_MAX);
                const int z1 = __reduce_max_sync(0xffffffffu, positive ? z : INT_MIN);
                if ((threadIdx.x & 31) == 0) {
                    int* bb = s.bbox + 6 * ea;
                    atomicMin(bb + 0, x0); atomicMax(bb + 1, x1);
                    atomicMin(bb + 2, y0); atomicMax(bb + 3, y1);
                    atomicMin(bb + 4, z0); atomicMax(bb + 5, z1);
                }
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
            const int* bb = s.bbox + 6 * e;
            if (bb[0] == INT_MAX) continue;
            int* nb = a.newbox + 6 * s.id[e];
            atomicMin(nb + 0, bb[0]); atomicMax(nb + 1, bb[1]);
            atomicMin(nb + 2, bb[2]); atomicMax(nb + 3, bb[3]);
            atomicMin(nb + 4, bb[4]); atomicMax(nb + 5, bb[5]);
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

size_t compare_smem_bytes(int mcap, bool fp64) {
    const size_t e = fp64 ? 8 : 4;
    return 24 * (size_t)mcap + e * (size_t)mcap * kVS + e * kTV * kTop + 4 * (size_t)mcap +
           48 * (size_t)mcap + 4 * (size_t)mcap + 4 * kTV + 48 + 2 * (size_t)mcap * kUCap + 512 +
           kTV * kTop + kTV + (size_t)mcap + 64;
}

long long bin_capacity(int G, int side) {
    const long long tx = side / kTX + 2, ty = side / kTY + 2, tz = side / kTZ + 2;
    return (long long)G * tx * ty * tz;
}

void launch_copy_lists(const ListCopyArgs& a, int grid, cudaStream_t s) {
    copy_lists_kernel<<<grid, 256, 0, s>>>(a);
}

void launch_bin(const TileBins& tb, int G, const int* exists, const int* box, int* err, cudaStream_t s) {
    const int n_tiles = tb.ntx * tb.nty * tb.ntz;
    cudaMemsetAsync(tb.count, 0, sizeof(int) * (n_tiles + 1), s);
    cudaMemsetAsync(tb.cursor, 0, sizeof(int) * (n_tiles + 1), s);
    const int grid = (G + 4) / 4;  // one warp per grain, 4 warps per block
    bin_kernel<false><<<grid, 128, 0, s>>>(tb, G, exists, box, err);
    if (tb.temp) {  // device-wide: the one-CTA scan below walks the tiles serially
        launch_exclusive_scan(tb.temp, tb.temp_bytes, tb.count, tb.off, n_tiles + 1, s);
        cudaMemsetAsync(tb.max_count, 0, sizeof(int), s);
        bin_check_kernel<<<(n_tiles + 255) / 256 < 1184 ? (n_tiles + 255) / 256 : 1184, 256, 0, s>>>(tb, n_tiles, err);
    } else {
        bin_scan_kernel<<<1, 1024, 0, s>>>(tb, n_tiles, err);
    }
    bin_kernel<true><<<grid, 128, 0, s>>>(tb, G, exists, box, err);
}

template <typename T>
void launch_compare(const CompareArgs<T>& a, int grid, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(compare_kernel<T>);
    });
    compare_kernel<T><<<grid, kThreads, compare_smem_bytes(a.mcap, sizeof(T) == 8), s>>>(a);
}

void launch_newbox_init(int G, const int* present, const int* exists, const int* box, int* newbox, cudaStream_t s) {
    newbox_init_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, present, exists, box, newbox);
}

template void launch_compare<double>(const CompareArgs<double>&, int, cudaStream_t);
template void launch_compare<float>(const CompareArgs<float>&, int, cudaStream_t);

}  // namespace gg

// gg_common.cuh -- device-side state shared by the level-set kernels.
//
// All grain boxes live in two SDF arenas in HBM.  Arena a holds the buffer that
// the reference calls m_inputDistance or m_outputDistance depending on a parity
// the host flips at every switchDistancebuffer (grainhdl.cpp:1166-1178), so a
// swap costs nothing.  Each arena has its own per-grain box and element offset:
// the two layouts agree except while redistancing writes the new (resized) boxes
// (box.cpp:2322-2586).  IDLocal lives in two more arenas with the same scheme, so
// the flat-prefix resize of the reference (dimensionalBuffer.h:120-131) becomes a
// read from the previous layout.
#pragma once

#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

namespace gg {

// Error bits set by kernels (atomicOr) and reported by the host.
enum : int {
    ERR_POOL = 1,        // arena or scratch capacity exceeded
    ERR_LIST = 2,        // comparison list capacity exceeded
    ERR_NEIGHBORS = 4,   // hull neighbour set capacity exceeded
    ERR_HASH = 8,        // list-update hash table overflow
    ERR_BOX = 16,        // a box outside the grid or larger than supported
    ERR_TIMEOUT = 32,    // a bounded wait on the tensor-core pipeline gave up
    ERR_HULL = 64,       // hull capture or interfacial-element capacity exceeded
    ERR_BOUNDS = 128,    // an index failed a kernel's own bounds check (access skipped)
};

struct Box {
    int x0, x1, y0, y1, z0, z1;
    __host__ __device__ int nx() const { return x1 - x0; }
    __host__ __device__ int ny() const { return y1 - y0; }
    __host__ __device__ int nz() const { return z1 - z0; }
    __host__ __device__ long long count() const { return (long long)nx() * ny() * nz(); }
    // getValueAt(row=i (y), column=j (x), depth=k (z)), dimensionalBuffer.h:71-76
    __host__ __device__ long long at(int i, int j, int k) const {
        return ((long long)(k - z0) * ny() + (i - y0)) * nx() + (j - x0);
    }
};

__host__ __device__ inline Box load_box(const int* b6) { return Box{b6[0], b6[1], b6[2], b6[3], b6[4], b6[5]}; }
__host__ __device__ inline void store_box(int* b6, const Box& b) {
    b6[0] = b.x0; b6[1] = b.x1; b6[2] = b.y0; b6[3] = b.y1; b6[4] = b.z0; b6[5] = b.z1;
}

// One arena's view: data, per-grain boxes (6 ints) and element offsets.
template <typename T>
struct Arena {
    T* data;
    int* box;
    long long* off;
    __device__ Box grain_box(int g) const { return load_box(box + 6 * g); }
    __device__ T* grain_ptr(int g) const { return data + off[g]; }
};

// Per-grain bookkeeping (entries 0..G, entry 0 = boundary grain, never processed).
struct Grains {
    int G;               // n_grains
    int* present;        // grains[id] != NULL
    int* exists;         // LSbox::m_exists
    int* newbox;         // m_newXMin.. from executeSetComparison (6 per grain)
    double* volume;      // m_volume
    double* surface;     // m_surface
    int* n_nb;           // distinct hull neighbours
    uint32_t* nb;        // nb_cap per grain
    int nb_cap;
    uint32_t* cmp;       // m_comparisonList, list_cap per grain
    int* n_cmp;
    uint32_t* son;       // m_secondOrderNeighbours, list_cap per grain
    int* n_son;
    int list_cap;
};

struct Geometry {
    int N;          // realDomainSize
    int gb;         // grid_blowup = DomainBorderSize
    int M;          // ngridpoints = N + 2 gb
    double h;       // 1 / N
    double delta;   // gb / N
    double time_step;
};

// Map a flat tile index to (grain, local tile) through an exclusive scan of
// per-grain tile counts (toff has G + 2 entries; toff[g] = first tile of g).
__device__ __forceinline__ int tile_grain(const int* __restrict__ toff, int G, int t) {
    int lo = 1, hi = G + 1;  // find the last g in [1, G] with toff[g] <= t
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(toff + mid) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// This CTA's share of the tiles, a contiguous range walked in order: one binary
// search at the start, then (grain, tile within the grain) advance incrementally.
// A binary search per tile would put ~log2(G) dependent loads in front of every tile.
struct TileWalk {
    const int* toff;
    int G, t, end;
    int g, local, count;  // grain, its tile index, its tile count
    __device__ TileWalk(const int* toff_, int G_, int part, int parts) : toff(toff_), G(G_) {
        const int total = toff[G + 1];
        t = (int)((long long)total * part / parts);
        end = (int)((long long)total * (part + 1) / parts);
        g = 1;
        local = count = 0;
        if (t < end) {
            g = tile_grain(toff, G, t);
            local = t - toff[g];
            count = toff[g + 1] - toff[g];
        }
    }
    __device__ bool valid() const { return t < end; }
    __device__ void next() {
        ++t;
        if (++local < count) return;
        local = 0;
        while (t < end && g < G) {  // next grain with tiles; g stays in [1, G]
            ++g;
            count = toff[g + 1] - toff[g];
            if (count > 0) break;
        }
    }
};

// Asynchronous 4- or 8-byte global -> shared copy (cp.async): staging loops issue all
// their copies without waiting on each load, then wait once.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst_smem, const T* src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// Asynchronous 16-byte global -> shared copy through L2 (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// Opt a kernel into the largest dynamic shared memory the device allows next to
// its static shared memory.
template <typename K>
inline cudaError_t allow_max_dynamic_smem(K* kernel) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

// DimensionalBuffer::resizeToCube, dimensionalBuffer.h:139-219
__host__ __device__ inline Box resize_to_cube(Box b, int maximumLength) {
    const int grid_size = maximumLength - 1;
    const unsigned height = b.y1 - b.y0, width = b.x1 - b.x0, depth = b.z1 - b.z0;
    if (width == height && width == depth) return b;
    int ref = width > height ? (int)width : (int)height;
    if (ref < (int)depth) ref = (int)depth;
    if (ref > (int)width) { const int d = ref - (int)width; b.x0 -= d / 2; b.x1 += d / 2 + d % 2; }
    if (ref > (int)height) { const int d = ref - (int)height; b.y0 -= d / 2; b.y1 += d / 2 + d % 2; }
    if (ref > (int)depth) { const int d = ref - (int)depth; b.z0 -= d / 2; b.z1 += d / 2 + d % 2; }
    if (b.x0 < 0) { const int d = -b.x0; b.x1 += d; b.x0 += d; }
    else if (b.x1 > grid_size) { const int d = grid_size - b.x1; b.x1 += d; b.x0 += d; }
    if (b.y0 < 0) { const int d = -b.y0; b.y1 += d; b.y0 += d; }
    else if (b.y1 > grid_size) { const int d = grid_size - b.y1; b.y1 += d; b.y0 += d; }
    if (b.z0 < 0) { const int d = -b.z0; b.z1 += d; b.z0 += d; }
    else if (b.z1 > grid_size) { const int d = grid_size - b.z1; b.z1 += d; b.z0 += d; }
    return b;
}

// Runs a set-up action once per CUDA device, on the device current at the call.
// Kernel attributes such as the dynamic shared-memory opt-in belong to the
// device (context) they were set on, so a process that drives a second device
// must set them there again.  Calls from several host threads are serialised.
class PerDevice {
  public:
    template <typename F>
    void once(F&& f) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
            f();
            return;
        }
        std::lock_guard<std::mutex> lock(mu_);
        if ((done_ >> dev) & 1ull) return;
        f();
        done_ |= 1ull << dev;
    }

  private:
    std::mutex mu_;
    unsigned long long done_ = 0;
};

__device__ __forceinline__ int isgn(double v) { return (0.0 < v) - (v < 0.0); }  // utilities.h:27-30
__device__ __forceinline__ int isgn(float v) { return (0.0f < v) - (v < 0.0f); }

}  // namespace gg

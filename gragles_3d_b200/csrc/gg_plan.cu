// gg_plan.cu -- device-side layout planner for the box pool.
//
// The reference allocates every box with std::vector and resizes it every step
// (dimensionalBuffer.h:120-131, jemalloc underneath).  Here the boxes of all grains
// are packed into one arena per buffer role; after every change of box sizes one
// CTA re-plans the packing (exclusive scan of the aligned n^3 over grains, a chunk of
// consecutive grains at a time), the
// half-spectrum scratch, and the tile offsets that the batched stage kernels use
// to map their CTAs to (grain, tile).  Nothing goes back to the host, so a whole
// timestep can be launched without synchronisation.
#include "gg_kernels.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>

namespace gg {

namespace {

constexpr int kPlanThreads = 1024;
constexpr long long kAlign = 32;  // elements; 256 B for FP64, 128 B for FP32

struct Counts {
    long long vox, spec, tot;
    int tn, ts, t1, tb;
};

__device__ __forceinline__ Counts add(const Counts& a, const Counts& b) {
    return Counts{a.vox + b.vox, a.spec + b.spec, a.tot + b.tot, a.tn + b.tn, a.ts + b.ts, a.t1 + b.t1, a.tb + b.tb};
}

__device__ __forceinline__ Counts shfl_up(const Counts& c, int o) {
    Counts r;
    r.vox = __shfl_up_sync(0xffffffffu, c.vox, o);
    r.spec = __shfl_up_sync(0xffffffffu, c.spec, o);
    r.tot = __shfl_up_sync(0xffffffffu, c.tot, o);
    r.tn = __shfl_up_sync(0xffffffffu, c.tn, o);
    r.ts = __shfl_up_sync(0xffffffffu, c.ts, o);
    r.t1 = __shfl_up_sync(0xffffffffu, c.t1, o);
    r.tb = __shfl_up_sync(0xffffffffu, c.tb, o);
    return r;
}

__device__ __forceinline__ Counts grain_counts(const PlanArgs& a, int g) {
    Counts c{0, 0, 0, 0, 0, 0, 0};
    if (g < 1 || g > a.G || !a.present[g] || (a.only_existing && !a.exists[g])) return c;
    const Box b = load_box(a.box + 6 * g);
    const long long n = b.nx();
    const long long v = b.count();
    c.vox = (v + kAlign - 1) / kAlign * kAlign;
    const long long sp = n * n * (n / 2 + 1);
    c.spec = (sp + kAlign - 1) / kAlign * kAlign;
    c.tot = v;
    c.tn = (int)n;
    const bool big = a.class_side > 0 && n > a.class_side;
    c.ts = a.row_tile > 0 ? (big ? 0 : (int)((n * n + a.row_tile - 1) / a.row_tile))
                          : (a.slab > 0 ? (int)((n + a.slab - 1) / a.slab) : 0);
    c.t1 = 1;
    c.tb = big ? (int)n : 0;
    return c;
}

// Grains 0..G in chunks of kPlanThreads consecutive IDs (coalesced loads and stores):
// a block exclusive scan per chunk on top of the running total of the earlier chunks.
__global__ void __launch_bounds__(kPlanThreads) plan_kernel(PlanArgs a) {
    __shared__ Counts warp_tot[32];
    __shared__ Counts carry_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Counts carry{0, 0, 0, 0, 0, 0, 0};
    for (int g0 = 0; g0 <= a.G; g0 += kPlanThreads) {
        const int g = g0 + threadIdx.x;
        const Counts mine = g <= a.G ? grain_counts(a, g) : Counts{0, 0, 0, 0, 0, 0, 0};
        Counts incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Counts u = shfl_up(incl, o);
            if (lane >= o) incl = add(incl, u);
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            Counts wi = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const Counts u = shfl_up(wi, o);
                if (lane >= o) wi = add(wi, u);
            }
            warp_tot[lane] = wi;  // inclusive over warps
        }
        __syncthreads();
        Counts run = add(carry, warp > 0 ? warp_tot[warp - 1] : Counts{0, 0, 0, 0, 0, 0, 0});
        run = add(run, Counts{incl.vox - mine.vox, incl.spec - mine.spec, incl.tot - mine.tot, incl.tn - mine.tn,
                              incl.ts - mine.ts, incl.t1 - mine.t1, incl.tb - mine.tb});
        if (g <= a.G) {
            if (a.off) a.off[g] = run.vox;
            if (a.spec_off) a.spec_off[g] = run.spec;
            if (a.toff_n) a.toff_n[g] = run.tn;
            if (a.toff_slab) a.toff_slab[g] = run.ts;
            if (a.toff_one) a.toff_one[g] = run.t1;
            if (a.toff_big) a.toff_big[g] = run.tb;
            if (a.box_copy) {
#pragma unroll
                for (int q = 0; q < 6; q++) a.box_copy[6 * g + q] = a.box[6 * g + q];
            }
            if (a.off_copy && a.off) a.off_copy[g] = run.vox;
        }
        if (threadIdx.x == 0) carry_s = add(carry, warp_tot[31]);
        __syncthreads();
        carry = carry_s;
        __syncthreads();  // warp_tot and carry_s are rewritten by the next chunk
    }
    if (threadIdx.x == kPlanThreads - 1) {
        const Counts T = carry;
        // Over capacity: report, and give the stage kernels no tiles so that nothing
        // is written past the end of an arena.
        const bool over = (a.off && T.vox > a.capacity) || (a.spec_off && T.spec > a.spec_capacity);
        if (over) atomicOr(a.err, ERR_POOL);
        if (a.toff_n) a.toff_n[a.G + 1] = over ? 0 : T.tn;
        if (a.toff_slab) a.toff_slab[a.G + 1] = over ? 0 : T.ts;
        if (a.toff_one) a.toff_one[a.G + 1] = over ? 0 : T.t1;
        if (a.toff_big) a.toff_big[a.G + 1] = over ? 0 : T.tb;
        if (a.total_voxels) *a.total_voxels = T.tot;
    }
}

__global__ void copy_layout_kernel(int G, const int* present, const int* box_src, const long long* off_src,
                                   int* box_dst, long long* off_dst) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        if (!present[g]) continue;
#pragma unroll
        for (int q = 0; q < 6; q++) box_dst[6 * g + q] = box_src[6 * g + q];
        off_dst[g] = off_src[g];
    }
}

}  // namespace

void launch_plan(const PlanArgs& a, cudaStream_t s) { plan_kernel<<<1, kPlanThreads, 0, s>>>(a); }

void launch_copy_layout(int G, const int* present, const int* box_src, const long long* off_src, int* box_dst,
                        long long* off_dst, cudaStream_t s) {
    copy_layout_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, present, box_src, off_src, box_dst, off_dst);
}


namespace {
// Sort keys of the work order: box voxels + 1 for the grains with a tile, 0 for the rest
// (all of them when the plan overflowed and gave no tiles).
__global__ void order_keys_kernel(int G, const int* toff_one, const int* box, int* keys, int* vals) {
    const bool none = toff_one[G + 1] == 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        int key = 0;
        if (g >= 1 && !none && toff_one[g + 1] - toff_one[g] > 0) {
            const Box b = load_box(box + 6 * g);
            key = (int)min(b.count() + 1, (long long)INT_MAX);
        }
        keys[g] = key;
        vals[g] = g;
    }
}
// Items per grain in order (item_off[i + 1]; item_off[0] = 0), summed afterwards.
__global__ void item_count_kernel(int G, const int* keys_out, int item_vox, int* item_off) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= G; i += gridDim.x * blockDim.x) {
        const long long v = (long long)keys_out[i] - 1;  // box voxels, -1: no tile
        item_off[i + 1] = v < 0 ? 0 : (item_vox > 0 ? (int)((v + item_vox - 1) / item_vox) : 1);
        if (i == 0) item_off[0] = 0;
    }
}
}  // namespace

size_t exclusive_scan_temp_bytes(int n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int*)nullptr, (int*)nullptr, n);
    return bytes;
}

void launch_exclusive_scan(void* temp, size_t temp_bytes, const int* in, int* out, int n, cudaStream_t s) {
    cub::DeviceScan::ExclusiveSum(temp, temp_bytes, in, out, n, s);
}

size_t work_order_temp_bytes(int G) {
    size_t sort = 0, scan = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, sort, (const int*)nullptr, (int*)nullptr,
                                              (const int*)nullptr, (int*)nullptr, G + 1);
    cub::DeviceScan::InclusiveSum(nullptr, scan, (const int*)nullptr, (int*)nullptr, G + 1);
    return sort > scan ? sort : scan;
}

void launch_work_order(const WorkOrder& w, int G, const int* toff_one, const int* box, int item_vox,
                       cudaStream_t s) {
    order_keys_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, toff_one, box, w.keys, w.vals);
    size_t bytes = w.temp_bytes;
    cub::DeviceRadixSort::SortPairsDescending(w.temp, bytes, w.keys, w.keys_out, w.vals, w.order, G + 1, 0,
                                              31, s);
    item_count_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, w.keys_out, item_vox, w.item_off);
    bytes = w.temp_bytes;
    cub::DeviceScan::InclusiveSum(w.temp, bytes, w.item_off + 1, w.item_off + 1, G + 1, s);
    cudaMemsetAsync(w.queue, 0, sizeof(int) * kQueues, s);
}

}  // namespace gg

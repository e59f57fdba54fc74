// gg_lists.cu -- comparison-list maintenance of every grain.
//
// Stands in for LSbox::computeSecondOrderNeighbours (box.cpp:1090-1134), called
// from grainhdl::updateSecondOrderNeighbors (grainhdl.cpp:1015-1027).  The new list
// is: the members of the previous list that still exist, in order; then every
// grain that appears in a member's own list, exists, is not the grain itself nor
// the boundary grain, and whose box touches this grain's box (inclusive overlap,
// box.cpp:880-889), in order of first appearance.
//
// The reference scans member lists pairwise with linear de-duplication.  Here one
// CTA per grain walks every (member i, entry j) of the neighbours' lists against two
// bitmaps over all grain IDs in shared memory: the previous list's existing members
// (plus the grain itself and the boundary grain), which most entries are, and the IDs
// already found not to qualify.  Whether an ID qualifies depends on the ID alone, so
// each distinct ID is checked about once, and only the qualifying new IDs go into a
// small hash keeping their smallest enumeration position i * cap + j.  Their first
// position overall is their first qualifying position; ranked by it, they come in
// the reference's order exactly.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr int kThreads = 512;
constexpr int kSel = 2048;          // new IDs of one grain per step
constexpr int kNewHash = 2 * kSel;  // slots of the new-ID hash (power of two)
constexpr unsigned kEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ int hash_slot(unsigned* hkey, unsigned id, int cap, int* err) {
    unsigned h = (id * 2654435761u) & (unsigned)(cap - 1);
    for (int probe = 0; probe < cap; probe++) {
        const unsigned prev = atomicCAS(hkey + h, kEmpty, id);
        if (prev == kEmpty || prev == id) return (int)h;
        h = (h + 1) & (unsigned)(cap - 1);
    }
    atomicOr(err, ERR_HASH);
    return -1;
}

__device__ __forceinline__ bool touch(const Box& a, const Box& b) {  // LSbox::checkIntersection
    return !(a.x0 > b.x1 || a.x1 < b.x0 || a.y0 > b.y1 || a.y1 < b.y0 || a.z0 > b.z1 || a.z1 < b.z0);
}

__global__ void __launch_bounds__(kThreads) update_lists_kernel(ListArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = list_bitmap_words(a.G);
    unsigned* member = reinterpret_cast<unsigned*>(smem_raw);  // W words
    unsigned* rejected = member + W;                          // W words
    unsigned* nkey = rejected + W;                            // kNewHash
    unsigned* npos = nkey + kNewHash;                         // kNewHash
    unsigned* sel_pos = npos + kNewHash;                      // kSel
    unsigned* sel_id = sel_pos + kSel;                        // kSel
    __shared__ int warp_sums[33];
    __shared__ int n_sel;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int total = a.toff[a.G + 1];
    const unsigned G = (unsigned)a.G;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int g = tile_grain(a.toff, a.G, t);
        const int K = a.n_son[g];
        const uint32_t* son = a.son + (long long)g * a.list_cap;
        uint32_t* cmp = a.cmp + (long long)g * a.list_cap;
        for (int q = threadIdx.x; q < 2 * W; q += blockDim.x) member[q] = 0u;
        for (int q = threadIdx.x; q < kNewHash; q += blockDim.x) { nkey[q] = kEmpty; npos[q] = kEmpty; }
        if (threadIdx.x == 0) n_sel = 0;
        __syncthreads();
        if (threadIdx.x == 0) {  // never candidates: the grain itself and the boundary grain
            atomicOr(member + (g >> 5), 1u << (g & 31));
            atomicOr(member, 1u);
        }
        // 1. existing members of the previous list, in order (block compaction)
        int prefix = 0;
        for (int base = 0; base < K; base += blockDim.x) {
            const int i = base + threadIdx.x;
            const unsigned id = i < K ? son[i] : 0u;
            const int f = (i < K && id <= G && a.exists[id]) ? 1 : 0;
            int incl = f;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += u;
            }
            if (lane == 31) warp_sums[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                const int w = lane < nw ? warp_sums[lane] : 0;
                int wi = w;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, wi, o);
                    if (lane >= o) wi += u;
                }
                if (lane < nw) warp_sums[lane] = wi - w;
                if (lane == 31) warp_sums[32] = wi;
            }
            __syncthreads();
            if (f) {
                const int pos = prefix + warp_sums[warp] + incl - f;
                if (pos < a.list_cap) cmp[pos] = id;
                atomicOr(member + (id >> 5), 1u << (id & 31));
            }
            prefix += warp_sums[32];
            __syncthreads();
        }
        // 2. every entry of every member's list: skip members and known rejects, check
        //    the rest (exists, box touches), keep the first position of each new ID
        const Box self = load_box(a.box + 6 * g);
        for (int i = warp; i < K; i += nw) {
            const unsigned c = son[i];
            if (c > G) continue;
            const int Kc = min(a.n_son[c], a.list_cap);
            const uint32_t* sc = a.son + (long long)c * a.list_cap;
            for (int j = lane; j < Kc; j += 32) {
                const unsigned id = sc[j];
                if (id > G) continue;
                const unsigned bit = 1u << (id & 31);
                if ((member[id >> 5] | rejected[id >> 5]) & bit) continue;
                if (!a.exists[id] || !touch(self, load_box(a.box + 6 * id))) {
                    atomicOr(rejected + (id >> 5), bit);
                    continue;
                }
                const int slot = hash_slot(nkey, id, kNewHash, a.err);
                if (slot >= 0) atomicMin(npos + slot, (unsigned)i * (unsigned)a.list_cap + (unsigned)j);
            }
        }
        __syncthreads();
        // 3. collect the new IDs
        for (int q = threadIdx.x; q < kNewHash; q += blockDim.x) {
            const unsigned id = nkey[q];
            if (id == kEmpty) continue;
            const int s = atomicAdd(&n_sel, 1);
            if (s < kSel) { sel_pos[s] = npos[q]; sel_id[s] = id; }
        }
        __syncthreads();
        // 4. append them by first position
        const int ns = min(n_sel, kSel);
        for (int q = threadIdx.x; q < ns; q += blockDim.x) {
            const unsigned pq = sel_pos[q];
            int rank = 0;
            for (int r = 0; r < ns; r++) rank += sel_pos[r] < pq;
            const int pos = prefix + rank;
            if (pos < a.list_cap) cmp[pos] = sel_id[q];
        }
        if (threadIdx.x == 0) {
            const int n = prefix + n_sel;
            if (n_sel > kSel || n > a.list_cap) atomicOr(a.err, ERR_LIST);
            a.n_cmp[g] = min(n, a.list_cap);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(128) pos_table_kernel(PosTableArgs a) {
    constexpr unsigned long long kFree = ~0ull;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const int K = a.n_cmp[g];
        const int size = pos_table_size(K, a.pos_cap);
        unsigned long long* tab = a.table + (long long)g * a.pos_cap;
        const uint32_t* list = a.cmp + (long long)g * a.list_cap;
        for (int q = threadIdx.x; q < size; q += blockDim.x) tab[q] = kFree;
        __syncthreads();
        for (int i = threadIdx.x; i < K; i += blockDim.x) {
            const uint32_t id = list[i];
            const unsigned long long e = ((unsigned long long)id << 32) | (unsigned)i;
            unsigned h = (id * 2654435761u) & (unsigned)(size - 1);
            int probe = 0;
            for (; probe < size; probe++) {
                if (atomicCAS(tab + h, kFree, e) == kFree) break;
                h = (h + 1) & (unsigned)(size - 1);
            }
            if (probe == size) atomicOr(a.err, ERR_HASH);
        }
        __syncthreads();
    }
}

// One warp per grain: the lanes test 32 candidate IDs at a time in ascending order and
// append the touching ones by ballot, so the row comes out sorted.
__global__ void __launch_bounds__(256) default_lists_kernel(DefaultListArgs a) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int g = 1 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); g <= a.G; g += warps) {
        uint32_t* cmp = a.cmp + (long long)g * a.list_cap;
        uint32_t* son = a.son + (long long)g * a.list_cap;
        int n = 0;
        if (a.present[g]) {
            const Box self = load_box(a.box + 6 * g);
            for (int o0 = 1; o0 <= a.G; o0 += 32) {
                const int o = o0 + lane;
                bool hit = false;
                if (o <= a.G && o != g && a.present[o]) hit = touch(self, load_box(a.box + 6 * o));
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                const int at = n + __popc(m & ((1u << lane) - 1));
                if (hit && at < a.list_cap) {
                    cmp[at] = (uint32_t)o;
                    son[at] = (uint32_t)o;
                }
                n += __popc(m);
            }
        }
        if (lane == 0) {
            if (n > a.list_cap) atomicOr(a.err, ERR_LIST);
            a.n_cmp[g] = a.n_son[g] = min(n, a.list_cap);
        }
    }
}

__global__ void scatter_lists_kernel(int G, const int64_t* offsets, const uint32_t* ids, uint32_t* cmp, int* n_cmp,
                                     uint32_t* son, int* n_son, int list_cap) {
    for (int g = blockIdx.x; g <= G; g += gridDim.x) {
        const long long o = g >= 1 ? offsets[g] : 0, len = g >= 1 ? offsets[g + 1] - o : 0;
        for (int k = threadIdx.x; k < len; k += blockDim.x) {
            cmp[(long long)g * list_cap + k] = ids[o + k];
            son[(long long)g * list_cap + k] = ids[o + k];
        }
        if (threadIdx.x == 0) n_cmp[g] = n_son[g] = (int)len;
    }
}

}  // namespace

void launch_default_lists(const DefaultListArgs& a, cudaStream_t s) {
    const int warps = a.G + 1;
    default_lists_kernel<<<(warps + 7) / 8, 256, 0, s>>>(a);
}

void launch_scatter_lists(int G, const int64_t* offsets, const uint32_t* ids, uint32_t* cmp, int* n_cmp,
                          uint32_t* son, int* n_son, int list_cap, cudaStream_t s) {
    scatter_lists_kernel<<<G + 1 < 4096 ? G + 1 : 4096, 128, 0, s>>>(G, offsets, ids, cmp, n_cmp, son, n_son,
                                                                   list_cap);
}

void launch_pos_tables(const PosTableArgs& a, int grid, cudaStream_t s) {
    pos_table_kernel<<<grid, 128, 0, s>>>(a);
}

void launch_update_lists(const ListArgs& a, int grid, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(update_lists_kernel);
    });
    const size_t smem = list_smem_bytes(a.G);
    update_lists_kernel<<<grid, kThreads, smem, s>>>(a);
}

}  // namespace gg

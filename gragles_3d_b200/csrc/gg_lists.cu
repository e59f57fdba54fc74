// gg_lists.cu -- comparison-list maintenance of every grain.
//
// Stands in for LSbox::computeSecondOrderNeighbours (box.cpp:1090-1134), called
// from grainhdl::updateSecondOrderNeighbors (grainhdl.cpp:1015-1027).  The new list
// is: the members of the previous list that still exist, in order; then every
// grain that appears in a member's own list, exists, is not the grain itself nor
// the boundary grain, and whose box touches this grain's box (inclusive overlap,
// box.cpp:880-889), in order of first appearance.
//
// The reference scans member lists pairwise with linear de-duplication: with K members
// of K entries each that is K^2 entries per grain, most of them members already.  Here
// one CTA per grain turns it around.  A new ID must exist and touch the grain's box, so
// the candidates are the existing grains binned in the domain cells the grain's
// inclusive box reaches (kListCell^3 cells, binned once per step); a bitmap over all IDs
// in shared memory holds the previous list's existing members (plus the grain itself and
// the boundary grain) and another the IDs already seen, so each distinct ID is checked
// once.  A candidate is kept when some member's list holds it: its first enumeration
// position i * cap + j is the first member i (in list order) whose list holds it, found
// through the members' position tables (built from the previous lists before the
// update), and j its place there.  Ranked by that position, the new IDs come in the
// reference's order exactly.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr int kThreads = 512;
constexpr int kSel = 2048;          // candidate IDs of one grain per step
constexpr unsigned kEmpty = 0xFFFFFFFFu;

// Position of `id` in the list whose position table is tab (size slots), or -1.
__device__ __forceinline__ int table_position(const unsigned long long* __restrict__ tab, int size, uint32_t id) {
    unsigned h = (id * 2654435761u) & (unsigned)(size - 1);
    for (int probe = 0; probe < size; probe++) {
        const unsigned long long e = __ldg(tab + h);
        const uint32_t k = (uint32_t)(e >> 32);
        if (k == id) return (int)(e & 0xFFFFFFFFu);
        if (k == kEmpty) return -1;
        h = (h + 1) & (unsigned)(size - 1);
    }
    return -1;
}

__device__ __forceinline__ bool touch(const Box& a, const Box& b) {  // LSbox::checkIntersection
    return !(a.x0 > b.x1 || a.x1 < b.x0 || a.y0 > b.y1 || a.y1 < b.y0 || a.z0 > b.z1 || a.z1 < b.z0);
}

__global__ void __launch_bounds__(kThreads) update_lists_kernel(ListArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = list_bitmap_words(a.G);
    unsigned* member = reinterpret_cast<unsigned*>(smem_raw);  // W words
    unsigned* seen = member + W;                              // W words
    unsigned* sel_pos = seen + W;                             // kSel
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
        // 2. candidates: the existing grains binned in the cells of the grain's inclusive
        //    box that are not members, seen once each, whose boxes touch (box.cpp:880-889)
        const Box self = load_box(a.box + 6 * g);
        const TileBins& cb = a.cells;
        const int n = cb.ntx;
        const int cx0 = max(self.x0, 0) / kListCell, cx1 = min(max(self.x1, 0) / kListCell, n - 1);
        const int cy0 = max(self.y0, 0) / kListCell, cy1 = min(max(self.y1, 0) / kListCell, n - 1);
        const int cz0 = max(self.z0, 0) / kListCell, cz1 = min(max(self.z1, 0) / kListCell, n - 1);
        const int ncx = cx1 - cx0 + 1, ncy = cy1 - cy0 + 1, ncells = ncx * ncy * (cz1 - cz0 + 1);
        for (int c = warp; c < ncells; c += nw) {
            const int cx = cx0 + c % ncx, cy = cy0 + (c / ncx) % ncy, cz = cz0 + c / (ncx * ncy);
            const int cell = (cz * n + cy) * n + cx;
            const int e0 = cb.off[cell], e1 = cb.off[cell + 1];
            for (int e = e0 + lane; e < e1; e += 32) {
                const unsigned id = cb.entries[e];
                if (id > G || id == 0u) continue;
                const unsigned bit = 1u << (id & 31);
                if ((member[id >> 5] | seen[id >> 5]) & bit) continue;
                if (atomicOr(seen + (id >> 5), bit) & bit) continue;  // another lane has it
                if (!touch(self, load_box(a.box + 6 * id))) continue;
                const int slot = atomicAdd(&n_sel, 1);
                if (slot < kSel) sel_id[slot] = id;
            }
        }
        __syncthreads();
        // 3. the first enumeration position of each candidate: the first member (in list
        //    order) whose list holds it, 32 members per round, and its place there
        const int nc = min(n_sel, kSel);
        for (int q = warp; q < nc; q += nw) {
            const uint32_t id = sel_id[q];
            unsigned key = kEmpty;
            for (int i0 = 0; i0 < K; i0 += 32) {
                const int i = i0 + lane;
                int pos = -1;
                if (i < K) {
                    const unsigned c = son[i];
                    if (c <= G) {
                        const int Kc = min(a.n_son[c], a.list_cap);
                        pos = table_position(a.pos + (long long)c * a.pos_cap, pos_table_size(Kc, a.pos_cap), id);
                        if (pos >= Kc) pos = -1;
                    }
                }
                const unsigned hit = __ballot_sync(0xffffffffu, pos >= 0);
                if (hit) {
                    const int f = __ffs(hit) - 1;
                    const int pf = __shfl_sync(0xffffffffu, pos, f);
                    key = (unsigned)(i0 + f) * (unsigned)a.list_cap + (unsigned)pf;
                    break;
                }
            }
            if (lane == 0) sel_pos[q] = key;
        }
        __syncthreads();
        // 4. append the held ones by first position
        for (int q = threadIdx.x; q < nc; q += blockDim.x) {
            const unsigned pq = sel_pos[q];
            if (pq == kEmpty) continue;
            int rank = 0;
            for (int r = 0; r < nc; r++) rank += sel_pos[r] < pq;
            const int pos = prefix + rank;
            if (pos < a.list_cap) cmp[pos] = sel_id[q];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int held = 0;
            for (int r = 0; r < nc; r++) held += sel_pos[r] != kEmpty;
            n_sel = n_sel > kSel ? -1 : held;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int total_n = prefix + max(n_sel, 0);
            if (n_sel < 0 || total_n > a.list_cap) atomicOr(a.err, ERR_LIST);
            a.n_cmp[g] = min(total_n, a.list_cap);
        }
        __syncthreads();
    }
}

__device__ void build_pos_table(const PosTableArgs& a, int g) {
    constexpr unsigned long long kFree = ~0ull;
    {
        const int K = min(a.n_cmp[g], a.list_cap);
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

__global__ void __launch_bounds__(128) pos_table_kernel(PosTableArgs a) {
    if (a.toff) {
        for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) build_pos_table(a, w.g);
    } else {
        for (int g = 1 + blockIdx.x; g <= a.G; g += gridDim.x)
            if (a.present[g]) build_pos_table(a, g);  // uniform across the CTA
    }
}

// Cells of kListCell^3 voxels per existing grain's inclusive box; one warp per grain.
template <bool FILL>
__global__ void cell_bin_kernel(TileBins tb, int G, const int* exists, const int* box, int* err) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int n = tb.ntx;
    for (int g = 1 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); g <= G; g += warps) {
        if (!exists[g]) continue;
        const Box b = load_box(box + 6 * g);
        if (b.nx() <= 0) continue;
        const int cx0 = max(b.x0, 0) / kListCell, cx1 = min(max(b.x1, 0) / kListCell, n - 1);
        const int cy0 = max(b.y0, 0) / kListCell, cy1 = min(max(b.y1, 0) / kListCell, n - 1);
        const int cz0 = max(b.z0, 0) / kListCell, cz1 = min(max(b.z1, 0) / kListCell, n - 1);
        const int ncx = cx1 - cx0 + 1, ncy = cy1 - cy0 + 1, nn = ncx * ncy * (cz1 - cz0 + 1);
        for (int i = lane; i < nn; i += 32) {
            const int cell = ((cz0 + i / (ncx * ncy)) * n + cy0 + (i / ncx) % ncy) * n + cx0 + i % ncx;
            if (!FILL) {
                atomicAdd(tb.count + cell, 1);
            } else {
                const long long slot = tb.off[cell] + atomicAdd(tb.cursor + cell, 1);
                if (slot < tb.capacity) tb.entries[slot] = (uint32_t)g;
                else atomicOr(err, ERR_POOL);
            }
        }
    }
}

// Exclusive scan of the cell counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) cell_scan_kernel(TileBins tb, int n_cells, int* err) {
    __shared__ long long sums[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (n_cells + blockDim.x - 1) / blockDim.x;
    const int t0 = threadIdx.x * per, t1 = min(n_cells, t0 + per);
    long long mine = 0;
    for (int t = t0; t < t1; t++) mine += tb.count[t];
    long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) sums[warp] = incl;
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
    }
    __syncthreads();
    long long run = sums[warp] + incl - mine;
    for (int t = t0; t < t1; t++) {
        tb.off[t] = (int)run;
        run += tb.count[t];
    }
    if (threadIdx.x == 0) {
        tb.off[n_cells] = (int)sums[32];
        if (sums[32] > tb.capacity) atomicOr(err, ERR_POOL);
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

void launch_list_bins(const TileBins& tb, int G, const int* exists, const int* box, int* err, cudaStream_t s) {
    const int n_cells = tb.ntx * tb.nty * tb.ntz;
    cudaMemsetAsync(tb.count, 0, sizeof(int) * (n_cells + 1), s);
    cudaMemsetAsync(tb.cursor, 0, sizeof(int) * (n_cells + 1), s);
    const int grid = (G + 4) / 4;  // one warp per grain, 4 warps per block
    cell_bin_kernel<false><<<grid, 128, 0, s>>>(tb, G, exists, box, err);
    cell_scan_kernel<<<1, 1024, 0, s>>>(tb, n_cells, err);
    cell_bin_kernel<true><<<grid, 128, 0, s>>>(tb, G, exists, box, err);
}

long long list_bin_capacity(int G, int side) {
    const long long c = side / kListCell + 2;  // cells an inclusive box of `side` reaches per axis
    return (long long)G * c * c * c;
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

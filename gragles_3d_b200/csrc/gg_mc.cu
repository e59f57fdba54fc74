// gg_mc.cu -- zero-isosurface extraction and hull statistics of every grain.
//
// Stands in for grainhdl::level_set's per-grain work (grainhdl.cpp:669-718):
// deleting grains whose hull vanished in the previous step, then
// LSbox::extractContour (box.cpp:1144-1161) = MarchingCubesAlgorithm::generateHull
// (marchingCubes.cpp:364-478), GrainHull::generateHull (grainHull.cpp:146-155),
// computeGrainVolume / computeSurfaceArea (grainHull.cpp:40-55, 120-131) and the
// resize of the output box to the new bounding box (dimensionalBuffer.h:120-219).
//
// One CTA owns one grain and walks its cubes in the reference's z, y, x order in
// slabs of whole cube layers.  A slab's voxel signs are staged as bits (a warp ballot
// per 32 voxels); 32 cubes of a row are classified at once from their corners' bit
// vectors, and only the active cubes (not all corners alike) are listed, in cube
// order, and processed further.  A block scan of per-cube triangle counts gives each
// triangle its place in the reference's emission order; the FP64 volume and area
// terms of a chunk are then added by one thread in that order, so the sums are
// bit-identical to the reference's sequential loop.  The distinct neighbour IDs
// keep the reference's first-seen order through a shared-memory hash holding, per
// ID, the smallest (cube index, rank in the cube's sorted list) key.
#include "gg_kernels.cuh"

namespace gg {

#include "gg_mc_tables.inc"

namespace {

constexpr int kThreads = 256;
constexpr int kHash = 1024;  // distinct neighbour IDs per grain (power of two)
static_assert(kThreads * 5 * sizeof(double) >= 2 * kHash * sizeof(unsigned), "ID collection aliases the volume buffer");
constexpr int kSlabBytes = 36 * 1024;  // shared memory for a slab's sign bytes and cube lists

// cubeindex bit q <-> corner offset (dx, dy, dz), marchingCubes.cpp:376-385:
// (0,0,1) (1,0,1) (1,0,0) (0,0,0) (0,1,1) (1,1,1) (1,1,0) (0,1,0); compile-time
// functions, so that every unrolled corner offset folds into the address.
__host__ __device__ constexpr int corner_dx(int q) { return ((q & 3) == 1 || (q & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int corner_dy(int q) { return q >> 2; }
__host__ __device__ constexpr int corner_dz(int q) { return (q & 3) < 2 ? 1 : 0; }
// edge e joins corners (edge_a(e), edge_b(e)) in VertexInterp argument order,
// marchingCubes.cpp:392-469: (0,1) (1,2) (2,3) (3,0) (4,5) (5,6) (6,7) (7,4) (0,4) (1,5) (2,6) (3,7)
__host__ __device__ constexpr int edge_a(int e) { return e < 8 ? e : e - 8; }
__host__ __device__ constexpr int edge_b(int e) { return e < 8 ? ((e & 4) | ((e + 1) & 3)) : e - 4; }
// neighbour-list corner order, marchingCubes.cpp:505-553:
// (0,0,0) (1,0,0) (1,1,0) (0,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1)
__host__ __device__ constexpr int nbc_dx(int k) { return ((k & 3) == 1 || (k & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int nbc_dy(int k) { return (k & 3) >= 2 ? 1 : 0; }
__host__ __device__ constexpr int nbc_dz(int k) { return k >> 2; }
static_assert(corner_dx(1) == 1 && corner_dz(2) == 0 && corner_dy(7) == 1 && corner_dz(4) == 1, "corner table");
static_assert(edge_b(3) == 0 && edge_b(7) == 4 && edge_b(6) == 7 && edge_a(11) == 3 && edge_b(11) == 7, "edge table");
static_assert(nbc_dx(2) == 1 && nbc_dy(3) == 1 && nbc_dx(3) == 0 && nbc_dz(5) == 1, "neighbour corner table");
// A cube crosses the zero level unless its 8 corners agree: the edge table is 0 exactly
// for cube indices 0 and 255, so the active cubes are found from the corners' sign bits
// alone (any & ~all over the eight corner bit vectors of a row of 32 cubes).

struct V3 { double x, y, z; };

// MarchingCubesAlgorithm::VertexInterp, marchingCubes.cpp:484-499
__device__ __forceinline__ V3 vinterp(V3 p1, V3 p2, double v1, double v2) {
    if (fabs(v1) < 0.00001) return p1;
    if (fabs(v2) < 0.00001) return p2;
    if (fabs(v1 - v2) < 0.00001) return p1;
    const double mu = v1 / (v1 - v2);
    return V3{p1.x + mu * (p2.x - p1.x), p1.y + mu * (p2.y - p1.y), p1.z + mu * (p2.z - p1.z)};
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < nw ? warp_sums[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < nw) warp_sums[lane] = wi - w;
        if (lane == nw - 1) warp_sums[32] = wi;
    }
    __syncthreads();
    total = warp_sums[32];
    const int r = warp_sums[warp] + incl - v;
    __syncthreads();  // warp_sums is reused by the next scan
    return r;
}

__device__ __forceinline__ void hash_insert(unsigned* hkey, unsigned* hval, unsigned id, unsigned key, int* err) {
    unsigned h = (id * 2654435761u) & (kHash - 1);
    for (int probe = 0; probe < kHash; probe++) {
        const unsigned prev = atomicCAS(hkey + h, 0xFFFFFFFFu, id);
        if (prev == 0xFFFFFFFFu || prev == id) {
            atomicMin(hval + h, key);
            return;
        }
        h = (h + 1) & (kHash - 1);
    }
    atomicOr(err, ERR_NEIGHBORS);
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 3) mc_kernel(MCArgs<T> a, int slab_bytes) {
    __shared__ double vbuf[kThreads * 5];
    __shared__ double abuf[kThreads * 5];
    __shared__ int warp_sums[33];
    __shared__ unsigned hkey[kHash];
    __shared__ unsigned hval[kHash];
    // the cube tables, read per active cube with scattered indices: triangle edges as
    // nibbles with the triangle count in bits 60-63, and the edge masks
    __shared__ unsigned long long s_tri[256];
    __shared__ unsigned short s_edge[256];
    __shared__ unsigned g_key;  // the grain's own ID: its smallest key (first active cube)
    __shared__ int n_found;
    __shared__ int next_item;
    extern __shared__ __align__(16) unsigned char slab_raw[];
    const int n_items = a.item_off[a.G + 1];
    for (int ci = threadIdx.x; ci < 256; ci += blockDim.x) {
        unsigned long long t = 0;
        int k = 0;
        while (k < 15 && gg_mc_tri_table[ci][k] != -1) {
            t |= (unsigned long long)gg_mc_tri_table[ci][k] << (4 * k);
            k++;
        }
        s_tri[ci] = t | ((unsigned long long)(k / 3) << 60);
        s_edge[ci] = (unsigned short)gg_mc_edge_table[ci];
    }
    for (;;) {  // grains largest first, fetched on demand
        __syncthreads();
        if (threadIdx.x == 0) next_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int t = next_item;
        if (t >= n_items) break;
        const int g = a.order[work_position(a.item_off, a.G, t)];
        if (g < 1 || g > a.G) continue;
        if (!a.exists[g] && !a.regrid) {  // the hull vanished last step: delete, grainhdl.cpp:678-680
            if (threadIdx.x == 0) a.present[g] = 0;
            continue;
        }
        const Box b = a.in.grain_box(g);
        const T* sdf = a.in.grain_ptr(g);
        const uint32_t* idl = a.idl + a.idoff[g];
        for (int q = threadIdx.x; q < kHash; q += blockDim.x) { hkey[q] = 0xFFFFFFFFu; hval[q] = 0xFFFFFFFFu; }
        if (threadIdx.x == 0) {
            n_found = 0;
            g_key = 0xFFFFFFFFu;
        }
        const int ncx = b.nx() - 1, ncy = b.ny() - 1, ncz = b.nz() - 1;
        const int ncplane = (ncx > 0 && ncy > 0 && ncz > 0) ? ncx * ncy : 0;
        double vol = 0.0, area = 0.0;
        long long ntri = 0;
        int nrec = 0;  // active cubes so far (hull capture)
        const bool capture = a.hull.cap > 0;
        const long long hbase = (long long)g * a.hull.cap;
        const int nxb = b.nx(), plane = b.nx() * b.ny();
        // Slabs of LZ cube layers.  The signs of their LZ + 1 voxel layers are staged as
        // bits (one coalesced load per voxel, a warp ballot per 32 voxels in x, y, z
        // order); a row of 32 cubes is active where its 8 corner bit vectors disagree,
        // found with a few word operations; the active cubes are listed in cube order.
        const int wr = (ncx + 31) >> 5;          // active-mask words per cube row
        const int pw = (plane + 31) >> 5;        // sign words per voxel layer (bound)
        int LZ = ncplane > 0 ? (slab_bytes - 4 * pw - 16) / (4 * pw + 4 * ncy * wr + 2 * ncplane + 4) : 0;
        if (ncplane > 0 && LZ > 65535 / ncplane) LZ = 65535 / ncplane;
        if (LZ > ncz) LZ = ncz;
        if (ncplane > 0 && LZ < 1) {  // a single layer does not fit the shared memory
            if (threadIdx.x == 0) atomicOr(a.err, ERR_BOX);
            LZ = 0;
        }
        unsigned* sb = reinterpret_cast<unsigned*>(slab_raw);  // sign bits of the slab's voxels
        const int sbw = ((LZ + 1) * plane + 31) / 32 + 1;      // + 1: 32-bit reads at any bit
        unsigned* am = sb + sbw;                                // active bits, wr words per cube row
        unsigned short* act = reinterpret_cast<unsigned short*>(am + LZ * ncy * wr);
        __syncthreads();
        for (int zc0 = 0; LZ > 0 && zc0 < ncz; zc0 += LZ) {
          const int lz = min(LZ, ncz - zc0);
          // sign bits of voxel layers zc0 .. zc0 + lz (inside = value >= 0, marchingCubes.cpp:12-15)
          {
              const T* src = sdf + (long long)zc0 * plane;
              const int nv = (lz + 1) * plane;
              constexpr int kMB = sizeof(T) == 4 ? 16 : 8;  // loads in flight per thread
              for (int v0 = 0; v0 < nv; v0 += kMB * kThreads) {
                  T r[kMB];
#pragma unroll
                  for (int u = 0; u < kMB; u++) {
                      const int v = v0 + u * kThreads + threadIdx.x;
                      r[u] = v < nv ? src[v] : T(-1);
                  }
#pragma unroll
                  for (int u = 0; u < kMB; u++) {
                      const unsigned m = __ballot_sync(0xffffffffu, r[u] >= T(0));
                      const int w0 = v0 + u * kThreads + (threadIdx.x & ~31);  // a multiple of 32
                      if ((threadIdx.x & 31) == 0 && w0 < nv) sb[w0 >> 5] = m;
                  }
              }
          }
          __syncthreads();
          // active bits: word j of cube row (cz, cy) covers cubes x = 32 j .. 32 j + 31
          const int nrow = lz * ncy, nw = nrow * wr;
          for (int q = threadIdx.x; q < nw; q += kThreads) {
              const int row = q / wr, j = q - row * wr;
              const int cz = row / ncy, cy = row - cz * ncy;
              const int v0 = (cz * ncy + cy + cz) * nxb + 32 * j;  // voxel (32 j, cy, cz): (cz ny + cy) nx
              unsigned all = 0xffffffffu, any = 0u;
#pragma unroll
              for (int c = 0; c < 8; c++) {
                  const int v = v0 + corner_dz(c) * plane + corner_dy(c) * nxb + corner_dx(c);
                  const unsigned bits = __funnelshift_r(sb[v >> 5], sb[(v >> 5) + 1], v & 31);
                  all &= bits;
                  any |= bits;
              }
              const int left = ncx - 32 * j;
              const unsigned valid = left >= 32 ? 0xffffffffu : (1u << left) - 1u;
              am[q] = any & ~all & valid;
          }
          __syncthreads();
          // the active cubes in cube order: thread t takes words [t seg, (t + 1) seg)
          const int seg = (nw + kThreads - 1) / kThreads;
          const int s0 = threadIdx.x * seg, s1 = min(s0 + seg, nw);
          int nloc = 0;
          for (int m = s0; m < s1; m++) nloc += __popc(am[m]);
          int n_act;
          int w = block_exclusive_scan(nloc, warp_sums, n_act);
          for (int m = s0; m < s1; m++) {
              const int row = m / wr, x0 = 32 * (m - row * wr);
              for (unsigned bits = am[m]; bits; bits &= bits - 1)
                  act[w++] = (unsigned short)(row * ncx + x0 + __ffs(bits) - 1);
          }
          __syncthreads();
          for (int ab = 0; ab < n_act; ab += kThreads) {
            const int ia = ab + threadIdx.x;
            int nt = 0, ci = 0;
            int x = 0, y = 0, z = 0, base = 0;
            int c = 0;
            double val[8];
            if (ia < n_act) {
                const int cl = act[ia];
                c = zc0 * ncplane + cl;  // cube index in the reference's z, y, x order
                const int lzl = cl / ncplane, rem = cl - lzl * ncplane;
                const int ly = rem / ncx, lx = rem - ly * ncx, lzz = zc0 + lzl;
                const int sv = (lzl * ncy + ly + lzl) * nxb + lx;  // slab-relative voxel of the cube
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int v = sv + corner_dz(q) * plane + corner_dy(q) * nxb + corner_dx(q);
                    ci |= (int)((sb[v >> 5] >> (v & 31)) & 1u) << q;
                }
                x = b.x0 + lx;
                y = b.y0 + ly;
                z = b.z0 + lzz;
                base = lzz * plane + ly * nxb + lx;
#pragma unroll
                for (int k = 0; k < 8; k++)
                    val[k] = (double)sdf[base + corner_dz(k) * plane + corner_dy(k) * nxb + corner_dx(k)];
                nt = (int)(s_tri[ci] >> 60);
            }
            int chunk_total;
            const int off = block_exclusive_scan(nt, warp_sums, chunk_total);
            unsigned lst[8];
            int cnt = 0;
            if (nt > 0) {
                const int et = s_edge[ci];
                const unsigned long long tri = s_tri[ci];
                V3 vl[12];
#pragma unroll
                for (int e = 0; e < 12; e++) {
                    if (!(et & (1 << e))) continue;
                    const int ka = edge_a(e), kb = edge_b(e);
                    const V3 p1{(double)(x + corner_dx(ka)), (double)(y + corner_dy(ka)), (double)(z + corner_dz(ka))};
                    const V3 p2{(double)(x + corner_dx(kb)), (double)(y + corner_dy(kb)), (double)(z + corner_dz(kb))};
                    vl[e] = vinterp(p1, p2, val[ka], val[kb]);
                }
                for (int q = 0; q < nt; q++) {
                    const V3 p0 = vl[(tri >> (12 * q)) & 15];
                    const V3 p1 = vl[(tri >> (12 * q + 4)) & 15];
                    const V3 p2 = vl[(tri >> (12 * q + 8)) & 15];
                    if (capture) {  // Triangle::computeBarycenter, triangle.h:12-18
                        const long long ti = ntri + off + q;
                        if (ti < a.hull.cap) {
                            double* bb = a.hull.bary + 3 * (hbase + ti);
                            bb[0] = (p0.x + p1.x + p2.x) / 3;
                            bb[1] = (p0.y + p1.y + p2.y) / 3;
                            bb[2] = (p0.z + p1.z + p2.z) / 3;
                        } else {
                            { atomicOr(a.err, ERR_HULL); atomicOr(a.hull.diag, HULL_TRIANGLES); }
                        }
                    }
                    // GrainHull::computeGrainVolume, grainHull.cpp:42-51
                    const double v321 = p2.x * p1.y * p0.z;
                    const double v231 = p1.x * p2.y * p0.z;
                    const double v312 = p2.x * p0.y * p1.z;
                    const double v132 = p0.x * p2.y * p1.z;
                    const double v213 = p1.x * p0.y * p2.z;
                    const double v123 = p0.x * p1.y * p2.z;
                    vbuf[off + q] = (double)(1.0f / 6.0f) * (-v321 + v231 + v312 - v132 - v213 + v123);
                    // GrainHull::computeSurfaceArea, grainHull.cpp:122-127 (Eigen sums c0 + (c1 + c2))
                    const double abx = p0.x - p1.x, aby = p0.y - p1.y, abz = p0.z - p1.z;
                    const double bcx = p0.x - p2.x, bcy = p0.y - p2.y, bcz = p0.z - p2.z;
                    const double cx = aby * bcz - abz * bcy, cy = abz * bcx - abx * bcz, cz = abx * bcy - aby * bcx;
                    abuf[off + q] = sqrt(cx * cx + (cy * cy + cz * cz)) / 2.0;
                    if (capture && ntri + off + q < a.hull.cap) a.hull.tarea[hbase + ntri + off + q] = abuf[off + q];
                }
                // generateAdditionalInformation: sorted distinct corner IDs, marchingCubes.cpp:501-583
                // (the eight IDs loaded first, then an insertion sort in registers)
                unsigned ids[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int at = base + nbc_dz(k) * plane + nbc_dy(k) * nxb + nbc_dx(k);
                    // inside = value >= 0: the staged sign bit of the corner (slab-relative)
                    const int sat = at - zc0 * plane;
                    const unsigned outside_id = idl[at];
                    ids[k] = ((sb[sat >> 5] >> (sat & 31)) & 1u) ? (unsigned)g : outside_id;
                }
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    unsigned id = ids[k];
                    bool found = false;
#pragma unroll
                    for (int q = 0; q < k; q++) found |= q < cnt && lst[q] == id;
                    if (!found) {
#pragma unroll
                        for (int q = 0; q < k; q++)
                            if (q < cnt && id < lst[q]) { const unsigned tmp = lst[q]; lst[q] = id; id = tmp; }
#pragma unroll
                        for (int q = 0; q <= k; q++)
                            if (q == cnt) lst[q] = id;
                        cnt++;
                    }
                }
                if (threadIdx.x == 0) {  // the chunk's first cube; the first chunk's is the grain's first
#pragma unroll
                    for (int q = 0; q < 8; q++)
                        if (q < cnt && lst[q] == (unsigned)g) g_key = min(g_key, ((unsigned)c << 3) | q);
                }
                if (capture) {  // the cube's list, in cube order, for the interfacial elements
                    const int ri = nrec + ia;
                    if (ri < a.hull.cap) {
                        uint32_t* rl = a.hull.rec_list + 8 * (hbase + ri);
#pragma unroll
                        for (int q = 0; q < 8; q++) rl[q] = q < cnt ? lst[q] : 0xFFFFFFFFu;
                        a.hull.rec_ntri[hbase + ri] = nt;
                    } else {
                        { atomicOr(a.err, ERR_HULL); atomicOr(a.hull.diag, HULL_RECORDS); }
                    }
                }
            }
            {
                // the IDs other than g into the hash, key (cube << 3 | rank): one insert per
                // distinct ID per warp and round, with the warp's smallest key for it
                const int lane = threadIdx.x & 31;
                const unsigned ck = (unsigned)c << 3;
                const int rounds = __reduce_max_sync(0xffffffffu, cnt);
                for (int r = 0; r < rounds; r++) {
                    unsigned id = 0xFFFFFFFFu;
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == r && k < cnt) id = lst[k];
                    if (id == (unsigned)g) id = 0xFFFFFFFFu;
                    const unsigned key = id != 0xFFFFFFFFu ? (ck | (unsigned)r) : 0xFFFFFFFFu;
                    const unsigned grp = __match_any_sync(0xffffffffu, id);
                    const unsigned kmin = __reduce_min_sync(grp, key);
                    if (id != 0xFFFFFFFFu && lane == __ffs(grp) - 1) hash_insert(hkey, hval, id, kmin, a.err);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {  // in triangle order; eight terms' loads in flight at a time
                int q = 0;
                for (; q + 8 <= chunk_total; q += 8) {
                    double tv[8], ta[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        tv[u] = vbuf[q + u];
                        ta[u] = abuf[q + u];
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        vol += tv[u];
                        area += ta[u];
                    }
                }
                for (; q < chunk_total; q++) {
                    vol += vbuf[q];
                    area += abuf[q];
                }
            }
            ntri += chunk_total;
            __syncthreads();
          }
          nrec += n_act;
        }
        // collect the distinct IDs and order them by first appearance (g with its key first)
        if (threadIdx.x == 0 && g_key != 0xFFFFFFFFu) hash_insert(hkey, hval, (unsigned)g, g_key, a.err);
        __syncthreads();
        unsigned* nb_id = reinterpret_cast<unsigned*>(vbuf);  // the chunk buffers are done with
        unsigned* nb_key = nb_id + kHash;
        for (int q = threadIdx.x; q < kHash; q += blockDim.x) {
            if (hkey[q] != 0xFFFFFFFFu) {
                const int slot = atomicAdd(&n_found, 1);
                nb_id[slot] = hkey[q];
                nb_key[slot] = hval[q];
            }
        }
        __syncthreads();
        const int nf = n_found;
        uint32_t* nbo = a.nb + (long long)g * a.nb_cap;
        for (int q = threadIdx.x; q < nf; q += blockDim.x) {
            const unsigned kq = nb_key[q];
            int rank = 0;
            for (int r = 0; r < nf; r++) rank += nb_key[r] < kq;
            if (rank < a.nb_cap) nbo[rank] = nb_id[q];
        }
        if (threadIdx.x == 0) {
            if (nf > a.nb_cap) atomicOr(a.err, ERR_NEIGHBORS);
            a.n_nb[g] = nf;
            if (capture) {
                a.hull.n_rec[g] = nrec < a.hull.cap ? nrec : a.hull.cap;
                a.hull.n_tri[g] = ntri < a.hull.cap ? (int)ntri : a.hull.cap;
            }
            const double h = a.geo.h;
            a.volume[g] = fabs(vol) * h * h * h;
            a.surface[g] = area * h * h;
            const bool ex = ntri > 0;
            a.exists[g] = ex;
            if (ex) {
                // tail of executeSetComparison (box.cpp:858-877), then extractContour's resize
                const int* nbx = a.newbox + 6 * g;
                const int gb = a.regrid ? 0 : a.geo.gb, M = a.geo.M;
                int x0 = nbx[0] - gb, x1 = nbx[1] + gb, y0 = nbx[2] - gb, y1 = nbx[3] + gb;
                int z0 = nbx[4] - gb, z1 = nbx[5] + gb;
                if (!a.regrid) {  // the clamp of executeSetComparison (box.cpp:868-877)
                    if (x0 < 0) x0 = 0;
                    if (y0 < 0) y0 = 0;
                    if (z0 < 0) z0 = 0;
                    if (x1 >= M) x1 = M - 1;
                    if (y1 >= M) y1 = M - 1;
                    if (z1 >= M) z1 = M - 1;
                }
                const Box nb = resize_to_cube(Box{x0, x1, y0, y1, z0, z1}, M);
                if (nb.x0 < 0 || nb.y0 < 0 || nb.z0 < 0 || nb.nx() <= 0) atomicOr(a.err, ERR_BOX);
                store_box(a.out_box + 6 * g, nb);
            }
        }
        __syncthreads();
    }
}

// out3 = {present grains, present and existing grains, largest box side among those}
__global__ void count_kernel(int G, const int* present, const int* exists, const int* box, int* out3) {
    int np = 0, ne = 0, mx = 0;
    for (int g = 1 + blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        np += present[g] != 0;
        if (present[g] && exists[g]) {
            ne++;
            mx = max(mx, box[6 * g + 1] - box[6 * g]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        np += __shfl_xor_sync(0xffffffffu, np, o);
        ne += __shfl_xor_sync(0xffffffffu, ne, o);
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out3, np);
        atomicAdd(out3 + 1, ne);
        atomicMax(out3 + 2, mx);
    }
}

}  // namespace

size_t mc_slab_bytes(int side) {
    // at least one cube layer: two voxel layers of sign bits, the cube layer's active bits
    // and a list entry per cube
    const size_t n = side > 1 ? side : 2;
    const size_t pw = (n * n + 31) / 32, wr = (n - 1 + 31) / 32;
    const size_t one_layer = 8 * pw + 16 + 4 * (n - 1) * wr + 2 * (n - 1) * (n - 1) + 4;
    return one_layer > kSlabBytes ? one_layer : kSlabBytes;
}

template <typename T>
void launch_mc(const MCArgs<T>& a, int grid, int side, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(mc_kernel<T>);
    });
    const size_t bytes = mc_slab_bytes(side);
    mc_kernel<T><<<grid, kThreads, bytes, s>>>(a, (int)bytes);
}

void launch_count(int G, const int* present, const int* exists, const int* box, int* out3, cudaStream_t s) {
    cudaMemsetAsync(out3, 0, 3 * sizeof(int), s);
    count_kernel<<<64, 256, 0, s>>>(G, present, exists, box, out3);
}

template void launch_mc<double>(const MCArgs<double>&, int, int, cudaStream_t);
template void launch_mc<float>(const MCArgs<float>&, int, int, cudaStream_t);

}  // namespace gg

// gg_hull.cu -- interfacial elements of every grain hull and the convolution correction.
//
// Stands in for LSbox::computeSurfaceElements (box.cpp:1175-1180) =
// GrainHull::computeGrainBoundaryElements, subDivideTrianglesToInterfacialElements,
// computeJunctionPosition and mergeJunction (grainHull.cpp:187-275, 483-531) with the
// element energies and mobilities of InterfacialElement.cpp:23-456, and for the
// convolution correction of LSbox::executeConvolution (box.cpp:426-535) with
// GrainHull::projectPointToGrainBoundary (grainHull.cpp:570-660).
//
//   elements_kernel: one warp per grain (the hull is small: ~10^3 triangles, ~10^2
//     distinct neighbour lists).  The warp dedupes the cube lists the marching-cubes
//     kernel captured (first-seen order = the reference's list keys), groups the
//     triangle barycenters by list (stable, in triangle order), builds one element per
//     list with its energy and mobility, merges junctions closer than 2 voxels exactly
//     as the reference does (including its ID-list quirks), and writes the elements in
//     search order with their barycenter segments, bounding boxes and an ID -> elements
//     index.
//   correction_kernel: a CTA per grain, with the grain's element index, element boxes
//     and FP32 barycenters staged in shared memory; pass by pass over runs of the box's
//     voxels, those with |input| < delta are grouped by IDLocal neighbour, and a warp
//     takes 32 voxels of one neighbour at a time.  The winner of the reference's search is the least (distance, element
//     index) over the barycenters of the elements holding that neighbour.  The warp
//     finds it with an FP32 filter -- per barycenter p, q = |p'|^2 - 2 v'.p' (three FMAs
//     on coordinates relative to an integer origin), minimised per element -- that
//     proves the winning element whenever the best and second-best elements are more
//     than twice the filter's error bound apart; otherwise (a near tie) the barycenters
//     within the band are re-measured with the reference's FP64 distance in the
//     reference's order.  The result is the reference's element, bit for bit.  The
//     energies use CUDA's acos/log/exp/pow: within a few ULP of the reference's libm,
//     not bit-identical.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr double kPi = 3.14159265358979323846;  // ggLS.h:25
constexpr int kLMax = 256;    // distinct neighbour lists (= elements) per hull
constexpr int kJIds = 8;      // IDs a junction brings itself (a list's IDs other than the grain's)
constexpr unsigned kNoId = 0xFFFFFFFFu;
constexpr int kLHash = 2 * kLMax;  // slots of the distinct-list hash (power of two)
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kIdxMax = 256;       // distinct neighbour IDs the elements of one hull search
constexpr int kIHash = 2 * kIdxMax;
constexpr int kPairMax = 1024;     // (element, searched ID) pairs of one hull
constexpr float kPadQ = 3.0e38f;   // |p|^2 of a padding barycenter: its q is never a minimum
constexpr int kJobMax = 9 * kLMax; // misorientations of one hull's elements (9 per QJ list)

// ---------------------------------------------------------------------------------
// misorientation and boundary properties
// ---------------------------------------------------------------------------------

// LSbox::computeMisorientation (box.cpp:2704-2719) of grain a (this) against b:
// myQuaternion::misorientationCubicQxQ (myQuaternion.cpp:309-367), floored at 1 degree.
__device__ double misorientation(const HullPhysics& ph, uint32_t a, uint32_t b) {
    const double4 s = ph.quat[a], p = ph.quat[b];
    const double m0 = s.x, m1 = -s.y, m2 = -s.z, m3 = -s.w;  // Inverse
    const double a0 = +m0 * p.x - m1 * p.y - m2 * p.z - m3 * p.w;
    const double a1 = +m1 * p.x + m0 * p.y - m3 * p.z + m2 * p.w;
    const double a2 = +m2 * p.x + m3 * p.y + m0 * p.z - m1 * p.w;
    const double a3 = +m3 * p.x - m2 * p.y + m1 * p.z + m0 * p.w;
    const double fac = 1.0 / sqrt(2.0);
    const double r[24] = {(a0 + a1) * fac, (a0 - a1) * fac, (a2 + a3) * fac, (a2 - a3) * fac,
                          (a0 + a2) * fac, (a0 - a2) * fac, (a1 + a3) * fac, (a1 - a3) * fac,
                          (a0 + a3) * fac, (a0 - a3) * fac, (a1 + a2) * fac, (a1 - a2) * fac,
                          (a0 + a1 + a2 + a3) * 0.5, (a0 + a1 - a2 - a3) * 0.5,
                          (a0 - a1 + a2 - a3) * 0.5, (a0 - a1 - a2 + a3) * 0.5,
                          (a0 + a1 + a2 - a3) * 0.5, (a0 + a1 - a2 + a3) * 0.5,
                          (a0 - a1 + a2 + a3) * 0.5, (a0 - a1 - a2 - a3) * 0.5,
                          a0, a1, a2, a3};
    double omega = 0.0;
#pragma unroll
    for (int i = 0; i < 24; i++)
        if (fabs(r[i]) > omega) omega = fabs(r[i]);
    if (omega > 1.0) omega = (double)(int)omega;
    omega = 2 * acos(omega);
    return omega > 1 * kPi / 180.0 ? omega : 1 * kPi / 180.0;
}

// InterfacialElement::computeMobilityMisori / computeReadShockleyEnergy (InterfacialElement.cpp:23-49)
__device__ double mobility_of(const HullPhysics& ph, double misori) {
    if (ph.mobility_model == 0) return 1.0;
    const double mob = 1.0 - (0.99 * exp(-5. * (pow(misori / (15 * kPi / 180), 9.))));
    return mob < 0.1 ? 0.1 : mob;
}
__device__ double energy_of(const HullPhysics& ph, double misori) {
    if (ph.unique_gb == 1) return 1.0;
    const double theta_ref = 15 * kPi / 180;
    if (misori > theta_ref) return 1.0;
    return 1.0 * (misori / theta_ref) * (1.0 - log(misori / theta_ref));
}

// Vector3d (a - b).squaredNorm(): Eigen's unrolled sum c0 + (c1 + c2).  The reference's
// junction test sqrt(d2) < 2 is d2 < 4 exactly: sqrt is correctly rounded and monotone, and
// the largest double below 4, 4 - 2^-51, has its square root below 2 - 2^-53, which rounds
// to 2 - 2^-52.
__device__ __forceinline__ double sqdist(const double* a, const double* b) {
    const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return d0 * d0 + (d1 * d1 + d2 * d2);
}

// ---------------------------------------------------------------------------------
// element construction
// ---------------------------------------------------------------------------------

// A junction being merged: its member lists (keys) chained through next_key.  Its IDs
// are a chain of per-junction segments: its own (at most kJIds, in the CTA's global
// scratch) followed by those of the junctions merged into it, linked through id_next.
// A merge appends the whole chain, duplicates included, as the reference's does.
struct JHead {
    int head, tail;   // member keys
    int own;          // IDs in this junction's own segment
    int nids;         // IDs along the whole chain
    int id_next, id_tail;  // junction whose segment follows (-1: none); last junction of the chain
    int type;         // 3 QJ, 4 HJ
    double pos[3];
};

// One CTA's global scratch: the junction IDs and heads and the (mobility, energy) of
// every misorientation job.  They are used by the junction phase, and keeping them out of
// shared memory lets more grains' warps share an SM.
constexpr size_t kAlignUp(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kJIdBytes = kAlignUp((size_t)kLMax * kJIds * 4);
constexpr size_t kJResBytes = kAlignUp(sizeof(double2) * kJobMax);
constexpr size_t kJHeadBytes = kAlignUp(sizeof(JHead) * kLMax);
constexpr size_t kElemScratch = kJIdBytes + kJResBytes + kJHeadBytes;

struct ElemSmem {
    uint32_t lists[kLMax][8];
    int cnt[kLMax];     // triangles per list
    int off[kLMax];     // first barycenter of the list in the grouped array
    int fill[kLMax];    // barycenters placed so far; then the list's first misorientation job
    int next_key[kLMax];
    double energy[kLMax], mobility[kLMax];
    int qlist[kLMax], hlist[kLMax];
    int lslot[kLHash];  // list hash: index into lists, -1 empty
    int lflat[kLMax];   // first position of each list's barycenters in the flattened FP32 copy
    // neighbour ID -> elements index under construction
    unsigned ikey[kIHash];
    short iden[kIHash];          // dense ID index of the slot
    uint32_t dkey[kIdxMax];
    int dcnt[kIdxMax], dlast[kIdxMax], doff[kIdxMax];
    unsigned short pe[kPairMax]; // (element, dense ID) pairs in search order
    unsigned short pd[kPairMax];
    // in this CTA's global scratch:
    JHead* jh;                   // kLMax working junctions
    uint32_t* jids;              // kLMax x kJIds junction IDs
    double2* jres;               // kJobMax (mobility, energy)
    int nl, nq, nh, nj, ne, nd, np, np_flat;
    double ubox[6];  // box of the grain's barycenters (lo, hi)
    int tnt[32];     // triangles of the 32 records being grouped
    int eseq[kLMax]; // the element sequence: (type << 16) | junction or list
    int next;  // the work item this warp fetched
};

// FNV-1a over the eight IDs of a cube's sorted list
__device__ __forceinline__ unsigned list_hash(const uint32_t (&L)[8]) {
    unsigned h = 2166136261u;
#pragma unroll
    for (int q = 0; q < 8; q++) h = (h ^ L[q]) * 16777619u;
    return h ^ (h >> 15);
}

__device__ __forceinline__ bool same_list(const uint32_t* A, const uint32_t (&L)[8]) {
    bool eq = true;
#pragma unroll
    for (int q = 0; q < 8; q++) eq = eq && A[q] == L[q];
    return eq;
}

// Index of list L among the distinct lists so far, or -1.
__device__ int find_list(const ElemSmem& S, const uint32_t (&L)[8], unsigned h) {
    unsigned s = h & (kLHash - 1);
    for (int probe = 0; probe < kLHash; probe++) {
        const int k = S.lslot[s];
        if (k < 0) return -1;
        if (same_list(S.lists[k], L)) return k;
        s = (s + 1) & (kLHash - 1);
    }
    return -1;
}

__device__ void insert_list(ElemSmem& S, unsigned h, int k, int* err) {
    unsigned s = h & (kLHash - 1);
    for (int probe = 0; probe < kLHash; probe++) {
        if (atomicCAS(&S.lslot[s], -1, k) == -1) return;
        s = (s + 1) & (kLHash - 1);
    }
    atomicOr(err, ERR_HULL);
}

// The mean of n barycenters of the grouped array from b on, summed in order (the
// loads run ahead of the sequential sums).
__device__ __forceinline__ void bary_sum(const double* b, int n, double& p0, double& p1, double& p2) {
    int i = 0;
    for (; i + 8 <= n; i += 8) {  // 24 loads in flight, the sums in order
        double v[24];
#pragma unroll
        for (int u = 0; u < 24; u++) v[u] = b[3 * i + u];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            p0 += v[3 * u];
            p1 += v[3 * u + 1];
            p2 += v[3 * u + 2];
        }
    }
    for (; i < n; i++) {
        p0 += b[3 * i];
        p1 += b[3 * i + 1];
        p2 += b[3 * i + 2];
    }
}

// The junction's position: the mean of its barycenters in member order
// (QuadrupleJunction / HighOrderJunction::computePosition, InterfacialElement.cpp:394-406)
__device__ void junction_position(JHead& J, const ElemSmem& S, const double* eb, int bary_cap, int* err) {
    double p0 = 0, p1 = 0, p2 = 0;
    int n = 0;
    for (int k = J.head; k >= 0; k = S.next_key[k]) {
        if (k >= kLMax || S.off[k] < 0 || S.off[k] + S.cnt[k] > bary_cap) {
            atomicOr(err, ERR_BOUNDS);
            break;
        }
        bary_sum(eb + 3 * (long long)S.off[k], S.cnt[k], p0, p1, p2);
        n += S.cnt[k];
    }
    const double d = (double)n;
    J.pos[0] = p0 / d;
    J.pos[1] = p1 / d;
    J.pos[2] = p2 / d;
}

// Starts junction j's own ID segment (j is its own chain).
__device__ __forceinline__ void start_ids(JHead& J, int j) {
    J.own = J.nids = 0;
    J.id_next = -1;
    J.id_tail = j;
}

__device__ __forceinline__ void push_id(JHead& J, uint32_t* ids, uint32_t id, int* err, int* diag) {
    if (J.own < kJIds) {
        ids[J.own++] = id;
        J.nids++;
    } else {
        atomicOr(err, ERR_HULL);
        atomicOr(diag, HULL_JUNCTION_IDS);
    }
}

// A takes B's member lists and then B's IDs (junction b's chain) after its own.
__device__ __forceinline__ void chain(ElemSmem& S, JHead& A, const JHead& B, int b) {
    S.next_key[A.tail] = B.head;
    A.tail = B.tail;
    S.jh[A.id_tail].id_next = b;
    A.id_tail = B.id_tail;
    A.nids += B.nids;
}

// A float as an int whose signed order is the float's order (and back).
__device__ __forceinline__ int order_key(float f) {
    const int b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float key_float(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

// Warp-wide exclusive scan of v[0, n) in place (n <= kLMax); returns the total.
__device__ int warp_scan_excl(int* v, int n) {
    const int lane = threadIdx.x & 31;
    int run = 0;
    for (int b = 0; b < n; b += 32) {
        const int i = b + lane;
        const int x = i < n ? v[i] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += u;
        }
        if (i < n) v[i] = run + incl - x;
        run += __shfl_sync(kFull, incl, 31);
    }
    __syncwarp();
    return run;
}

__device__ __forceinline__ int id_count(const uint32_t* L) {
    int count = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) count += L[j] == kNoId ? 0 : 1;
    return count;
}

// The neighbours computeGrainBoundaryElements takes from a list of `count` IDs:
// the other ID of a GB list, else the IDs other than g among the first min(count, 4).
__device__ __forceinline__ int list_neighbours(const uint32_t* L, int count, uint32_t g, uint32_t (&nb)[4]) {
    if (count == 2) {
        nb[0] = g != L[0] ? L[0] : L[1];
        return 1;
    }
    const int lim = count < 4 ? count : 4;
    int nn = 0;
    for (int i = 0; i < lim; i++)
        if (g != L[i]) nb[nn++] = L[i];
    return nn;
}

// Misorientation jobs of a list: 1 for a GB (2 IDs), 3 for a TL (3 IDs, one triple
// line), 9 for a QJ list (4 IDs, three triple lines); none otherwise (E = M = 1).
__device__ __forceinline__ int list_jobs(int count) { return count == 2 ? 1 : (count == 3 ? 3 : (count == 4 ? 9 : 0)); }

// The ordered grain pair of job jj of a list: TripleLine(me, n0, n1) computes
// (me, n0), (n0, n1), (me, n1) (InterfacialElement.cpp:119-170); a QJ list's three
// triple lines are (nb0, nb1), (nb1, nb2), (nb0, nb2) (InterfacialElement.cpp:436-456).
__device__ __forceinline__ void job_pair(int count, int jj, uint32_t g, const uint32_t (&nb)[4], uint32_t& x,
                                         uint32_t& y) {
    if (count == 2) {
        x = g;
        y = nb[0];
        return;
    }
    uint32_t u = nb[0], v = nb[1];
    const int tl = jj / 3, r = jj % 3;
    if (tl == 1) { u = nb[1]; v = nb[2]; }
    if (tl == 2) { u = nb[0]; v = nb[2]; }
    if (r == 0) { x = g; y = u; }
    else if (r == 1) { x = u; y = v; }
    else { x = g; y = v; }
}

// TripleLine's energy and mobility (InterfacialElement.cpp:117-160) from its three
// jobs' (mobility, energy).
__device__ __forceinline__ void triple_line_of(const HullPhysics& ph, const double2* r, double& energy,
                                               double& mobility) {
    double avg = 0;
    avg += r[0].x;
    avg += r[1].x;
    avg += r[2].x;
    avg /= 3;
    const double ds = 3 * sqrt(3 * ph.ds * ph.ds);
    mobility = 1. / ((1. / (ds * ph.tl_drag)) + 1. / avg);
    double sigma = r[0].y - r[1].y + r[2].y;
    if (sigma < 0.01) sigma = 0.01;
    if (sigma > 1.0) sigma = 1.0;
    energy = sigma;
}

__global__ void __launch_bounds__(32) elements_kernel(ElementArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ElemSmem& S = *reinterpret_cast<ElemSmem*>(smem_raw);
    const int lane = threadIdx.x;
    if (lane == 0) {  // the bulky, rarely touched arrays live in this CTA's slice of global scratch
        unsigned char* scr = a.scratch + (long long)blockIdx.x * kElemScratch;
        S.jids = reinterpret_cast<uint32_t*>(scr);
        S.jres = reinterpret_cast<double2*>(scr + kJIdBytes);
        S.jh = reinterpret_cast<JHead*>(scr + kJIdBytes + kJResBytes);
    }
    __syncwarp();
    const int n_items = a.item_off[a.G + 1];
    for (;;) {  // grains largest first, fetched on demand
        if (lane == 0) S.next = atomicAdd(a.queue, 1);
        __syncwarp();
        const int t = S.next;
        __syncwarp();
        if (t >= n_items) break;
        const int g = a.order[work_position(a.item_off, a.G, t)];
        if (g < 1 || g > a.G || !a.exists[g]) continue;
        const long long cb = (long long)g * a.cap.cap;
        const int nrec = a.cap.n_rec[g], ntri = a.cap.n_tri[g];
        uint32_t* rec_list = a.cap.rec_list + 8 * cb;
        int* rec_ntri = a.cap.rec_ntri + cb;
        const double* bary = a.cap.bary + 3 * cb;
        const double* tarea = a.cap.tarea + cb;
        double* eb = a.el.ebary + 3 * (long long)g * a.el.bary_cap;
        double* ea = a.el.earea + (long long)g * a.el.bary_cap;
        // 1. distinct lists in first-seen order (MarchingCubesAlgorithm::insertNeighborList,
        //    marchingCubes.cpp:605-618), 32 records at a time: lanes holding the same list
        //    follow the lowest of them, which looks the list up among the earlier ones; new
        //    lists take the next keys in lane order.  The key goes into the record's upper bits.
        for (int q = lane; q < kLHash; q += 32) S.lslot[q] = -1;
        int nl = 0;
        __syncwarp();
        // a record's list (32 bytes, two 16-byte loads) and triangle count; the next chunk's
        // are loaded while this one is deduplicated
        auto load_rec = [&](int r, uint4& l0, uint4& l1, int& nt) {
            if (r < nrec) {
                const uint4* src = reinterpret_cast<const uint4*>(rec_list + 8 * (long long)r);
                l0 = src[0];
                l1 = src[1];
                nt = rec_ntri[r];
            } else {
                l0 = l1 = make_uint4(kNoId, kNoId, kNoId, kNoId);
                nt = 0;
            }
        };
        uint4 n0, n1;
        int n_nt;
        load_rec(lane, n0, n1, n_nt);
        for (int base = 0; base < nrec; base += 32) {
            const int r = base + lane;
            const bool valid = r < nrec;
            const uint32_t mine[8] = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, n1.z, n1.w};
            const int nt_rec = n_nt;
            load_rec(r + 32, n0, n1, n_nt);
            const unsigned h = list_hash(mine);
            const unsigned vmask = __ballot_sync(kFull, valid);
            const unsigned peers = __match_any_sync(kFull, h) & vmask;
            const int leader = valid ? __ffs(peers) - 1 : lane;
            bool same = true;
#pragma unroll
            for (int q = 0; q < 8; q++) same = same && __shfl_sync(kFull, mine[q], leader) == mine[q];
            int found = -1;
            if (__any_sync(kFull, valid && !same)) {
                // two lists of this chunk share a hash: one record at a time
                for (int src = 0; src < 32; src++) {
                    if (!((vmask >> src) & 1)) break;
                    uint32_t L[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) L[q] = __shfl_sync(kFull, mine[q], src);
                    const unsigned hs = __shfl_sync(kFull, h, src);
                    int k = find_list(S, L, hs);
                    if (k < 0) {
                        k = nl < kLMax ? nl : 0;
                        if (nl < kLMax) {
                            if (lane < 8) S.lists[nl][lane] = L[lane];
                            __syncwarp();
                            if (lane == 0) insert_list(S, hs, nl, a.err);
                        } else if (lane == 0) {
                            { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, HULL_LISTS); }
                        }
                        nl++;
                    }
                    if (lane == src) found = k;
                    __syncwarp();
                }
            } else {
                const bool lead = valid && leader == lane;
                if (lead) found = find_list(S, mine, h);
                const bool fresh = lead && found < 0;
                const unsigned fm = __ballot_sync(kFull, fresh);
                if (fresh) {
                    const int k = nl + __popc(fm & ((1u << lane) - 1));
                    if (k < kLMax) {
#pragma unroll
                        for (int q = 0; q < 8; q++) S.lists[k][q] = mine[q];
                        insert_list(S, h, k, a.err);
                        found = k;
                    } else {
                        { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, HULL_LISTS); }
                        found = 0;
                    }
                }
                nl += __popc(fm);
                found = __shfl_sync(kFull, found, leader);
            }
            if (valid) rec_ntri[r] = (nt_rec & 0xFF) | ((found < kLMax && found >= 0 ? found : 0) << 8);
            __syncwarp();
        }
        if (nl > kLMax) nl = kLMax;
        if (lane == 0) S.nl = nl;
        // 2. triangles per list and the grouped offsets
        for (int k = lane; k < nl; k += 32) {
            S.cnt[k] = 0;
            S.fill[k] = 0;
            S.next_key[k] = -1;
            S.lflat[k] = -1;
        }
        __syncwarp();
        for (int r = lane; r < nrec; r += 32) atomicAdd(&S.cnt[rec_ntri[r] >> 8], rec_ntri[r] & 0xFF);
        __syncwarp();
        for (int k = lane; k < nl; k += 32) S.off[k] = S.cnt[k];
        __syncwarp();
        const int nbary = warp_scan_excl(S.off, nl);
        if (nbary > a.el.bary_cap && lane == 0) { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, HULL_TRIANGLES); }
        // 3. barycenters grouped by list, in triangle order (subDivideTrianglesToInterfacialElements):
        //    a record's triangles go after those of the earlier records of its list.  The
        //    warp first places its 32 records, then copies their triangles together,
        //    taking the box of all barycenters on the way (the correction's origin).
        double ulo0 = 1e300, ulo1 = 1e300, ulo2 = 1e300, uhi0 = -1e300, uhi1 = -1e300, uhi2 = -1e300;
        for (int base = 0, tbase = 0; base < nrec; base += 32) {
            const int r = base + lane;
            const bool valid = r < nrec;
            const int v = valid ? rec_ntri[r] : 0;
            const int k = valid ? (v >> 8) : -1;
            const int nt = v & 0xFF;
            int incl = nt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += u;
            }
            const int excl = incl - nt;
            const int total = __shfl_sync(kFull, incl, 31);
            const unsigned peers = __match_any_sync(kFull, k);
            // triangles of the earlier records of this record's list among the 32
            S.tnt[lane] = nt;
            __syncwarp();
            int before = 0;
            for (unsigned m = peers & ((1u << lane) - 1u); m; m &= m - 1) before += S.tnt[__ffs(m) - 1];
            const int dst = valid ? S.off[k] + S.fill[k] + before : 0;
            __syncwarp();
            if (valid && 31 - __clz(peers) == lane) S.fill[k] += before + nt;
            // triangle tbase + q belongs to the last record whose first triangle is <= it
            // (the loop is warp-uniform: every lane takes part in the shuffles)
            for (int q0 = 0; q0 < total; q0 += 32) {
                const int q = q0 + lane;
                int rr = 0;
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int cand = rr + st;
                    const int ex = __shfl_sync(kFull, excl, cand & 31);
                    if (cand < 32 && ex <= q) rr = cand;
                }
                const int pos = __shfl_sync(kFull, dst, rr) + q - __shfl_sync(kFull, excl, rr);
                const int t = tbase + q;
                if (q < total && pos >= 0 && pos < a.el.bary_cap && t < ntri) {
                    const double b0 = bary[3 * (long long)t], b1 = bary[3 * (long long)t + 1],
                                 b2 = bary[3 * (long long)t + 2], ta = tarea[t];
                    eb[3 * (long long)pos] = b0;
                    eb[3 * (long long)pos + 1] = b1;
                    eb[3 * (long long)pos + 2] = b2;
                    ea[pos] = ta;
                    ulo0 = fmin(ulo0, b0); ulo1 = fmin(ulo1, b1); ulo2 = fmin(ulo2, b2);
                    uhi0 = fmax(uhi0, b0); uhi1 = fmax(uhi1, b1); uhi2 = fmax(uhi2, b2);
                }
            }
            tbase += total;
            __syncwarp();
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ulo0 = fmin(ulo0, __shfl_xor_sync(kFull, ulo0, o));
            ulo1 = fmin(ulo1, __shfl_xor_sync(kFull, ulo1, o));
            ulo2 = fmin(ulo2, __shfl_xor_sync(kFull, ulo2, o));
            uhi0 = fmax(uhi0, __shfl_xor_sync(kFull, uhi0, o));
            uhi1 = fmax(uhi1, __shfl_xor_sync(kFull, uhi1, o));
            uhi2 = fmax(uhi2, __shfl_xor_sync(kFull, uhi2, o));
        }
        if (lane == 0) {
            S.ubox[0] = ulo0; S.ubox[1] = ulo1; S.ubox[2] = ulo2;
            S.ubox[3] = uhi0; S.ubox[4] = uhi1; S.ubox[5] = uhi2;
        }
        // 4. one element per list: energy and mobility (computeGrainBoundaryElements).
        //    Every misorientation a list needs is a job; the warp runs the jobs of all
        //    lists side by side, then each list combines its own in the reference's order.
        for (int k = lane; k < nl; k += 32) S.fill[k] = list_jobs(id_count(S.lists[k]));
        __syncwarp();
        int njobs = warp_scan_excl(S.fill, nl);
        if (njobs > kJobMax) {
            if (lane == 0) { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, HULL_JOBS); }
            njobs = kJobMax;
        }
        for (int j = lane; j < njobs; j += 32) {
            int lo = 0, hi = nl - 1;  // the last list whose first job is <= j
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (S.fill[mid] <= j) lo = mid;
                else hi = mid - 1;
            }
            const uint32_t* L = S.lists[lo];
            const int count = id_count(L);
            uint32_t nb[4] = {0, 0, 0, 0};
            list_neighbours(L, count, (uint32_t)g, nb);
            uint32_t x, y;
            job_pair(count, j - S.fill[lo], (uint32_t)g, nb, x, y);
            const double t = misorientation(a.ph, x, y);
            S.jres[j] = make_double2(mobility_of(a.ph, t), energy_of(a.ph, t));
        }
        __syncwarp();
        for (int k = lane; k < nl; k += 32) {
            const int count = id_count(S.lists[k]);
            const int j0 = S.fill[k];
            double E = 1.0, M = 1.0;
            if (j0 + list_jobs(count) <= njobs) {
                const double2* r = S.jres + j0;
                if (count == 2) {
                    M = r[0].x;
                    E = r[0].y;
                } else if (count == 3) {
                    triple_line_of(a.ph, r, E, M);
                } else if (count == 4) {
                    double E1, M1, E2, M2, E3, M3;
                    triple_line_of(a.ph, r, E1, M1);
                    triple_line_of(a.ph, r + 3, E2, M2);
                    triple_line_of(a.ph, r + 6, E3, M3);
                    M = (M1 + M2 + M3) / 3.0;
                    E = (E1 + E2 + E3) / 3.0;
                }
            }
            S.energy[k] = E;
            S.mobility[k] = M;
        }
        __syncwarp();
        // 5. junctions and their merging (computeJunctionPosition + mergeJunction,
        //    grainHull.cpp:267-275, 483-531).  Every list with 4 IDs (QJ) or with 5 or more,
        //    or fewer than 2 (HJ), starts a junction, in list order; the lanes build them
        //    side by side.  The merges are sequential, as the reference's.
        {
            int nj = 0, nq = 0, nh = 0;
            for (int b = 0; b < nl; b += 32) {
                const int k = b + lane;
                const int count = k < nl ? id_count(S.lists[k]) : 2;
                const bool isj = k < nl && !(count < 4 && count > 1);
                const bool isq = isj && count == 4;
                const unsigned bj = __ballot_sync(kFull, isj), bq = __ballot_sync(kFull, isq),
                               bh = __ballot_sync(kFull, isj && !isq);
                const unsigned lt = (1u << lane) - 1;
                if (isj) {
                    const int j = nj + __popc(bj & lt);
                    JHead& J = S.jh[j];
                    J.head = J.tail = k;
                    J.type = isq ? 3 : 4;
                    start_ids(J, j);
                    uint32_t* ids = S.jids + (long long)j * kJIds;
                    for (int i = 0; i < count; i++)
                        if ((uint32_t)g != S.lists[k][i]) push_id(J, ids, S.lists[k][i], a.err, a.cap.diag);
                    junction_position(J, S, eb, a.el.bary_cap, a.err);
                    if (isq) S.qlist[nq + __popc(bq & lt)] = j;
                    else S.hlist[nh + __popc(bh & lt)] = j;
                }
                nj += __popc(bj);
                nq += __popc(bq);
                nh += __popc(bh);
            }
            __syncwarp();
            if (lane == 0) {
                S.nj = nj;
                S.nq = nq;
                S.nh = nh;
            }
            __syncwarp();
        }
        // The merges below are sequential, as the reference's: each scan takes the first
        // pair closer than 2 in the reference's order and restarts from there.  The warp
        // tests 32 candidates of a scan at a time; one lane merges.
        {
            // quadruple points closer than 2: a new high-order junction from the pair
            int i = 0;
            while (i < S.nq) {
                const double* ap = S.jh[S.qlist[i]].pos;
                int found = -1;
                for (int j0 = i + 1; j0 < S.nq && found < 0; j0 += 32) {
                    const int j = j0 + lane;
                    const bool hit = j < S.nq && sqdist(ap, S.jh[S.qlist[j]].pos) < 4.0;
                    const unsigned m = __ballot_sync(kFull, hit);
                    if (m) found = j0 + __ffs(m) - 1;
                }
                if (found < 0) {
                    i++;
                    continue;
                }
                if (S.nj >= kLMax) {
                    if (lane == 0) { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, HULL_JUNCTIONS); }
                    i++;
                    continue;
                }
                if (lane == 0) {
                    const int j = found;
                    JHead& A = S.jh[S.qlist[i]];
                    JHead& B = S.jh[S.qlist[j]];
                    const uint32_t* aid = S.jids + (long long)S.qlist[i] * kJIds;
                    const uint32_t* bid = S.jids + (long long)S.qlist[j] * kJIds;
                    const uint32_t a0 = aid[0], a1 = aid[1], a2 = aid[2], b0 = bid[0], b1 = bid[1], b2 = bid[2];
                    JHead& H = S.jh[S.nj];
                    uint32_t* hid = S.jids + (long long)S.nj * kJIds;
                    H.type = 4;
                    start_ids(H, S.nj);
                    push_id(H, hid, a0, a.err, a.cap.diag);
                    push_id(H, hid, a1, a.err, a.cap.diag);
                    push_id(H, hid, a2, a.err, a.cap.diag);
                    const uint32_t bq[3] = {b0, b1, b2};
                    for (int q = 0; q < 3; q++)  // B's IDs that A already has (sic)
                        if (bq[q] == a0 || bq[q] == a1 || bq[q] == a2) push_id(H, hid, bq[q], a.err, a.cap.diag);
                    H.head = A.head;
                    H.tail = A.tail;
                    S.next_key[H.tail] = B.head;  // the lists of A, then of B; IDs as above
                    H.tail = B.tail;
                    junction_position(H, S, eb, a.el.bary_cap, a.err);
                    // erase i and j (j - 1 after the first erase), then append H
                    for (int u = j; u < S.nq - 1; u++) S.qlist[u] = S.qlist[u + 1];
                    for (int u = i; u < S.nq - 2; u++) S.qlist[u] = S.qlist[u + 1];
                    S.nq -= 2;
                    S.hlist[S.nh++] = S.nj++;
                }
                __syncwarp();  // i again: the next quadruple point moved into it
            }
            // quadruple points closer than 2 to a high-order junction join it (its
            // position moves with every join)
            for (int k = 0; k < S.nh; k++) {
                int i = 0;
                for (;;) {
                    const double* hp = S.jh[S.hlist[k]].pos;
                    int found = -1;
                    for (int i0 = i; i0 < S.nq && found < 0; i0 += 32) {
                        const int ii = i0 + lane;
                        const bool hit = ii < S.nq && sqdist(S.jh[S.qlist[ii]].pos, hp) < 4.0;
                        const unsigned m = __ballot_sync(kFull, hit);
                        if (m) found = i0 + __ffs(m) - 1;
                    }
                    if (found < 0) break;
                    if (lane == 0) {
                        JHead& H = S.jh[S.hlist[k]];
                        chain(S, H, S.jh[S.qlist[found]], S.qlist[found]);
                        junction_position(H, S, eb, a.el.bary_cap, a.err);
                        for (int u = found; u < S.nq - 1; u++) S.qlist[u] = S.qlist[u + 1];
                        S.nq--;
                    }
                    __syncwarp();
                    i = found;
                }
            }
            // high-order junctions closer than 2 merge
            for (int i = 0; i < S.nh; i++) {
                int k = i + 1;
                for (;;) {
                    const double* ap = S.jh[S.hlist[i]].pos;
                    int found = -1;
                    for (int k0 = k; k0 < S.nh && found < 0; k0 += 32) {
                        const int kk = k0 + lane;
                        const bool hit = kk < S.nh && sqdist(ap, S.jh[S.hlist[kk]].pos) < 4.0;
                        const unsigned m = __ballot_sync(kFull, hit);
                        if (m) found = k0 + __ffs(m) - 1;
                    }
                    if (found < 0) break;
                    if (lane == 0) {
                        JHead& A = S.jh[S.hlist[i]];
                        chain(S, A, S.jh[S.hlist[found]], S.hlist[found]);
                        junction_position(A, S, eb, a.el.bary_cap, a.err);
                        for (int u = found; u < S.nh - 1; u++) S.hlist[u] = S.hlist[u + 1];
                        S.nh--;
                    }
                    __syncwarp();
                    k = found;
                }
            }
        }
        __syncwarp();
        // 6. the element table in search order: HJ, QJ, TL, GB, with its barycenter
        //    segments, and the (element, searched ID) pairs.  The sequence is listed first;
        //    then 32 elements at a time each lane sizes one (IDs, segments, barycenters),
        //    warp scans place them and each lane writes its own.  An element that does not
        //    fit a capacity ends the table (the step then reports the overflow).  The ID
        //    index (dense IDs in first-seen order) is built by one lane.
        for (int q = lane; q < kIHash; q += 32) S.ikey[q] = kNoId;
        int* eidoff = S.qlist;  // per element: its first ID; the lists are copied into eseq
        int* enid = S.hlist;    // per element: its IDs
        int* esid = S.lslot;    // per TL / GB element e: its searched IDs at 2 e, 2 e + 1
        {
            const int nh = S.nh, nq = S.nq;
            for (int i = lane; i < nh; i += 32) S.eseq[i] = (4 << 16) | S.hlist[i];
            for (int i = lane; i < nq; i += 32) S.eseq[nh + i] = (3 << 16) | S.qlist[i];
            int nseq = nh + nq;
            for (int pass = 2; pass >= 1; pass--)  // TL, then GB, each in key order
                for (int k0 = 0; k0 < nl; k0 += 32) {
                    const int k = k0 + lane;
                    const bool take = k < nl && id_count(S.lists[k]) == pass + 1;
                    const unsigned m = __ballot_sync(kFull, take);
                    const int at = nseq + __popc(m & ((1u << lane) - 1u));
                    if (take && at < kLMax) S.eseq[at] = (pass << 16) | k;
                    nseq += __popc(m);
                }
            if (nseq > kLMax) {  // each element holds a distinct list: cannot happen
                if (lane == 0) atomicOr(a.err, ERR_BOUNDS);
                nseq = kLMax;
            }
            __syncwarp();
            HullElem* E = a.el.elem + (long long)g * a.el.elem_cap;
            uint32_t* ids = a.el.ids + (long long)g * a.el.id_cap;
            int2* segs = a.el.segs + (long long)g * a.el.seg_cap;
            int ne = 0, ni = 0, ns = 0, pb = 0;
            bool over = false;
            for (int c0 = 0; c0 < nseq; c0 += 32) {
                const int e = c0 + lane;
                const bool have = e < nseq;
                int type = 0, src = 0, nid = 0, nseg = 0, pcnt = 0, head = -1;
                uint32_t nb[3] = {0u, 0u, 0u};
                if (have) {
                    const int v = S.eseq[e];
                    type = v >> 16;
                    src = v & 0xFFFF;
                    if (type >= 3) {
                        // the junction's IDs: its segment chain, up to J.nids of them
                        const JHead& J = S.jh[src];
                        head = J.head;
                        int n = 0;
                        for (int j = src, walk = 0; j >= 0 && walk < kLMax && n < J.nids; walk++, j = S.jh[j].id_next)
                            n += min(S.jh[j].own, J.nids - n);
                        if (n != J.nids) atomicOr(a.err, ERR_BOUNDS);
                        nid = n;
                    } else {
                        head = src;
                        const uint32_t* L = S.lists[src];
                        if (type == 1) {
                            nb[nid++] = (uint32_t)g != L[0] ? L[0] : L[1];
                        } else {
#pragma unroll
                            for (int q = 0; q < 3; q++)
                                if ((uint32_t)g != L[q]) {
#pragma unroll
                                    for (int r = 0; r < 3; r++)
                                        if (r == nid) nb[r] = L[q];
                                    nid++;
                                }
                        }
                    }
                    for (int k = head, walk = 0; k >= 0 && walk < kLMax; walk++, k = type >= 3 ? S.next_key[k] : -1) {
                        if (k >= kLMax || S.off[k] < 0 || S.off[k] + S.cnt[k] > a.el.bary_cap) {
                            atomicOr(a.err, ERR_BOUNDS);
                            break;
                        }
                        nseg++;
                        pcnt += S.cnt[k];
                    }
                }
                // every element's run starts on a pair boundary; an odd run gets a padding entry
                const int padded = pcnt + (pcnt & 1);
                int xi = nid, xs = nseg, xp = padded;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int ui = __shfl_up_sync(kFull, xi, o), us = __shfl_up_sync(kFull, xs, o),
                              up = __shfl_up_sync(kFull, xp, o);
                    if (lane >= o) { xi += ui; xs += us; xp += up; }
                }
                const int id_off = ni + xi - nid, seg_off = ns + xs - nseg, pbase = pb + xp - padded;
                const bool fits = ne + lane < a.el.elem_cap && id_off + nid <= a.el.id_cap &&
                                  seg_off + nseg <= a.el.seg_cap && pbase + padded <= a.el.flat_cap;
                const unsigned bad = __ballot_sync(kFull, have && !fits);
                const int cnt = bad ? __ffs(bad) - 1 : min(32, nseq - c0);  // elements placed
                if (lane < cnt) {
                    const int ei = ne + lane;
                    if (type >= 3) {
                        int w = id_off;
                        for (int j = src, walk = 0; j >= 0 && walk < kLMax && w < id_off + nid; walk++, j = S.jh[j].id_next) {
                            const uint32_t* seg = S.jids + (long long)j * kJIds;
                            for (int q = 0; q < S.jh[j].own && w < id_off + nid; q++) ids[w++] = seg[q];
                        }
                    } else {
                        for (int q = 0; q < nid; q++) ids[id_off + q] = nb[q];
                        esid[2 * ei] = (int)nb[0];
                        esid[2 * ei + 1] = (int)nb[1];
                    }
                    int sg = seg_off, pc = 0;
                    for (int k = head, walk = 0; k >= 0 && walk < nseg; walk++, k = type >= 3 ? S.next_key[k] : -1) {
                        const int off = S.off[k], c = S.cnt[k];
                        segs[sg++] = make_int2(off, c);
                        S.lflat[k] = pbase + pc;
                        S.fill[k] = ei;  // fill is free after the jobs: the list's element
                        pc += c;
                    }
                    HullElem& el = E[ei];
                    el.type = type;
                    el.id_off = id_off;
                    el.nids = nid;
                    el.seg_off = seg_off;
                    el.nseg = nseg;
                    // a junction made from one list keeps that list's energy (1 for HJ)
                    el.energy = type == 4 ? 1.0 : S.energy[head];
                    el.mobility = type == 4 ? 1.0 : S.mobility[head];
                    el.area = 0.0;
                    el.pbase = pbase;
                    el.pcount = pcnt;
                    eidoff[ei] = id_off;
                    enid[ei] = nid;
                }
                if (cnt > 0) {
                    ni += __shfl_sync(kFull, xi, cnt - 1);
                    ns += __shfl_sync(kFull, xs, cnt - 1);
                    pb += __shfl_sync(kFull, xp, cnt - 1);
                }
                ne += cnt;
                if (bad) {
                    over = true;
                    break;
                }
            }
            __syncwarp();
            if (lane == 0) {
                // the index: each element's searched IDs -- all for a high-order junction,
                // else the first 3 (QJ), 2 (TL), 1 (GB) -- in element order, each element once
                // per ID; IDs numbered by first appearance
                int nd = 0, np = 0;
                bool over_index = false;
                for (int e = 0; e < ne; e++) {
                    const int type = S.eseq[e] >> 16, nid = enid[e];
                    const int nc = type == 4 ? nid : min(nid, type);
                    for (int q = 0; q < nc; q++) {
                        const uint32_t id = type <= 2 ? (uint32_t)esid[2 * e + q] : ids[eidoff[e] + q];
                        unsigned hs = (id * 2654435761u) & (kIHash - 1);
                        int d = -1;
                        for (int probe = 0; probe < kIHash; probe++) {
                            if (S.ikey[hs] == id) { d = S.iden[hs]; break; }
                            if (S.ikey[hs] == kNoId) {
                                if (nd >= kIdxMax) break;
                                S.ikey[hs] = id;
                                S.iden[hs] = (short)nd;
                                S.dkey[nd] = id;
                                S.dcnt[nd] = 0;
                                S.dlast[nd] = -1;
                                d = nd++;
                                break;
                            }
                            hs = (hs + 1) & (kIHash - 1);
                        }
                        if (d < 0 || np >= kPairMax) { over = over_index = true; break; }
                        if (S.dlast[d] == e) continue;
                        S.dlast[d] = e;
                        S.dcnt[d]++;
                        S.pe[np] = (unsigned short)e;
                        S.pd[np] = (unsigned short)d;
                        np++;
                    }
                }
                // IDs with their element ranges, elements in search order
                int run = 0;
                for (int d = 0; d < nd; d++) {
                    S.doff[d] = run;
                    run += S.dcnt[d];
                    S.dcnt[d] = 0;
                }
                if (run > a.el.pair_cap) over = over_index = true;
                unsigned short* pairs = a.el.idx_elem + (long long)g * a.el.pair_cap;
                for (int q = 0; q < np; q++) {
                    const int d = S.pd[q];
                    const int at = S.doff[d] + S.dcnt[d]++;
                    if (at < a.el.pair_cap) pairs[at] = S.pe[q];
                }
                if (over) { atomicOr(a.err, ERR_HULL); atomicOr(a.cap.diag, over_index ? HULL_INDEX : HULL_TABLE); }
                a.el.n_elem[g] = ne;
                a.el.n_idx[g] = nd;
                a.el.n_flat[g] = pb;
                S.np_flat = pb;
                S.ne = ne;
                S.nd = nd;
            }
        }
        __syncwarp();
        {
            const int ne = S.ne, nd = S.nd;
            HullElem* E = a.el.elem + (long long)g * a.el.elem_cap;
            uint32_t* ikey = a.el.idx_key + (long long)g * a.el.idx_cap;
            int2* irng = a.el.idx_rng + (long long)g * a.el.idx_cap;
            for (int d = lane; d < nd && d < a.el.idx_cap; d += 32) {
                ikey[d] = S.dkey[d];
                irng[d] = make_int2(S.doff[d], S.dcnt[d]);
            }
            // GrainBoundary::computeArea (InterfacialElement.cpp:81-91): its triangles'
            // terms summed in triangle order, times h^2
            for (int e = lane; e < ne; e += 32) {
                HullElem& el = E[e];
                if (el.type != 1 || el.nseg != 1) continue;
                const int2 sg = a.el.segs[(long long)g * a.el.seg_cap + el.seg_off];
                if (sg.x < 0 || sg.y < 0 || sg.x + sg.y > a.el.bary_cap) continue;
                double surface = 0;
                int i = 0;
                for (; i + 4 <= sg.y; i += 4) {  // the loads run ahead of the sums, which stay in order
                    const double t0 = ea[sg.x + i], t1 = ea[sg.x + i + 1], t2 = ea[sg.x + i + 2], t3 = ea[sg.x + i + 3];
                    surface += t0;
                    surface += t1;
                    surface += t2;
                    surface += t3;
                }
                for (; i < sg.y; i++) surface += ea[sg.x + i];
                el.area = surface * a.ph.ds * a.ph.ds;  // ds = h = 1 / realDomainSize
            }
            // the correction's FP32 barycenters, relative to the integer centre of the box
            // of the grain's barycenters (taken while they were grouped)
            const int nl = S.nl, total = min(nbary, a.el.bary_cap), nflat = min(S.np_flat, a.el.flat_cap);
            double org[3] = {0, 0, 0};
            if (ne > 0 && S.ubox[3] >= S.ubox[0])
#pragma unroll
                for (int q = 0; q < 3; q++) org[q] = floor(0.5 * (S.ubox[q] + S.ubox[q + 3]));
            // element boxes relative to the origin, rounded outward to FP32, as orderable
            // integer keys in the index arrays' shared memory (dead by now): 6 per element
            int* bkey = reinterpret_cast<int*>(S.ikey);
            static_assert(sizeof(unsigned) * kIHash + sizeof(short) * kIHash + sizeof(uint32_t) * kIdxMax +
                                  3 * sizeof(int) * kIdxMax + 2 * sizeof(unsigned short) * kPairMax >=
                              6 * sizeof(int) * kLMax,
                          "the index arrays hold the element-box keys");
            for (int q = lane; q < 6 * min(ne, kLMax); q += 32) bkey[q] = (q % 6) < 3 ? INT_MAX : INT_MIN;
            __syncwarp();
            // every barycenter to its element's run: lane-parallel over the grouped array,
            // barycenter i of list k (the last list whose first barycenter is <= i) going to
            // lflat[k] + (i - off[k])
            float* pf = reinterpret_cast<float*>(a.el.ebf + (long long)g * a.el.flat_cap);
            int* pidx = a.el.eidx + (long long)g * a.el.flat_cap;
            float r2 = 0.f;
            // the barycenter of the lane's next index is loaded while this one is placed
            double p0 = 0, p1 = 0, p2 = 0;
            if (lane < total) { p0 = eb[3 * (long long)lane]; p1 = eb[3 * (long long)lane + 1]; p2 = eb[3 * (long long)lane + 2]; }
            for (int i = lane; i < total; i += 32) {
                const double b0 = p0, b1 = p1, b2 = p2;
                if (i + 32 < total) {
                    p0 = eb[3 * (long long)(i + 32)];
                    p1 = eb[3 * (long long)(i + 32) + 1];
                    p2 = eb[3 * (long long)(i + 32) + 2];
                }
                int lo = 0, hi = nl - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.off[mid] <= i) lo = mid;
                    else hi = mid - 1;
                }
                const int base = nl > 0 ? S.lflat[lo] : -1;
                const int dst = base < 0 ? -1 : base + (i - S.off[lo]);
                if (dst < 0 || dst >= nflat) continue;  // a list no element holds
                const double dx = b0 - org[0], dy = b1 - org[1], dz = b2 - org[2];
                const double w = dx * dx + dy * dy + dz * dz;
                float* pp = pf + 8 * (dst >> 1) + (dst & 1);  // pair layout: x0 x1 y0 y1 z0 z1 w0 w1
                pp[0] = (float)dx;
                pp[2] = (float)dy;
                pp[4] = (float)dz;
                pp[6] = (float)w;
                pidx[dst] = i;
                r2 = fmaxf(r2, (float)w);
                const int e = S.fill[lo];  // the element list lo went to (emit)
                if (e >= 0 && e < ne && e < kLMax) {
                    int* bk = bkey + 6 * e;
                    atomicMin(bk + 0, order_key(__double2float_rd(dx)));
                    atomicMin(bk + 1, order_key(__double2float_rd(dy)));
                    atomicMin(bk + 2, order_key(__double2float_rd(dz)));
                    atomicMax(bk + 3, order_key(__double2float_ru(dx)));
                    atomicMax(bk + 4, order_key(__double2float_ru(dy)));
                    atomicMax(bk + 5, order_key(__double2float_ru(dz)));
                }
            }
            __syncwarp();
            // the element boxes, stored as origin + the FP32 bound (exact in FP64), so that
            // the correction's outward rounding of (box - origin) gives the bound back
            for (int e = lane; e < min(ne, kLMax); e += 32) {
                HullElem& el = E[e];
                const int* bk = bkey + 6 * e;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    el.lo[q] = bk[q] == INT_MAX ? 1e300 : org[q] + (double)key_float(bk[q]);
                    el.hi[q] = bk[q + 3] == INT_MIN ? -1e300 : org[q] + (double)key_float(bk[q + 3]);
                }
            }
            // the padding entry of every odd run: at the origin with q = kInf, never a minimum
            {
                for (int e = lane; e < S.ne; e += 32) {
                    const int n = E[e].pcount, dst = E[e].pbase + n;
                    if ((n & 1) && dst >= 0 && dst < nflat) {
                        float* pp = pf + 8 * (dst >> 1) + (dst & 1);
                        pp[0] = 0.f;
                        pp[2] = 0.f;
                        pp[4] = 0.f;
                        pp[6] = kPadQ;
                        pidx[dst] = -1;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r2 = fmaxf(r2, __shfl_xor_sync(kFull, r2, o));
            if (lane == 0) a.el.eorg[g] = make_float4((float)org[0], (float)org[1], (float)org[2], r2);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------
// the correction
// ---------------------------------------------------------------------------------

constexpr int kCHash = 512;  // slots of a CTA's ID -> elements hash (>= 2 kIdxMax)

// Squared distance of (x, y, z) to b, summed as Vector3d::squaredNorm (c0 + (c1 + c2)).
__device__ __forceinline__ double sqdist3(double x, double y, double z, const double* b) {
    const double d0 = x - b[0], d1 = y - b[1], d2 = z - b[2];
    return d0 * d0 + (d1 * d1 + d2 * d2);
}

constexpr int kCThreads = 256;
constexpr int kCVox = 4096;           // voxels of one pass: a run of the box in [z][y][x] order
constexpr int kCItem = 4 * kCVox;     // voxels of one work item: a grain's box is cut into runs of these
constexpr int kLV = 2;                // voxels per lane: a packet is 32 kLV voxels of one neighbour
constexpr int kPacket = 32 * kLV;
constexpr int kWarpTies = 8;          // near ties a packet settles voxel by voxel with the whole warp
constexpr unsigned short kNoD = 0xFFFF;
constexpr float kInf = 3.0e38f;
constexpr int kSPts = 2304;           // barycenters staged in shared memory (more: read from HBM)
constexpr int kSElem = kLMax;         // elements per grain: one per distinct list at most
constexpr int kSPairs = kPairMax;     // the index's (element, ID) pairs per grain
static_assert(kSElem <= 0xFFFF && kSPairs <= 0xFFFF, "16-bit element and pair indices");
static_assert(kSPairs % 8 == 0, "pair lists are copied 16 bytes at a time");

// One grain's search data, staged once per grain, and the slice pass's voxel groups.
struct CorrSmem {
    float4 pts[kSPts];            // FP32 barycenters, element by element, in pairs (ebf)
    float box[kSElem][6];         // element boxes relative to the origin, rounded outward
    int2 erun[kSElem];            // element e's run in ebf: (first, count), both even
    alignas(16) unsigned short pairs[kSPairs];  // the index's element lists (search order per ID)
    uint32_t hkey[kCHash];        // neighbour ID -> dense index d
    unsigned short hden[kCHash];
    int2 drng[kIdxMax];           // dense index d -> its elements in pairs
    int dcnt[kIdxMax], doff[kIdxMax], dcur[kIdxMax], dpk[kIdxMax + 1];
    unsigned short vd[kCVox];     // dense neighbour index of the pass's voxels, kNoD: no search
    unsigned short vlist[kCVox];  // pass voxels grouped by neighbour
    int next;                     // the work item this CTA fetched
    int pk_next;                  // the pass's next unclaimed packet
};

// q of barycenter p for the voxel whose relative coordinates give (ax, ay, az) = -2 v':
// |p'|^2 - 2 v'.p' = |v' - p'|^2 - |v'|^2.
__device__ __forceinline__ float qval(const float4 p, float ax, float ay, float az) {
    return fmaf(az, p.z, fmaf(ay, p.y, fmaf(ax, p.x, p.w)));
}

// Barycenter i of the pair layout (x0 x1 y0 y1 | z0 z1 w0 w1 per pair) as (x, y, z, w).
__device__ __forceinline__ float4 pt_at(const float4* pts, int i) {
    const float* f = reinterpret_cast<const float*>(pts + 2 * (i >> 1)) + (i & 1);
    return make_float4(f[0], f[2], f[4], f[6]);
}

// Two FP32 lanes packed in 64 bits: the operands of the packed FMA.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

// fma.rn per lane: each half rounds exactly as fmaf does.
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// min(m, both halves of r).
__device__ __forceinline__ float min_of(float m, unsigned long long r) {
    float lo, hi, d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(m), "f"(lo), "f"(hi));
    return d;
}

// The least q, for each of a lane's V voxels, over the n (even) barycenters of a run
// starting at pair boundary `first`: two barycenters per packed FMA chain, the same
// three roundings per barycenter as qval.  Each loaded pair serves all V voxels.
template <int V>
__device__ __forceinline__ void run_min(const float4* pts, int first, int n, const unsigned long long (&A2)[V],
                                        const unsigned long long (&B2)[V], const unsigned long long (&C2)[V],
                                        float (&m)[V]) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(pts + first);  // 2 per pair
    const int np = n >> 1;
#pragma unroll
    for (int u = 0; u < V; u++) m[u] = kInf;
#pragma unroll 2
    for (int i = 0; i < np; i++) {
        const ulonglong2 xy = p[2 * i], zw = p[2 * i + 1];
#pragma unroll
        for (int u = 0; u < V; u++) m[u] = min_of(m[u], fma2(C2[u], zw.x, fma2(B2[u], xy.y, fma2(A2[u], xy.x, zw.y))));
    }
}

// The near-tie case: the barycenters whose q is within the band, measured with the
// reference's FP64 distance (Vector3d::squaredNorm, c0 + (c1 + c2)) and kept only when
// strictly nearer, visiting elements in search order and each element's barycenters in
// order, as projectPointToGrainBoundary does (grainHull.cpp:570-660).  Every barycenter
// that can be the reference's winner has q <= best + eps2, so the subset has the same
// winner.
// `band` marks (bit c, when count <= 32) the candidates whose least q came within the band
// of the best so far when they were scanned: a superset of those within the final band,
// the only ones that can hold such a barycenter; the rest are not visited.
__device__ int exact_winner(const CorrSmem& S, const float4* pts, int first, int count, int ne,
                            const int* __restrict__ eidx, const double* __restrict__ eb, double x, double y, double z,
                            float ax, float ay, float az, float limit, unsigned band) {
    double bd = 10000000.0;
    int bw = -1;
    for (int c = 0; c < count; c++) {
        if (count <= 32 && !((band >> c) & 1u)) continue;
        const int e = S.pairs[first + c];
        if (e >= ne) continue;
        const int2 r = S.erun[e];  // the element's barycenters in order (a padding entry: q = kInf)
        for (int i = r.x; i < r.x + r.y; i++) {
            if (qval(pt_at(pts, i), ax, ay, az) > limit) continue;
            const int src = eidx[i];
            if (src < 0) continue;
            const double d = sqdist3(x, y, z, eb + 3 * (long long)src);
            if (d < bd) {
                bd = d;
                bw = e;
            }
        }
    }
    return bw;
}

// exact_winner for one voxel with the whole warp: lane l takes barycenters l, l + 32, ...
// of each element the band holds, keeping the least FP64 distance and, among equal
// ones, the first in its own order; the warp then reduces on (distance, element position
// c, barycenter) -- the first in search order among the least, as the sequential walk.
__device__ int exact_winner_warp(const CorrSmem& S, const float4* pts, int first, int count, int ne,
                                 const int* __restrict__ eidx, const double* __restrict__ eb, int i, int j, int k,
                                 float4 org, float limit, unsigned band) {
    const int lane = threadIdx.x & 31;
    const float ax = -2.f * ((float)i - org.x), ay = -2.f * ((float)j - org.y), az = -2.f * ((float)k - org.z);
    const double x = (double)i, y = (double)j, z = (double)k;
    double bd = 10000000.0;
    int bkey = 0x7FFFFFFF;  // (c << 20) | barycenter position in the element's run
    for (int c = 0; c < count; c++) {
        if (count <= 32 && !((band >> c) & 1u)) continue;
        const int e = S.pairs[first + c];
        if (e >= ne) continue;
        const int2 r = S.erun[e];
        for (int t = lane; t < r.y; t += 32) {
            if (qval(pt_at(pts, r.x + t), ax, ay, az) > limit) continue;
            const int src = eidx[r.x + t];
            if (src < 0) continue;
            const double d = sqdist3(x, y, z, eb + 3 * (long long)src);
            if (d < bd) {
                bd = d;
                bkey = (c << 20) | t;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double od = __shfl_xor_sync(kFull, bd, o);
        const int ok = __shfl_xor_sync(kFull, bkey, o);
        if (od < bd || (od == bd && ok < bkey)) {
            bd = od;
            bkey = ok;
        }
    }
    return bkey == 0x7FFFFFFF ? -1 : S.pairs[first + (bkey >> 20)];
}

// Lower bound of q over a box [lo, hi] (relative, rounded outward) for the voxel v':
// |v' - box|^2 in FP32, scaled down past its rounding, - |v'|^2 - eps.
__device__ __forceinline__ float box_bound(float vx, float vy, float vz, float vv, float lx, float ly, float lz,
                                           float hx, float hy, float hz, float eps) {
    const float dx = vx < lx ? lx - vx : (vx > hx ? vx - hx : 0.f);
    const float dy = vy < ly ? ly - vy : (vy > hy ? vy - hy : 0.f);
    const float dz = vz < lz ? lz - vz : (vz > hz ? vz - hz : 0.f);
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    return d2 * (1.f - 1.0f / 1048576.f) - vv - eps;
}

// The elements whose (energy, mobility) a lane's V voxels (i, j, k) take: the
// reference's winner among the elements S.pairs[first, first + count) (-1: none,
// weight (1, 1)).  All lanes of the warp call it with the same elements (a packet of one
// neighbour).  Per voxel, each element's least q is compared with the best and
// second-best so far; when the best element beats every other by more than eps2 (twice
// the filter's error bound) it is the reference's winner, else the near tie is settled
// in FP64 (exact_winner).  Elements are taken in reverse search order, so the grain
// boundary (last in search order, and the usual winner) sets a tight best first, and an
// element is skipped when no voxel of the warp can come within the band of its best
// through the element's box.
template <int V>
__device__ __forceinline__ void search_packet(const CorrSmem& S, const float4* pts, int first, int count,
                                              const bool (&active)[V], const int (&ii)[V], const int (&jj)[V],
                                              const int (&kk)[V], float4 org, float eps2, int ne,
                                              const int* __restrict__ eidx, const double* __restrict__ eb, int* err,
                                              int (&win)[V]) {
    float vx[V], vy[V], vz[V], vv[V], best[V], second[V];
    unsigned long long A2[V], B2[V], C2[V];
    int beste[V];
    unsigned band[V];  // candidates within the band of the best when scanned (count <= 32)
#pragma unroll
    for (int u = 0; u < V; u++) {
        vx[u] = (float)ii[u] - org.x;  // exact
        vy[u] = (float)jj[u] - org.y;
        vz[u] = (float)kk[u] - org.z;
        vv[u] = vx[u] * vx[u] + vy[u] * vy[u] + vz[u] * vz[u];  // exact (integers below 2^24)
        A2[u] = pack2(-2.f * vx[u], -2.f * vx[u]);
        B2[u] = pack2(-2.f * vy[u], -2.f * vy[u]);
        C2[u] = pack2(-2.f * vz[u], -2.f * vz[u]);
        best[u] = second[u] = kInf;
        beste[u] = -1;
        band[u] = 0u;
    }
    const float eps = 0.5f * eps2;
    for (int c = count - 1; c >= 0; c--) {
        const int e = S.pairs[first + c];
        if (e >= ne) {
            if ((threadIdx.x & 31) == 0) atomicOr(err, ERR_BOUNDS);
            continue;
        }
        // skipped when no voxel can come within the band of its best through the
        // element's box (best = kInf: never skipped)
        const float* bx = S.box[e];
        const float lx = bx[0], ly = bx[1], lz = bx[2], hx = bx[3], hy = bx[4], hz = bx[5];
        bool need = false;
#pragma unroll
        for (int u = 0; u < V; u++)
            need = need || (active[u] && box_bound(vx[u], vy[u], vz[u], vv[u], lx, ly, lz, hx, hy, hz, eps) <=
                                             best[u] + eps2);
        if (!__any_sync(kFull, need)) continue;
        const int2 r = S.erun[e];
        float m[V];
        run_min<V>(pts, r.x, r.y, A2, B2, C2, m);
#pragma unroll
        for (int u = 0; u < V; u++) {
            if (m[u] < best[u]) {
                second[u] = best[u];
                best[u] = m[u];
                beste[u] = e;
            } else {
                second[u] = fminf(second[u], m[u]);
            }
            if (m[u] <= best[u] + eps2) band[u] |= 1u << (c & 31);
        }
    }
    // proven when every other element is farther by more than the band; a few near ties
    // are settled one voxel at a time by the whole warp, many by each lane for its own
    unsigned tie[V];
    int nties = 0;
#pragma unroll
    for (int u = 0; u < V; u++) {
        win[u] = beste[u];
        tie[u] = __ballot_sync(kFull, active[u] && beste[u] >= 0 && !(second[u] - best[u] > eps2));
        nties += __popc(tie[u]);
    }
    if (nties == 0) return;
    const int lane = threadIdx.x & 31;
    if (nties <= kWarpTies) {
#pragma unroll
        for (int u = 0; u < V; u++)
            for (unsigned m = tie[u]; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                const int si = __shfl_sync(kFull, ii[u], src), sj = __shfl_sync(kFull, jj[u], src),
                          sk = __shfl_sync(kFull, kk[u], src);
                const float lim = __shfl_sync(kFull, best[u] + eps2, src);
                const unsigned bnd = __shfl_sync(kFull, band[u], src);
                const int w = exact_winner_warp(S, pts, first, count, ne, eidx, eb, si, sj, sk, org, lim, bnd);
                if (lane == src) win[u] = w;
            }
    } else {
#pragma unroll
        for (int u = 0; u < V; u++)
            if ((tie[u] >> lane) & 1u)
                win[u] = exact_winner(S, pts, first, count, ne, eidx, eb, (double)ii[u], (double)jj[u],
                                      (double)kk[u], -2.f * vx[u], -2.f * vy[u], -2.f * vz[u], best[u] + eps2,
                                      band[u]);
    }
}

// q = n / d and r = n % d for 0 <= n < 2^24 and d >= 1, from rcp = RN(1 / d): the float
// quotient is within 2 of n / d (two roundings of relative size 2^-24 on a value below
// 2^24), and two correction steps each way make it exact.
__device__ __forceinline__ void divmod24(int n, int d, float rcp, int& q, int& r) {
    q = __float2int_rz((float)n * rcp);
    r = n - q * d;
    if (r < 0) { q--; r += d; }
    if (r < 0) { q--; r += d; }
    if (r >= d) { q++; r -= d; }
    if (r >= d) { q++; r -= d; }
}

// The update of one band voxel, box.cpp:476-533, given the element that won (-1: none).
template <typename T>
__device__ __forceinline__ void correct_voxel(const CorrectionArgs<T>& a, const HullElem* elem, int g, int win,
                                              uint32_t id, double val, double conv, T* outp) {
    const double ts = 1 / 1.21;  // TimeSlope, grainhdl.cpp:1432
    const double E = win >= 0 ? elem[win].energy : 1.0, M = win >= 0 ? elem[win].mobility : 1.0;
    // GBInfo(m_energy, m_mobility) fills (mobility, energy): field energy = M, field mobility = E
    const double fe = M, fm = E;
    double o = val + (conv - val) * fe * fm * 1.0;
    if (a.ph.use_see) {
        const bool alive = id == 0 || (id <= (uint32_t)a.G && a.present[id]);
        const double fs = alive ? (a.ph.see[g] - a.ph.see[id]) * fm * a.ph.dt / (ts * ts) : 0.0;
        o = o - fs;
    }
    *outp = (T)o;
}

// A CTA per grain: the grain's element index, element boxes and FP32 barycenters are
// staged in shared memory once; then, pass by pass over runs of kCVox consecutive voxels
// of the box, the band voxels are grouped by IDLocal neighbour (counting sort in shared
// memory) and the warps take packets of 32 voxels of one neighbour.
template <typename T>
__global__ void __launch_bounds__(kCThreads, 3) correction_kernel(CorrectionArgs<T> a) {
    extern __shared__ __align__(16) unsigned char corr_smem[];
    CorrSmem& S = *reinterpret_cast<CorrSmem*>(corr_smem);
    const double delta = a.geo.delta;
    const HullElements& el = a.el;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int n_items = a.item_off[a.G + 1];
    for (;;) {
        __syncthreads();  // the previous item's packets are done with the shared arrays
        if (threadIdx.x == 0) S.next = atomicAdd(a.queue, 1);
        __syncthreads();
        const int t = S.next;
        if (t >= n_items) break;
        const int pos = work_position(a.item_off, a.G, t);
        const int g = a.order[pos];
        const long long item = t - a.item_off[pos];  // the run of box voxels this CTA takes
        if (g < 1 || g > a.G) {
            if (threadIdx.x == 0) atomicOr(a.err, ERR_BOUNDS);
            continue;
        }
        const int ne = min(max(el.n_elem[g], 0), min(el.elem_cap, kSElem));
        int nd = el.n_idx[g];
        if (nd < 0 || nd > el.idx_cap || nd > kIdxMax) {
            if (threadIdx.x == 0) atomicOr(a.err, ERR_BOUNDS);
            nd = 0;
        }
        const int nflat = min(max(el.n_flat[g], 0), el.flat_cap) & ~1;
        const int npairs = min(el.pair_cap, kSPairs);
        const float4 org = el.eorg[g];
        const float4* gpts = el.ebf + (long long)g * el.flat_cap;
        for (int q = threadIdx.x; q < kCHash; q += blockDim.x) S.hkey[q] = kNoId;
        {  // the pair lists and the barycenters, copied asynchronously (waited for below)
            const uint4* src = reinterpret_cast<const uint4*>(el.idx_elem + (long long)g * el.pair_cap);
            uint4* dst = reinterpret_cast<uint4*>(S.pairs);
            for (int q = threadIdx.x; q < npairs / 8; q += blockDim.x) cp_async16(dst + q, src + q);
            if (nflat <= kSPts)
                for (int q = threadIdx.x; q < nflat; q += blockDim.x) cp_async16(S.pts + q, gpts + q);
        }
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            const HullElem& E = el.elem[(long long)g * el.elem_cap + e];
            int2 run = make_int2(E.pbase, E.pcount + (E.pcount & 1));  // with its padding entry
            if (run.x < 0 || (run.x & 1) || run.y < 0 || run.x + run.y > nflat) {
                atomicOr(a.err, ERR_BOUNDS);
                run = make_int2(0, 0);
            }
            S.erun[e] = run;
            const float o[3] = {org.x, org.y, org.z};
#pragma unroll
            for (int q = 0; q < 3; q++) {
                S.box[e][q] = __double2float_rd(E.lo[q] - (double)o[q]);
                S.box[e][q + 3] = __double2float_ru(E.hi[q] - (double)o[q]);
            }
        }
        cp_async_wait_all();
        __syncthreads();  // the hash is cleared, the copies have landed
        for (int d = threadIdx.x; d < nd; d += blockDim.x) {
            const uint32_t id = el.idx_key[(long long)g * el.idx_cap + d];
            int2 r = el.idx_rng[(long long)g * el.idx_cap + d];
            if (r.x < 0 || r.y < 0 || r.x + r.y > npairs) {
                atomicOr(a.err, ERR_BOUNDS);
                r = make_int2(0, 0);
            }
            S.drng[d] = r;
            unsigned hs = (id * 2654435761u) & (kCHash - 1);
            for (int probe = 0; probe < kCHash; probe++) {
                if (atomicCAS(&S.hkey[hs], kNoId, id) == kNoId) {
                    S.hden[hs] = (unsigned short)d;
                    break;
                }
                hs = (hs + 1) & (kCHash - 1);
            }
        }
        __syncthreads();
        const float4* pts = nflat <= kSPts ? S.pts : gpts;
        const int* eidx = el.eidx + (long long)g * el.flat_cap;
        const Box b = load_box(a.box + 6 * g);
        const Box bo = load_box(a.idbox_old + 6 * g);
        const long long old_count = bo.count();
        const T* in = a.in + a.in_off[g];
        T* out = a.out + a.out_off[g];
        const uint32_t* idl = a.id_old + a.idoff_old[g];
        const HullElem* elem = el.elem + (long long)g * el.elem_cap;
        const double* eb = el.ebary + 3 * (long long)g * el.bary_cap;
        const int nx = b.nx(), ny = b.ny();
        const int nxy = nx * ny;
        const long long nvox = (long long)nxy * b.nz();
        // a packet voxel's (z, y, x) from its flat index without 64-bit division
        const bool fastdiv = nvox < (1LL << 24) && nx > 0;
        const float rnxy = fastdiv ? __frcp_rn((float)nxy) : 0.f, rnx = fastdiv ? __frcp_rn((float)nx) : 0.f;
        // the filter's error bound: q is within 16 R^2 2^-24 of |v' - p'|^2 - |v'|^2 (the
        // three FMAs, the FP32 rounding of p' and |p'|^2), R^2 the largest |v'|^2 or |p'|^2
        float r2 = org.w;
        {
            const float cx = fmaxf(fabsf((float)b.y0 - org.x), fabsf((float)(b.y1 - 1) - org.x));
            const float cy = fmaxf(fabsf((float)b.x0 - org.y), fabsf((float)(b.x1 - 1) - org.y));
            const float cz = fmaxf(fabsf((float)b.z0 - org.z), fabsf((float)(b.z1 - 1) - org.z));
            r2 = fmaxf(r2, cx * cx + cy * cy + cz * cz);
        }
        const float eps2 = fmaxf(2.f * 16.f * r2 * (1.0f / 16777216.f) * 1.0001f, 1e-6f);
        // passes over consecutive runs of kCVox voxels of the box, across rows and slices,
        // so that a pass holds many packets and few barriers are paid per voxel
        const long long v_end = min(nvox, (item + 1) * kCItem);
        for (long long v0 = item * kCItem; v0 < v_end; v0 += kCVox) {
            const int nv = (int)min((long long)kCVox, v_end - v0);
            for (int d = threadIdx.x; d < nd; d += blockDim.x) S.dcnt[d] = 0;
            if (threadIdx.x == 0) S.pk_next = nwarps;  // packet w goes to warp w, the rest on demand
            __syncthreads();
            // band voxels: their neighbour; voxels whose neighbour no element holds get (1, 1)
            // now.  A batch of voxels per thread: their loads are in flight together.
            constexpr int kBatch = sizeof(T) == 4 ? 16 : 8;
            for (int q0 = threadIdx.x; q0 < nv; q0 += kBatch * blockDim.x) {
                T vals[kBatch];
                uint32_t ids[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    const int q = q0 + u * blockDim.x;
                    const long long f = v0 + q;  // the box's flat [z][y][x] index
                    vals[u] = T(0);
                    ids[u] = 0u;
                    if (q < nv) {
                        vals[u] = in[f];
                        // IDLocal flat-resized onto the box (dimensionalBuffer.h:120-131)
                        ids[u] = f < old_count ? idl[f] : 0u;
                    }
                }
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    const int q = q0 + u * blockDim.x;
                    if (q >= nv) continue;
                    const long long fq = v0 + q;
                    unsigned short dd = kNoD;
                    if (fabs((double)vals[u]) < delta) {
                        const uint32_t id = ids[u];
                        unsigned hs = (id * 2654435761u) & (kCHash - 1);
                        for (int probe = 0; probe < kCHash; probe++) {
                            const uint32_t key = S.hkey[hs];
                            if (key == id) { dd = S.hden[hs]; break; }
                            if (key == kNoId) break;
                            hs = (hs + 1) & (kCHash - 1);
                        }
                        if (dd != kNoD) atomicAdd(&S.dcnt[dd], 1);
                        else correct_voxel(a, elem, g, -1, id, (double)vals[u], (double)out[fq], out + fq);
                    }
                    S.vd[q] = dd;
                }
            }
            __syncthreads();
            if (warp == 0) {  // bucket offsets and packet counts: warp scans over the neighbours
                int run = 0, prun = 0;
                for (int d0 = 0; d0 < nd; d0 += 32) {
                    const int d = d0 + lane;
                    const int c = d < nd ? S.dcnt[d] : 0, pk = (c + kPacket - 1) / kPacket;
                    int ic = c, ip = pk;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int u = __shfl_up_sync(kFull, ic, o), v = __shfl_up_sync(kFull, ip, o);
                        if (lane >= o) { ic += u; ip += v; }
                    }
                    if (d < nd) {
                        S.doff[d] = S.dcur[d] = run + ic - c;
                        S.dpk[d] = prun + ip - pk;
                    }
                    run += __shfl_sync(kFull, ic, 31);
                    prun += __shfl_sync(kFull, ip, 31);
                }
                if (lane == 0) S.dpk[nd] = prun;
            }
            __syncthreads();
            for (int q = threadIdx.x; q < nv; q += blockDim.x) {
                const unsigned short dd = S.vd[q];
                if (dd != kNoD) S.vlist[atomicAdd(&S.dcur[dd], 1)] = (unsigned short)q;
            }
            __syncthreads();
            const int P = S.dpk[nd];
            for (int pk = warp; pk < P;) {
                int lo = 0, hi = nd - 1;  // the neighbour whose packets hold pk
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.dpk[mid] <= pk) lo = mid;
                    else hi = mid - 1;
                }
                const int d = lo;
                const int start = S.doff[d] + (pk - S.dpk[d]) * kPacket;
                const int cnt = min(kPacket, S.doff[d] + S.dcnt[d] - start);
                bool active[kLV];
                int ii[kLV], jj[kLV], kk[kLV], win[kLV];
                long long f[kLV];
                T vin[kLV], vconv[kLV];
                uint32_t id[kLV];
#pragma unroll
                for (int u = 0; u < kLV; u++) {
                    const int slot = lane + 32 * u;
                    active[u] = slot < cnt;
                    const int q = S.vlist[start + (active[u] ? slot : 0)];
                    f[u] = v0 + q;
                    int qz, rem, qy, qx;
                    if (fastdiv) {
                        divmod24((int)f[u], nxy, rnxy, qz, rem);
                        divmod24(rem, nx, rnx, qy, qx);
                    } else {
                        qz = (int)(f[u] / nxy);
                        rem = (int)(f[u] % nxy);
                        qy = rem / nx;
                        qx = rem % nx;
                    }
                    // the point is Vector3d(i, j, k), box.cpp:481
                    kk[u] = b.z0 + qz;
                    ii[u] = b.y0 + qy;
                    jj[u] = b.x0 + qx;
                    // the voxel's input, convolved value and IDLocal, loaded while the search runs
                    vin[u] = T(0);
                    vconv[u] = T(0);
                    id[u] = 0u;
                    if (active[u]) {
                        vin[u] = in[f[u]];
                        vconv[u] = out[f[u]];
                        id[u] = f[u] < old_count ? idl[f[u]] : 0u;
                    }
                }
                const int2 dr = S.drng[d];
                search_packet<kLV>(S, pts, dr.x, dr.y, active, ii, jj, kk, org, eps2, ne, eidx, eb, a.err, win);
#pragma unroll
                for (int u = 0; u < kLV; u++)
                    if (active[u]) correct_voxel(a, elem, g, win[u], id[u], (double)vin[u], (double)vconv[u], out + f[u]);
                int nxt = 0;
                if (lane == 0) nxt = atomicAdd(&S.pk_next, 1);
                pk = __shfl_sync(kFull, nxt, 0);
            }
            __syncthreads();
        }
    }
}

}  // namespace

size_t elements_scratch_per_cta() { return kElemScratch; }
int correction_item_voxels() { return kCItem; }

namespace {
__global__ void faces_kernel(int G, const int* exists, HullElements el, const long long* off, int* count,
                             double* area, uint32_t* grain_a, uint32_t* grain_b) {
    for (int g = 1 + blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        int n = 0;
        if (exists[g]) {
            const int ne = min(max(el.n_elem[g], 0), el.elem_cap);
            const HullElem* E = el.elem + (long long)g * el.elem_cap;
            const uint32_t* ids = el.ids + (long long)g * el.id_cap;
            for (int e = 0; e < ne; e++) {
                if (E[e].type != 1 || E[e].nids < 1) continue;
                const uint32_t nb = ids[E[e].id_off];
                if ((uint32_t)g <= nb) continue;  // each face once, from its higher ID
                if (area) {
                    area[off[g] + n] = E[e].area;
                    grain_a[off[g] + n] = (uint32_t)g;
                    grain_b[off[g] + n] = nb;
                }
                n++;
            }
        }
        if (!area) count[g] = n;
    }
}
}  // namespace

void launch_faces(int G, const int* exists, HullElements el, double /*h*/, const long long* off, int* count,
                  double* area, uint32_t* grain_a, uint32_t* grain_b, cudaStream_t s) {
    faces_kernel<<<(G + 256) / 256, 256, 0, s>>>(G, exists, el, off, count, area, grain_a, grain_b);
}

void launch_elements(const ElementArgs& a, int grid, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(elements_kernel);
    });
    static int resident_on[64] = {};  // CTAs that fit on each device at once
    int dev = 0;
    cudaGetDevice(&dev);
    int& resident = resident_on[dev >= 0 && dev < 64 ? dev : 0];
    if (resident == 0) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, elements_kernel, 32, sizeof(ElemSmem));
        resident = sms * (per_sm > 0 ? per_sm : 1);
    }
    if (grid > resident) grid = resident;
    if (grid > a.scratch_ctas) grid = a.scratch_ctas;
    elements_kernel<<<grid, 32, sizeof(ElemSmem), s>>>(a);
}

template <typename T>
void launch_correction(const CorrectionArgs<T>& a, int grid, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] { allow_max_dynamic_smem(correction_kernel<T>); });
    correction_kernel<T><<<grid, kCThreads, sizeof(CorrSmem), s>>>(a);
}

template void launch_correction<double>(const CorrectionArgs<double>&, int, cudaStream_t);
template void launch_correction<float>(const CorrectionArgs<float>&, int, cudaStream_t);

}  // namespace gg

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
//   correction_kernel: a CTA per (grain, z-slice); every voxel with |input| < delta
//     looks its IDLocal neighbour up in the index and scans only the elements that hold
//     it, in search order, skipping an element when the distance to its bounding box is
//     already >= the best distance (an exact bound: no barycenter inside can win under
//     the strict <).  The energies use CUDA's acos/log/exp/pow: within a few ULP of the
//     reference's libm, not bit-identical.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr double kPi = 3.14159265358979323846;  // ggLS.h:25
constexpr int kLMax = 256;    // distinct neighbour lists (= elements) per hull
constexpr int kJIds = 48;     // IDs of one (merged) junction
constexpr unsigned kNoId = 0xFFFFFFFFu;

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

// TripleLine of (me, n0, n1): energy and mobility (InterfacialElement.cpp:119-170)
__device__ void triple_line(const HullPhysics& ph, uint32_t me, uint32_t n0, uint32_t n1, double& energy,
                            double& mobility) {
    const double t0 = misorientation(ph, me, n0), t1 = misorientation(ph, n0, n1), t2 = misorientation(ph, me, n1);
    double avg = 0;
    avg += mobility_of(ph, t0);
    avg += mobility_of(ph, t1);
    avg += mobility_of(ph, t2);
    avg /= 3;
    const double ds = 3 * sqrt(3 * ph.ds * ph.ds);
    mobility = 1. / ((1. / (ds * ph.tl_drag)) + 1. / avg);
    double sigma = energy_of(ph, t0) - energy_of(ph, t1) + energy_of(ph, t2);
    if (sigma < 0.01) sigma = 0.01;
    if (sigma > 1.0) sigma = 1.0;
    energy = sigma;
}

// Vector3d (a - b).squaredNorm(): Eigen's unrolled sum c0 + (c1 + c2)
__device__ __forceinline__ double sqdist(const double* a, const double* b) {
    const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return d0 * d0 + (d1 * d1 + d2 * d2);
}

// ---------------------------------------------------------------------------------
// element construction
// ---------------------------------------------------------------------------------

// A junction being merged: its member lists (keys) chained through next_key, its IDs.
struct Junction {
    int head, tail;   // member keys
    int nids;
    int type;         // 3 QJ, 4 HJ
    double pos[3];
    uint32_t ids[kJIds];
};

struct ElemSmem {
    uint32_t lists[kLMax][8];
    int cnt[kLMax];     // triangles per list
    int off[kLMax];     // first barycenter of the list in the grouped array
    int fill[kLMax];
    int next_key[kLMax];
    double energy[kLMax], mobility[kLMax];
    Junction jn[kLMax];  // working junctions
    int qlist[kLMax], hlist[kLMax];
    int nl, nq, nh, nj;
};

// The junction's position: the mean of its barycenters in member order
// (QuadrupleJunction / HighOrderJunction::computePosition, InterfacialElement.cpp:394-406)
__device__ void junction_position(Junction& J, const ElemSmem& S, const double* eb, int bary_cap, int* err) {
    double p0 = 0, p1 = 0, p2 = 0;
    int n = 0;
    for (int k = J.head; k >= 0; k = S.next_key[k]) {
        if (k >= kLMax || S.off[k] < 0 || S.off[k] + S.cnt[k] > bary_cap) {
            atomicOr(err, ERR_BOUNDS);
            break;
        }
        const double* b = eb + 3 * (long long)S.off[k];
        for (int i = 0; i < S.cnt[k]; i++) {
            p0 += b[3 * i];
            p1 += b[3 * i + 1];
            p2 += b[3 * i + 2];
        }
        n += S.cnt[k];
    }
    const double d = (double)n;
    J.pos[0] = p0 / d;
    J.pos[1] = p1 / d;
    J.pos[2] = p2 / d;
}

__device__ __forceinline__ void push_id(Junction& J, uint32_t id, int* err) {
    if (J.nids < kJIds) J.ids[J.nids++] = id;
    else atomicOr(err, ERR_HULL);
}

__device__ __forceinline__ void chain(ElemSmem& S, Junction& A, const Junction& B) {
    S.next_key[A.tail] = B.head;
    A.tail = B.tail;
}

__global__ void __launch_bounds__(32) elements_kernel(ElementArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ElemSmem& S = *reinterpret_cast<ElemSmem*>(smem_raw);
    const int lane = threadIdx.x;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        if (!a.exists[g]) continue;
        const long long cb = (long long)g * a.cap.cap;
        const int nrec = a.cap.n_rec[g], ntri = a.cap.n_tri[g];
        uint32_t* rec_list = a.cap.rec_list + 8 * cb;
        int* rec_ntri = a.cap.rec_ntri + cb;
        const double* bary = a.cap.bary + 3 * cb;
        double* eb = a.el.ebary + 3 * (long long)g * a.el.bary_cap;
        if (lane == 0) S.nl = 0;
        __syncwarp();
        // 1. distinct lists in first-seen order (MarchingCubesAlgorithm::insertNeighborList,
        //    marchingCubes.cpp:605-618); the key goes into the record's upper bits
        for (int r = 0; r < nrec; r++) {
            uint32_t mine[8];
#pragma unroll
            for (int q = 0; q < 8; q++) mine[q] = rec_list[8 * r + q];
            const int nl = S.nl;
            int found = -1;
            for (int base = 0; base < nl && found < 0; base += 32) {
                const int c = base + lane;
                bool eq = c < nl;
#pragma unroll
                for (int q = 0; q < 8; q++) eq = eq && S.lists[c < nl ? c : 0][q] == mine[q];
                const unsigned m = __ballot_sync(0xffffffffu, eq);
                if (m) found = base + __ffs(m) - 1;
            }
            if (found < 0) {
                found = nl;
                if (nl < kLMax) {
                    if (lane < 8) S.lists[nl][lane] = mine[lane];
                    if (lane == 0) S.nl = nl + 1;
                } else if (lane == 0) {
                    atomicOr(a.err, ERR_HULL);
                }
            }
            if (lane == 0) rec_ntri[r] = (rec_ntri[r] & 0xFF) | ((found < kLMax ? found : 0) << 8);
            __syncwarp();
        }
        const int nl = S.nl;
        // 2. triangles per list and the grouped offsets
        for (int k = lane; k < nl; k += 32) S.cnt[k] = 0;
        __syncwarp();
        if (lane == 0) {
            for (int r = 0; r < nrec; r++) S.cnt[rec_ntri[r] >> 8] += rec_ntri[r] & 0xFF;
            int run = 0;
            for (int k = 0; k < nl; k++) {
                S.off[k] = run;
                S.fill[k] = 0;
                S.next_key[k] = -1;
                run += S.cnt[k];
            }
            if (run > a.el.bary_cap) atomicOr(a.err, ERR_HULL);
        }
        __syncwarp();
        // 3. barycenters grouped by list, in triangle order (subDivideTrianglesToInterfacialElements)
        if (lane == 0) {
            int t = 0;
            for (int r = 0; r < nrec; r++) {
                const int k = rec_ntri[r] >> 8, nt = rec_ntri[r] & 0xFF;
                for (int q = 0; q < nt; q++, t++) {
                    const int pos = S.off[k] + S.fill[k]++;
                    if (pos < a.el.bary_cap && t < ntri) {
                        eb[3 * pos] = bary[3 * t];
                        eb[3 * pos + 1] = bary[3 * t + 1];
                        eb[3 * pos + 2] = bary[3 * t + 2];
                    }
                }
            }
        }
        // 4. one element per list: energy and mobility (computeGrainBoundaryElements)
        for (int k = lane; k < nl; k += 32) {
            const uint32_t* L = S.lists[k];
            int count = 0;
            for (int j = 0; j < 8; j++) count += L[j] == kNoId ? 0 : 1;
            double E = 1.0, M = 1.0;
            uint32_t nb[8];
            int nn = 0;
            if (count == 2) {
                nb[nn++] = (uint32_t)g != L[0] ? L[0] : L[1];
            } else {
                const int lim = count == 3 ? 3 : (count == 4 ? 4 : count);
                for (int i = 0; i < lim; i++)
                    if ((uint32_t)g != L[i]) nb[nn++] = L[i];
            }
            if (count == 2) {
                const double t = misorientation(a.ph, g, nb[0]);
                M = mobility_of(a.ph, t);
                E = energy_of(a.ph, t);
            } else if (count == 3) {
                triple_line(a.ph, g, nb[0], nb[1], E, M);
            } else if (count == 4) {
                double E1, M1, E2, M2, E3, M3;
                triple_line(a.ph, g, nb[0], nb[1], E1, M1);
                triple_line(a.ph, g, nb[1], nb[2], E2, M2);
                triple_line(a.ph, g, nb[0], nb[2], E3, M3);
                M = (M1 + M2 + M3) / 3.0;
                E = (E1 + E2 + E3) / 3.0;
            }
            S.energy[k] = E;
            S.mobility[k] = M;
        }
        __syncwarp();
        // 5. junctions and their merging (computeJunctionPosition + mergeJunction,
        //    grainHull.cpp:267-275, 483-531); sequential, as the reference
        if (lane == 0) {
            S.nq = S.nh = S.nj = 0;
            for (int k = 0; k < nl; k++) {
                int count = 0;
                for (int j = 0; j < 8; j++) count += S.lists[k][j] == kNoId ? 0 : 1;
                if (count < 4 && count > 1) continue;  // 2 GB, 3 TL; everything else is a junction
                Junction& J = S.jn[S.nj];
                J.head = J.tail = k;
                J.nids = 0;
                J.type = count == 4 ? 3 : 4;
                for (int i = 0; i < count; i++)
                    if ((uint32_t)g != S.lists[k][i]) push_id(J, S.lists[k][i], a.err);
                junction_position(J, S, eb, a.el.bary_cap, a.err);
                if (J.type == 3) S.qlist[S.nq++] = S.nj;
                else S.hlist[S.nh++] = S.nj;
                S.nj++;
            }
            // quadruple points closer than 2: a new high-order junction from the pair
            for (int i = 0; i < S.nq; i++) {
                for (int j = i + 1; j < S.nq; j++) {
                    Junction& A = S.jn[S.qlist[i]];
                    Junction& B = S.jn[S.qlist[j]];
                    if (sqrt(sqdist(A.pos, B.pos)) < 2) {
                        if (S.nj >= kLMax) { atomicOr(a.err, ERR_HULL); break; }
                        Junction& H = S.jn[S.nj];
                        H.type = 4;
                        H.nids = 0;
                        for (int q = 0; q < 3; q++) push_id(H, A.ids[q], a.err);
                        for (int q = 0; q < 3; q++) {  // B's IDs that A already has (sic)
                            bool dup = false;
                            for (int u = 0; u < 3; u++) dup |= H.ids[u] == B.ids[q];
                            if (dup) push_id(H, B.ids[q], a.err);
                        }
                        H.head = A.head;
                        H.tail = A.tail;
                        chain(S, H, B);
                        junction_position(H, S, eb, a.el.bary_cap, a.err);
                        // erase i and j (j - 1 after the first erase), then append H
                        for (int u = j; u < S.nq - 1; u++) S.qlist[u] = S.qlist[u + 1];
                        for (int u = i; u < S.nq - 2; u++) S.qlist[u] = S.qlist[u + 1];
                        S.nq -= 2;
                        S.hlist[S.nh++] = S.nj++;
                        i--;
                        break;
                    }
                }
            }
            // quadruple points closer than 2 to a high-order junction join it
            for (int k = 0; k < S.nh; k++)
                for (int i = 0; i < S.nq; i++) {
                    Junction& H = S.jn[S.hlist[k]];
                    Junction& Q = S.jn[S.qlist[i]];
                    if (sqrt(sqdist(Q.pos, H.pos)) < 2) {
                        chain(S, H, Q);
                        for (int q = 0; q < Q.nids; q++) push_id(H, Q.ids[q], a.err);
                        junction_position(H, S, eb, a.el.bary_cap, a.err);
                        for (int u = i; u < S.nq - 1; u++) S.qlist[u] = S.qlist[u + 1];
                        S.nq--;
                        i--;
                    }
                }
            // high-order junctions closer than 2 merge
            for (int i = 0; i < S.nh; i++)
                for (int k = i + 1; k < S.nh; k++) {
                    Junction& A = S.jn[S.hlist[i]];
                    Junction& B = S.jn[S.hlist[k]];
                    if (sqrt(sqdist(A.pos, B.pos)) < 2) {
                        chain(S, A, B);
                        for (int q = 0; q < B.nids; q++) push_id(A, B.ids[q], a.err);
                        junction_position(A, S, eb, a.el.bary_cap, a.err);
                        for (int u = k; u < S.nh - 1; u++) S.hlist[u] = S.hlist[u + 1];
                        S.nh--;
                        k--;
                    }
                }
        }
        __syncwarp();
        // 6. the element table in search order: HJ, QJ, TL, GB
        if (lane == 0) {
            HullElem* E = a.el.elem + (long long)g * a.el.elem_cap;
            uint32_t* ids = a.el.ids + (long long)g * a.el.id_cap;
            int2* segs = a.el.segs + (long long)g * a.el.seg_cap;
            int ne = 0, ni = 0, ns = 0;
            bool over = false;
            auto emit = [&](int type, const uint32_t* id_src, int nid, int head, bool chained, double en, double mo) {
                if (ne >= a.el.elem_cap || ni + nid > a.el.id_cap) { over = true; return; }
                HullElem& e = E[ne++];
                e.type = type;
                e.id_off = ni;
                e.nids = nid;
                for (int q = 0; q < nid; q++) ids[ni++] = id_src[q];
                e.seg_off = ns;
                e.nseg = 0;
                double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
                for (int k = head; k >= 0; k = chained ? S.next_key[k] : -1) {
                    if (ns >= a.el.seg_cap) { over = true; break; }
                    if (k >= kLMax || S.off[k] < 0 || S.off[k] + S.cnt[k] > a.el.bary_cap) {
                        atomicOr(a.err, ERR_BOUNDS);
                        break;
                    }
                    segs[ns++] = make_int2(S.off[k], S.cnt[k]);
                    e.nseg++;
                    for (int i = 0; i < S.cnt[k]; i++)
                        for (int c = 0; c < 3; c++) {
                            const double v = eb[3 * (long long)(S.off[k] + i) + c];
                            lo[c] = fmin(lo[c], v);
                            hi[c] = fmax(hi[c], v);
                        }
                }
                e.energy = en;
                e.mobility = mo;
                for (int c = 0; c < 3; c++) {
                    e.lo[c] = lo[c];
                    e.hi[c] = hi[c];
                }
            };
            for (int i = 0; i < S.nh; i++) {
                const Junction& J = S.jn[S.hlist[i]];
                // a junction made from one list keeps that list's energy (1 for HJ)
                emit(4, J.ids, J.nids, J.head, true, 1.0, 1.0);
            }
            for (int i = 0; i < S.nq; i++) {
                const Junction& J = S.jn[S.qlist[i]];
                emit(3, J.ids, J.nids, J.head, true, S.energy[J.head], S.mobility[J.head]);
            }
            for (int pass = 2; pass >= 1; pass--)  // TL, then GB, each in key order
                for (int k = 0; k < nl; k++) {
                    int count = 0;
                    for (int j = 0; j < 8; j++) count += S.lists[k][j] == kNoId ? 0 : 1;
                    if ((pass == 2 && count != 3) || (pass == 1 && count != 2)) continue;
                    uint32_t nb[3];
                    int nn = 0;
                    if (count == 2) nb[nn++] = (uint32_t)g != S.lists[k][0] ? S.lists[k][0] : S.lists[k][1];
                    else
                        for (int q = 0; q < 3; q++)
                            if ((uint32_t)g != S.lists[k][q]) nb[nn++] = S.lists[k][q];
                    emit(pass, nb, nn, k, false, S.energy[k], S.mobility[k]);
                }
            if (over) atomicOr(a.err, ERR_HULL);
            a.el.n_elem[g] = ne;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------
// the correction
// ---------------------------------------------------------------------------------

// projectPointToGrainBoundary: the nearest barycenter among the elements holding id;
// returns (m_energy, m_mobility) of its element, (1, 1) when none holds id.
__device__ void project(const HullElements& el, int g, const double* p, uint32_t id, double& E, double& M,
                        int* err) {
    int ne = el.n_elem[g];
    if (ne < 0 || ne > el.elem_cap) {
        atomicOr(err, ERR_BOUNDS);
        ne = 0;
    }
    const HullElem* elem = el.elem + (long long)g * el.elem_cap;
    const uint32_t* ids = el.ids + (long long)g * el.id_cap;
    const int2* segs = el.segs + (long long)g * el.seg_cap;
    const double* eb = el.ebary + 3 * (long long)g * el.bary_cap;
    double best = 10000000.0;
    E = 1.;
    M = 1.;
    for (int i = 0; i < ne; i++) {
        const HullElem& e = elem[i];
        // the IDs the reference compares: all for a high-order junction, else 3, 2, 1
        const int nc = e.type == 4 ? e.nids : min(e.nids, e.type);
        if (e.id_off < 0 || nc < 0 || e.id_off + nc > el.id_cap || e.seg_off < 0 || e.nseg < 0 ||
            e.seg_off + e.nseg > el.seg_cap) {
            atomicOr(err, ERR_BOUNDS);
            continue;
        }
        bool found = false;
        for (int q = 0; q < nc; q++) found |= ids[e.id_off + q] == id;
        if (!found) continue;
        // lower bound of every barycenter's distance: none can beat best if it is >= best
        double lo[3];
        for (int c = 0; c < 3; c++) lo[c] = p[c] < e.lo[c] ? e.lo[c] : (p[c] > e.hi[c] ? e.hi[c] : p[c]);
        if (sqdist(p, lo) >= best) continue;
        for (int sgi = 0; sgi < e.nseg; sgi++) {
            const int2 sg = segs[e.seg_off + sgi];
            if (sg.x < 0 || sg.y < 0 || sg.x + sg.y > el.bary_cap) {
                atomicOr(err, ERR_BOUNDS);
                continue;
            }
            for (int b = 0; b < sg.y; b++) {
                const double d = sqdist(p, eb + 3 * (long long)(sg.x + b));
                if (d < best) {
                    best = d;
                    E = e.energy;
                    M = e.mobility;
                }
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128) correction_kernel(CorrectionArgs<T> a) {
    const double delta = a.geo.delta;
    const double ts = 1 / 1.21;  // TimeSlope, grainhdl.cpp:1432
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box b = load_box(a.box + 6 * g);
        const int k = b.z0 + w.local;
        const Box bo = load_box(a.idbox_old + 6 * g);
        const long long old_count = bo.count();
        const T* in = a.in + a.in_off[g];
        T* out = a.out + a.out_off[g];
        const uint32_t* idl = a.id_old + a.idoff_old[g];
        const int nx = b.nx(), ny = b.ny();
        for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {
            const int i = b.y0 + q / nx, j = b.x0 + q % nx;
            const long long f = b.at(i, j, k);
            const double val = (double)in[f];
            if (!(fabs(val) < delta)) continue;
            // IDLocal flat-resized onto the box (dimensionalBuffer.h:120-131)
            const uint32_t id = f < old_count ? idl[f] : 0u;
            const double p[3] = {(double)i, (double)j, (double)k};  // Vector3d(i, j, k), box.cpp:481
            double E, M;
            project(a.el, g, p, id, E, M, a.err);
            // GBInfo(m_energy, m_mobility) fills (mobility, energy): field energy = M, field mobility = E
            const double fe = M, fm = E;
            double o = val + ((double)out[f] - val) * fe * fm * 1.0;
            if (a.ph.use_see) {
                const bool alive = id == 0 || (id <= (uint32_t)a.G && a.present[id]);
                const double fs = alive ? (a.ph.see[g] - a.ph.see[id]) * fm * a.ph.dt / (ts * ts) : 0.0;
                o = o - fs;
            }
            out[f] = (T)o;
        }
    }
}

}  // namespace

void launch_elements(const ElementArgs& a, int grid, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        allow_max_dynamic_smem(elements_kernel);
        configured = true;
    }
    elements_kernel<<<grid, 32, sizeof(ElemSmem), s>>>(a);
}

template <typename T>
void launch_correction(const CorrectionArgs<T>& a, int grid, cudaStream_t s) {
    correction_kernel<T><<<grid, 128, 0, s>>>(a);
}

template void launch_correction<double>(const CorrectionArgs<double>&, int, cudaStream_t);
template void launch_correction<float>(const CorrectionArgs<float>&, int, cudaStream_t);

}  // namespace gg

// gg_kernels.cuh -- launch interfaces of the level-set stage kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "gg_common.cuh"

namespace gg {

// ---- planner (gg_plan.cu) ----
struct PlanArgs {
    int G;
    const int* present;
    const int* exists;
    const int* box;           // boxes to plan from (6 per grain)
    int only_existing;        // 1: grains with present && exists; 0: present
    long long* off;           // out: element offsets (aligned), may be null
    long long capacity;       // arena capacity in elements (off != null)
    long long* spec_off;      // out: half-spectrum offsets (complex elements), may be null
    long long spec_capacity;
    int* toff_n;              // out: tile offsets with n tiles per grain, may be null
    int* toff_slab;           // out: tile offsets with ceil(n / slab) tiles per grain, or with
                              // ceil(n^2 / row_tile) when row_tile > 0; may be null
    int slab;
    int row_tile;
    // > 0 (with row_tile): grains with side above it get no row tiles in toff_slab and
    // their n tiles in toff_big instead (the convolution's two size classes)
    int class_side;
    int* toff_big;            // out: n tiles per grain of side > class_side, may be null
    int* toff_one;            // out: tile offsets with one tile per grain, may be null
    int* box_copy;            // out: copy of box (6 per grain), may be null
    long long* off_copy;      // out: copy of off, may be null
    long long* total_voxels;  // out: sum of n^3 over planned grains (device scalar), may be null
    int* err;
};
void launch_plan(const PlanArgs& a, cudaStream_t s);

// ---- largest-first work items for the per-grain kernels (gg_plan.cu) ----
// order[0, n) = the grains with a tile in `toff_one`, by decreasing box voxels; grain
// order[i] is cut into items of item_vox box voxels (the last one shorter), numbered
// from item_off[i] on (item_off[G + 1] = all items).  The kernels that take it fetch
// item numbers from a counter (*queue, zeroed here), so that the largest grains start
// first, the rest fill in, and no grain is longer than one item on one CTA.
struct WorkOrder {
    int* keys;               // G + 1 scratch keys
    int* keys_out;           // G + 1: box voxels + 1 in order, 0 for grains without a tile
    int* vals;               // G + 1 (grain IDs)
    int* order;              // G + 1 (out)
    int* item_off;           // G + 2 (out)
    void* temp;              // radix-sort and scan scratch
    size_t temp_bytes;
    int* queue;              // kQueues counters (out: zeroed)
};
constexpr int kQueues = 4;
size_t work_order_temp_bytes(int G);
void launch_work_order(const WorkOrder& w, int G, const int* toff_one, const int* box, int item_vox,
                       cudaStream_t s);

// The position i of work item t in the order: the last i in [0, G] with item_off[i] <= t.
__device__ __forceinline__ int work_position(const int* __restrict__ item_off, int G, int t) {
    int lo = 0, hi = G + 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(item_off + mid) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// Copy box + offsets of every present grain from one layout to another.
void launch_copy_layout(int G, const int* present, const int* box_src, const long long* off_src, int* box_dst,
                        long long* off_dst, cudaStream_t s);

// ---- comparison (gg_compare.cu) ----
constexpr int kTX = 8, kTY = 4, kTZ = 2;  // domain tile of the comparison

// Grains whose (input) boxes reach each domain tile, as CSR over tiles.
struct TileBins {
    int ntx, nty, ntz;
    int* count;               // n_tiles + 1
    int* off;                 // n_tiles + 1 (exclusive scan of count)
    int* cursor;              // n_tiles + 1
    uint32_t* entries;        // grain IDs
    long long capacity;
    int* max_count;           // device scalar: most grains reaching one tile
    void* temp;               // device-wide scan scratch (domain tiles), temp_bytes
    size_t temp_bytes;
};
// Scratch bytes of launch_exclusive_scan over n ints; the scan writes out[i] = sum of
// in[0 .. i - 1] for i < n.
size_t exclusive_scan_temp_bytes(int n);
void launch_exclusive_scan(void* temp, size_t temp_bytes, const int* in, int* out, int n, cudaStream_t s);
void launch_bin(const TileBins& tb, int G, const int* exists, const int* box, int* err, cudaStream_t s);
long long bin_capacity(int G, int side);

// son := cmp for every existing grain (m_secondOrderNeighbours = m_comparisonList).
struct ListCopyArgs {
    int G;
    const int* toff;          // one tile per existing grain
    const uint32_t* cmp;
    const int* n_cmp;
    uint32_t* son;
    int* n_son;
    int list_cap;
};
void launch_copy_lists(const ListCopyArgs& a, int grid, cudaStream_t s);

// Initial comparison lists (the reference's R-tree search, grainhdl.cpp:1029-1054):
// every present grain whose box touches the grain's box (inclusive), in ascending ID
// order, written to both list rows.
struct DefaultListArgs {
    int G;
    const int* present;
    const int* box;
    uint32_t* cmp;
    int* n_cmp;
    uint32_t* son;
    int* n_son;
    int list_cap;
    int* err;
};
void launch_default_lists(const DefaultListArgs& a, cudaStream_t s);

// Caller-given lists: packed IDs with per-grain offsets scattered into both list rows.
void launch_scatter_lists(int G, const int64_t* offsets, const uint32_t* ids, uint32_t* cmp, int* n_cmp,
                          uint32_t* son, int* n_son, int list_cap, cudaStream_t s);

template <typename T>
struct CompareArgs {
    Geometry geo;
    TileBins bins;
    int mcap;                 // most grains one tile holds (shared-memory sizing)
    Arena<T> in;              // convolved SDFs (self and neighbours)
    Arena<T> out;             // comparison result written here (same boxes as in)
    const uint32_t* id_old;   // IDLocal of the previous layout
    const int* idbox_old;
    const long long* idoff_old;
    uint32_t* id_new;         // IDLocal on the current boxes
    const long long* idoff_new;
    const uint32_t* cmp;      // comparison lists (position = list order)
    const int* n_cmp;
    int list_cap;
    const unsigned long long* pos_table;  // per grain: neighbour ID -> list position (pos_tables)
    int pos_cap;
    int* newbox;              // per grain min/max (pre-initialised)
    int* err;
    // 1: executeComparison then executeSetComparison (the loop's comparison stage);
    // 0: executeComparison alone (LSbox::recalculateIDLocal after a grid coarsening,
    //    box.cpp:2697-2700): out = the largest listed neighbour value, no new box, and
    //    grains that do not exist are left alone (box.cpp:892-893)
    int set_comparison;
    const int* exists;        // read when set_comparison == 0
};
template <typename T>
void launch_compare(const CompareArgs<T>& a, int grid, cudaStream_t s);
size_t compare_smem_bytes(int mcap, bool fp64);
void launch_newbox_init(int G, const int* present, const int* exists, const int* box, int* newbox, cudaStream_t s);

// ---- list update (gg_lists.cu) ----
struct ListArgs {
    int G;
    const int* toff;          // one tile per existing grain
    const int* exists;
    const int* box;           // in-arena boxes (LSbox::checkIntersection uses m_inputDistance)
    const uint32_t* son;
    const int* n_son;
    uint32_t* cmp;
    int* n_cmp;
    int list_cap;
    TileBins cells;           // existing grains by the kListCell^3 domain cells their boxes touch
    const unsigned long long* pos;  // position tables of the son lists (PosTableArgs)
    int pos_cap;
    int* err;
};
// Shared memory of the list update: two bitmaps over the IDs 0..G and 2048 selected
// (position, ID) pairs.
__host__ __device__ inline int list_bitmap_words(int G) { return (G + 32) >> 5; }
inline size_t list_smem_bytes(int G) { return (size_t)list_bitmap_words(G) * 8 + 2048 * 8; }
void launch_update_lists(const ListArgs& a, int grid, cudaStream_t s);
// The candidate cells of the list update: every existing grain under each cell of
// kListCell^3 voxels that its inclusive box [x0, x1] x [y0, y1] x [z0, z1] reaches.
constexpr int kListCell = 16;
void launch_list_bins(const TileBins& tb, int G, const int* exists, const int* box, int* err, cudaStream_t s);
long long list_bin_capacity(int G, int side);

// Per grain an open-addressing table (ID << 32 | list position) of the comparison list,
// pos_cap slots per grain of which pos_table_size(K) are used; built once per step
// and probed by every comparison tile the grain's box reaches.
struct PosTableArgs {
    int G;
    const int* toff;          // one tile per existing grain; null: every present grain
    const int* present;
    const uint32_t* cmp;
    const int* n_cmp;
    int list_cap;
    unsigned long long* table;
    int pos_cap;              // power of two >= 2 list_cap
    int* err;
};
void launch_pos_tables(const PosTableArgs& a, int grid, cudaStream_t s);
__host__ __device__ inline int pos_table_size(int K, int cap) {
    int n = 64;
    while (n < 4 * K && n < cap) n <<= 1;  // load factor <= 1/4 while it fits
    return n;
}

// ---- hull of the last level set, for the convolution correction (gg_hull.cu) ----
// Written by the marching-cubes kernel when the correction is on: per grain, the
// neighbour list of every active cube in cube order (8 IDs, 0xFFFFFFFF padded) with its
// triangle count, and every triangle's barycenter in emission order.
struct HullCapture {
    int cap;                  // cube records and triangles per grain
    uint32_t* rec_list;       // (G + 1) x cap x 8
    int* rec_ntri;            // (G + 1) x cap
    double* bary;             // (G + 1) x cap x 3
    double* tarea;            // (G + 1) x cap: |AB x BC| / 2 of each triangle (computeSurfaceArea's term)
    int* n_rec;               // G + 1
    int* n_tri;               // G + 1
    int* diag;                // which hull capacity overflowed (HULL_* bits)
};

// The capacity behind an ERR_HULL, for the error message.
enum HullDiag : int {
    HULL_TRIANGLES = 1,   // triangles of one hull beyond hull_capacity
    HULL_RECORDS = 2,     // active cubes of one hull beyond hull_capacity
    HULL_LISTS = 4,       // distinct neighbour lists of one hull (256)
    HULL_JUNCTION_IDS = 8,// IDs of one merged junction
    HULL_JUNCTIONS = 16,  // junctions of one hull (256)
    HULL_JOBS = 32,       // misorientations of one hull's elements
    HULL_TABLE = 64,      // element, ID, segment or chunk table of one hull
    HULL_INDEX = 128,     // neighbour -> elements index of one hull
};

// One interfacial element of a grain's mesh (grainHull.cpp:187-531), in the order
// projectPointToGrainBoundary searches them (high-order junctions, quadruple
// junctions, triple lines, grain boundaries).
struct HullElem {
    int type;                 // 1 GB, 2 TL, 3 QJ, 4 HJ
    int nids, id_off;         // neighbour IDs in the grain's ID pool
    int seg_off, nseg;        // barycenter segments (start, count) in the grain's segment pool
    int pbase, pcount;        // its barycenters, contiguous, in the flattened FP32 copy (ebf)
    double energy, mobility;  // m_energy, m_mobility
    double area;              // GrainBoundary::computeArea (InterfacialElement.cpp:81-91); 0 for junctions
    double lo[3], hi[3];      // bounding box of its barycenters
};

struct HullElements {
    int elem_cap, id_cap, seg_cap, bary_cap, idx_cap, pair_cap;
    int flat_cap;             // entries of ebf / eidx per grain: bary_cap + one padding per element
    int* n_elem;              // G + 1
    HullElem* elem;           // (G + 1) x elem_cap
    uint32_t* ids;            // (G + 1) x id_cap
    int2* segs;               // (G + 1) x seg_cap
    double* ebary;            // (G + 1) x bary_cap x 3, barycenters grouped by neighbour list
    double* earea;            // (G + 1) x bary_cap, their triangles' area terms in the same order
    // The same barycenters for the correction's FP32 filter, element by element in table
    // order (element e's at [pbase, pbase + pcount), pbase even, an odd run padded by one
    // entry with |p - o|^2 = 3e38): (p - o, |p - o|^2) in FP32, p - o and its square taken
    // in FP64 first, with o the grain's integer origin.  Pairs of entries are interleaved
    // as (x0, x1, y0, y1), (z0, z1, w0, w1) for the packed FMA.
    float4* ebf;              // (G + 1) x flat_cap
    int* eidx;                // (G + 1) x flat_cap: position of each of them in ebary (-1: padding)
    int* n_flat;              // G + 1: barycenters in ebf
    float4* eorg;             // G + 1: (o.x, o.y, o.z, largest |p - o|^2 of the grain)
    // neighbour ID -> the elements whose searched IDs hold it, in search order
    int* n_idx;               // G + 1: distinct IDs
    uint32_t* idx_key;        // (G + 1) x idx_cap
    int2* idx_rng;            // (G + 1) x idx_cap: (first, count) in idx_elem
    unsigned short* idx_elem; // (G + 1) x pair_cap
};

struct HullPhysics {
    const double4* quat;      // orientation of grain 0..G (0 = the boundary grain)
    const double* see;        // m_StoredElasticEnergy of grain 0..G
    int unique_gb;            // Settings::UniqueGBEnergies
    int mobility_model;       // Settings::UseMobilityModel
    int use_see;              // Settings::UseStoredElasticEnergy
    double tl_drag;           // Settings::TripleLineDrag
    double ds;                // 1 / realDomainSize
    double dt;                // TimeStepSize / realDomainSize^2
};

struct ElementArgs {
    int G;
    const int* toff;          // one tile per present grain
    const int* exists;
    HullCapture cap;
    HullElements el;
    HullPhysics ph;
    unsigned char* scratch;   // scratch_ctas x elements_scratch_per_cta() bytes
    int scratch_ctas;         // the launch uses at most this many CTAs
    const int* order;         // the grains of toff by decreasing box (WorkOrder, one item
    const int* item_off;      // each), fetched through *queue
    int* queue;
    int* err;
};
size_t elements_scratch_per_cta();
void launch_elements(const ElementArgs& a, int grid, cudaStream_t s);

// GrainHull::get_Faces (grainHull.cpp:1330-1339) of every existing grain: its grain
// boundary elements toward lower IDs.  Counting pass (out == nullptr: count[g] = faces of
// g), then writing pass at the exclusive offsets off[g].
void launch_faces(int G, const int* exists, HullElements el, double h, const long long* off, int* count,
                  double* area, uint32_t* grain_a, uint32_t* grain_b, cudaStream_t s);

template <typename T>
struct CorrectionArgs {
    int G;
    Geometry geo;
    const int* toff;          // one tile per convolved grain
    const int* present;
    const int* box;           // current (cubic) boxes
    const T* in;              // input of the convolution
    const long long* in_off;
    T* out;                   // convolved, corrected in place
    const long long* out_off;
    const uint32_t* id_old;   // IDLocal of the last comparison, flat-resized onto the box
    const int* idbox_old;
    const long long* idoff_old;
    HullElements el;
    HullPhysics ph;
    const int* order;         // grains by decreasing box (WorkOrder) and their work items,
    const int* item_off;      // fetched through *queue
    int* queue;
    int* err;
};
int correction_item_voxels();  // box voxels of one work item of the correction
template <typename T>
void launch_correction(const CorrectionArgs<T>& a, int grid, cudaStream_t s);

// ---- marching cubes + hull statistics (gg_mc.cu) ----
template <typename T>
struct MCArgs {
    int G;
    Geometry geo;
    const int* toff;          // one tile per present grain
    int* present;
    int* exists;
    Arena<T> in;              // compared SDF
    const uint32_t* idl;      // IDLocal (same layout as in)
    const long long* idoff;
    const int* newbox;        // from the comparison
    int* out_box;             // new box (resized to cube) written here for existing grains
    double* volume;
    double* surface;
    uint32_t* nb;
    int* n_nb;
    int nb_cap;
    HullCapture hull;         // hull.cap = 0: not captured
    int* err;
    // 1: extractContour after a grid coarsening (grainhdl.cpp:1486-1495): every present
    // grain's hull is rebuilt (none is deleted) and newbox is the resized grid's box,
    // taken as it is (then resized to a cube) rather than widened by the border
    int regrid;
    const int* order;         // the grains of toff by decreasing box (WorkOrder, one item
    const int* item_off;      // each), fetched through *queue
    int* queue;
};
template <typename T>
void launch_mc(const MCArgs<T>& a, int grid, int side, cudaStream_t s);
// Dynamic shared memory of the marching-cubes kernel for boxes up to `side`.
size_t mc_slab_bytes(int side);

// ---- grid coarsening (gg_coarsen.cu) ----
// LSbox::resizeGrid's new boxes (box.cpp:2595-2621): each present grain's output box
// scaled by h_old / h_new (`scaled`, the reference's m_newXMin..), then resized to a cube
// on the new grid (`new_box`).
struct RegridBoxArgs {
    int G;
    const int* present;
    const int* old_box;       // m_outputDistance's box on the old grid
    int* scaled;
    int* new_box;
    double ratio;             // h_old / h_new
    int gb, M_new;
    int* err;
};
void launch_regrid_boxes(const RegridBoxArgs& a, cudaStream_t s);
// The trilinear re-sampling of resizeGrid (box.cpp:2623-2690) into the new boxes.
template <typename T>
struct ResampleArgs {
    int G;
    const int* toff;          // z-slices of the new boxes
    Arena<const T> src;       // m_outputDistance on the old grid
    Arena<T> dst;             // m_inputDistance on the new grid
    double ratio_inv;         // h_new / h_old
    int gb;
    double delta_new;         // delta of the new grid
};
template <typename T>
void launch_resample(const ResampleArgs<T>& a, int grid, cudaStream_t s);
// IDLocal of present grains that do not exist, flat-resized onto their new box.
struct IdResizeArgs {
    int G;
    const int* present;
    const int* exists;
    const uint32_t* id_old;
    const int* idbox_old;
    const long long* idoff_old;
    uint32_t* id_new;
    const int* idbox_new;
    const long long* idoff_new;
};
void launch_id_resize(const IdResizeArgs& a, int grid, cudaStream_t s);

// ---- redistancing (gg_redist.cu) ----
template <typename T>
struct RedistArgs {
    int G;
    Geometry geo;
    const int* toff;          // n tiles per grain (n of the output box)
    const int* exists;
    Arena<T> in;
    Arena<T> out;
    int* err;
};
// Size classes of the redistancing: grains whose output box side n falls in class c
// (n <= redist_side(c), above the previous bound) run in launches whose block size,
// strides and shared memory fit that side, so that small boxes do not pay for the
// largest one; a CTA of class c runs redist_units(c) slices (or rows) of one grain side
// by side so that its lanes stay busy.
constexpr int kRedistClasses = 7;
__host__ __device__ constexpr int redist_side(int c) {
    return c <= 0 ? 24 : (c == 1 ? 32 : (c == 2 ? 40 : (c == 3 ? 48 : (c == 4 ? 56 : (c == 5 ? 64 : (1 << 30))))));
}
__host__ __device__ constexpr int redist_units(int c) {
    return c <= 0 ? 5 : (c == 1 ? 4 : (c == 2 ? 3 : (c == 3 ? 2 : 1)));
}
// class_toff: kRedistClasses tile tables of stride G + 2 (ceil(n / redist_units(c)) tiles
// per grain of class c),
// from launch_redist_classes; null: one launch over `a.toff` sized for `side`.
template <typename T>
void launch_redistance(const RedistArgs<T>& a, int grid, int side, const int* class_toff, cudaStream_t s);
void launch_redist_classes(int G, const int* toff_all, const int* box, int* class_toff, cudaStream_t s);
// Shared memory of one unit (one warp) at box side nmax; must fit one CTA.
size_t redist_smem_bytes(int nmax, bool fp64);

// ---- initial distance function (gg_init.cu) ----
template <typename T>
struct InitArgs {
    int G;
    Geometry geo;
    const int* toff;          // n tiles per present grain
    const int* present;
    Arena<T> dst;
    const uint32_t* labels;   // N^3 domain labels [z][y][x]
};
template <typename T>
void launch_init_sdf(const InitArgs<T>& a, int grid, cudaStream_t s);

// Voxel container of the network: N^3 grain IDs [z][y][x], 0 where no grain's SDF is >= 0.
template <typename T>
struct ContainerArgs {
    int G;
    Geometry geo;
    const int* toff;          // n tiles per existing grain of `src`
    Arena<const T> src;       // m_outputDistance of every grain
    uint32_t* labels;         // zeroed by the caller
};
template <typename T>
void launch_container(const ContainerArgs<T>& a, int grid, cudaStream_t s);

// out3 = {present grains, present and existing grains, largest side of `box` among the latter}
void launch_count(int G, const int* present, const int* exists, const int* box, int* out3, cudaStream_t s);

}  // namespace gg

// gg_api.cu -- host orchestration and the C ABI (include/gg_b200.h).
//
// This is the B200 replacement of grainhdl's per-timestep driver
// (grainhdl.cpp:821-943): it owns the device-resident box pool, sequences the
// batched stage kernels on one stream, and mirrors the reference's in/out buffer
// swaps with arena parities.  Host code only; the kernels live in the other .cu
// files.  Compiled without floating-point contraction so that the DFT twiddles
// and Gaussian tables match the oracle's bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gg_b200.h"
#include "gg_conv.cuh"
#include "gg_conv_tc.cuh"
#include "gg_kernels.cuh"

using namespace gg;

namespace {

constexpr double kPi = 3.14159265358979323846;  // ggLS.h:25
constexpr int kNbCap = 256;

struct Timer {
    cudaEvent_t e[6];
};

}  // namespace

struct gg_ctx {
    gg_params P{};
    std::string err;
    int G = 0, N = 0, gb = 0, M = 0;
    bool fp64 = true;
    size_t esz = 8;
    Geometry geo{};
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    int grid = 148 * 8;
    bool loaded = false;
    // per-grain device state
    int *d_present = nullptr, *d_exists = nullptr, *d_newbox = nullptr, *d_nnb = nullptr;
    double *d_volume = nullptr, *d_surface = nullptr;
    uint32_t* d_nb = nullptr;
    uint32_t *d_cmp = nullptr, *d_son = nullptr;
    unsigned long long* d_pt = nullptr;  // per-grain list position tables
    int pos_cap = 0;
    int *d_ncmp = nullptr, *d_nson = nullptr;
    // pool
    void* d_arena[2] = {nullptr, nullptr};
    int* d_box[2] = {nullptr, nullptr};
    long long* d_off[2] = {nullptr, nullptr};
    uint32_t* d_idarena[2] = {nullptr, nullptr};
    int* d_idbox[2] = {nullptr, nullptr};
    long long* d_idoff[2] = {nullptr, nullptr};
    double2* d_spec = nullptr;
    long long* d_spec_off = nullptr;
    long long pool_voxels = 0, spec_capacity = 0;
    // tiles
    int *d_toff_n = nullptr, *d_toff_slab = nullptr, *d_toff_one = nullptr, *d_toff_mc = nullptr, *d_toff_red = nullptr;
    int* d_toff_big = nullptr;  // mixed path: slices of the boxes above the tensor-core side
    WorkOrder work{};           // largest-first order of the per-grain kernels
    int* d_toff_rcls = nullptr; // redistancing size classes: kRedistClasses x (G + 2)
    TileBins lbins{};           // the list update's candidate cells
    int lbins_cells = 0;        // cells the count arrays hold
    // tables
    double2* d_tw = nullptr;
    long long* d_tw_off = nullptr;
    double* d_gtab = nullptr;
    long long* d_g_off = nullptr;
    float* d_circ = nullptr;          // FP32 circulant matrices (mixed path)
    long long* d_circ_off = nullptr;
    uint16_t* d_bmat = nullptr;       // the same, split FP16 hi/lo in the tensor-core operand layout
    long long* d_boff = nullptr;
    float* d_cscr = nullptr;          // mixed-path convolution scratch (out's layout); without the
                                      // correction the input arena serves, once read
    unsigned char* d_elscr = nullptr; // element build: per-CTA junction and pair scratch
    bool elements = false;            // interfacial elements built every step (correction or keep_elements)
    int elscr_ctas = 0;
    // convolution correction: orientations, stored energies, hull capture, elements
    bool correction = false;
    double4* d_quat = nullptr;
    double* d_see = nullptr;
    HullCapture hull{};
    HullElements el{};
    // scalars
    int* d_err = nullptr;
    long long* d_total_vox = nullptr;
    int* d_count3 = nullptr;
    int* h_count3 = nullptr;  // pinned
    long long* h_total_vox = nullptr;
    // comparison: grains per domain tile
    TileBins bins{};
    int* h_maxcount = nullptr;  // pinned
    // host mirror
    int p = 0;        // SDF arena holding m_inputDistance
    int q = 0;        // ID arena holding m_IDLocal
    int loop = 0;
    int grain_count = 0, live = 0;
    int side_max = 0;      // largest box side of the current layout
    int side_limit = 0;    // largest side the shared-memory kernels accept
    int list_cap = 4096, slab = 8;
    long long launches = 0;  // kernels launched by this context
    // grid coarsening (grainhdl::gridCoarsement): ngrains at the last coarsening, and
    // NumberOfPointsPerGrain
    int coarse_ref = 0, points_per_grain = 0;
    // launch configuration: CTAs per SM of each stage's grid-stride kernels (convolution
    // with the correction, lists, comparison, level set, redistancing), chosen by the
    // autotuner when it is on
    int mult[5] = {8, 8, 4, 8, 8};
    int tune_next = -1;         // candidate the next tuning step runs, -1: not tuning
    double tune_cost[5][8] = {};
    // element counts of the N-dependent tables' device buffers (reused when they fit)
    size_t tw_cap = 0, gt_cap = 0, circ_cap = 0, bmat_cap = 0;
    size_t tw_off_cap = 0, g_off_cap = 0, c_off_cap = 0, boff_cap = 0;
    cudaEvent_t ev[8] = {};  // stage boundaries (0-5), the comparison kernel (6, 7)
};

namespace {

// The autotuner's candidates: CTAs per SM for the grid-stride stage kernels.  Every stage
// kernel walks its tiles grid-stride and computes each grain's results inside one CTA, so
// the grid changes only the speed, never the results.
constexpr int kTuneCand[] = {2, 4, 8, 16, 32};
constexpr int kNumTune = 5;
enum Stage { ST_CONV = 0, ST_LISTS, ST_COMPARE, ST_LEVELSET, ST_REDIST };

int stage_grid(const gg_ctx* c, int s);

int fail(gg_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ctx, GG_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                   \
    } while (0)

template <typename X>
cudaError_t dalloc(X** p, size_t count) {
    return cudaMalloc((void**)p, sizeof(X) * (count ? count : 1));
}

// Gaussian multiplier of box.cpp:760-761 for every S = i2^2 + j2^2 + k2^2 of side n.
void gaussian_table(int n, int N, double time_step, std::vector<double>& out) {
    const double dt = time_step / double(N * N);  // grainhdl.cpp:1431
    const double nsq = N * N;
    const double local_nsq = n * n;
    const int h = n / 2;
    const int smax = 3 * h * h;
    for (int S = 0; S <= smax; S++) {
        const double G = std::exp(-std::sqrt(2 / kPi) * S * 4.0 * dt * nsq / local_nsq * kPi * kPi) / (local_nsq * n);
        out.push_back(G);
    }
}

// myQuaternion::euler2Quaternion (myQuaternion.cpp:168-191), Bunge ZXZ, host libm.
double4 euler_to_quat(double p1, double t, double p2) {
    const double co1 = std::cos(t / 2), s1 = std::sin(t / 2);
    return make_double4(co1 * std::cos((p1 + p2) / 2), s1 * std::cos((p1 - p2) / 2), s1 * std::sin((p1 - p2) / 2),
                        co1 * std::sin((p1 + p2) / 2));
}

HullPhysics physics(gg_ctx* ctx);

// Twiddles of the specified DFT: (cos, sin)(2 pi j / n), angle (6.283185307179586 * j) / n.
void twiddle_table(int n, std::vector<double2>& out) {
    for (int j = 0; j < n; j++) {
        const double a = 6.283185307179586476925286766559 * (double)j / (double)n;
        out.push_back(make_double2(std::cos(a), std::sin(a)));
    }
}

HullPhysics physics(gg_ctx* ctx) {
    HullPhysics h{};
    h.quat = ctx->d_quat;
    h.see = ctx->d_see;
    h.unique_gb = ctx->P.unique_gb_energies;
    h.mobility_model = ctx->P.mobility_model;
    h.use_see = ctx->P.use_stored_energy;
    h.tl_drag = ctx->P.triple_line_drag;
    h.ds = 1 / (double)ctx->N;                        // grainhdl.h:181-183
    h.dt = ctx->P.time_step / double(ctx->N * ctx->N);  // grainhdl.cpp:1431
    return h;
}

// Copies a host table into a device buffer, reallocating it only when it has grown.
template <typename X>
int put_table(gg_ctx* ctx, X** d, size_t* cap, const std::vector<X>& h) {
    if (h.size() > *cap || !*d) {
        if (*d) CK(cudaFree(*d));
        *d = nullptr;
        CK(dalloc(d, h.size()));
        *cap = h.size() ? h.size() : 1;
    }
    if (!h.empty()) CK(cudaMemcpy(*d, h.data(), sizeof(X) * h.size(), cudaMemcpyHostToDevice));
    return GG_OK;
}

// The tables of the current grid (N, M): DFT twiddles and the Gaussian multiplier per side,
// and on the mixed path the circulant matrices.  Run at set-up and after a grid coarsening
// (the Gaussian's dt N^2 is computed from the new N, grainhdl.cpp:1419-1442).
int upload_tables(gg_ctx* ctx) {
    const int M = ctx->M;
    std::vector<double2> tw;
    std::vector<long long> tw_off(M + 2, 0);
    std::vector<double> gt;
    std::vector<long long> g_off(M + 2, 0);
    for (int n = 1; n <= M; n++) {
        tw_off[n] = (long long)tw.size();
        twiddle_table(n, tw);
        g_off[n] = (long long)gt.size();
        gaussian_table(n, ctx->N, ctx->P.time_step, gt);
    }
    int rc = put_table(ctx, &ctx->d_tw, &ctx->tw_cap, tw);
    if (!rc) rc = put_table(ctx, &ctx->d_tw_off, &ctx->tw_off_cap, tw_off);
    if (!rc) rc = put_table(ctx, &ctx->d_gtab, &ctx->gt_cap, gt);
    if (!rc) rc = put_table(ctx, &ctx->d_g_off, &ctx->g_off_cap, g_off);
    if (rc) return rc;
    if (!ctx->fp64) {
        std::vector<float> circ;
        std::vector<long long> c_off(M + 2, 0);
        for (int n = 1; n <= M; n++) {
            c_off[n] = (long long)circ.size();
            circulant_matrix(n, ctx->N, ctx->P.time_step, circ);
        }
        rc = put_table(ctx, &ctx->d_circ, &ctx->circ_cap, circ);
        if (!rc) rc = put_table(ctx, &ctx->d_circ_off, &ctx->c_off_cap, c_off);
        std::vector<uint16_t> bmat;
        std::vector<long long> boff;
        umma_tables(ctx->N, ctx->P.time_step, std::min(M, kUmmaMaxSide), bmat, boff);
        if (!rc) rc = put_table(ctx, &ctx->d_bmat, &ctx->bmat_cap, bmat);
        if (!rc) rc = put_table(ctx, &ctx->d_boff, &ctx->boff_cap, boff);
        if (rc) return rc;
    }
    return GG_OK;
}

int check_err(gg_ctx* ctx, const char* where) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e & ERR_POOL) return fail(ctx, GG_ERR_POOL_EXHAUSTED, "%s: box pool or scratch capacity exceeded", where);
    if (e & (ERR_LIST | ERR_HASH)) return fail(ctx, GG_ERR_LIST_OVERFLOW, "%s: comparison list capacity exceeded", where);
    if (e & ERR_NEIGHBORS) return fail(ctx, GG_ERR_LIST_OVERFLOW, "%s: hull neighbour capacity exceeded", where);
    if (e & ERR_BOX) return fail(ctx, GG_ERR_UNSUPPORTED, "%s: a box left the grid or exceeded the supported side", where);
    // a capacity overflow comes before the bounds checks it may trip further down the step
    if (e & ERR_HULL) {
        int d = 0;
        if (ctx->hull.diag) CK(cudaMemcpy(&d, ctx->hull.diag, sizeof(int), cudaMemcpyDeviceToHost));
        const char* what = (d & (HULL_TRIANGLES | HULL_RECORDS)) ? "triangles or active cubes of a hull beyond hull_capacity"
                           : (d & HULL_LISTS)        ? "more than 256 distinct neighbour lists on one hull"
                           : (d & HULL_JUNCTION_IDS) ? "a merged junction with more IDs than the element build holds"
                           : (d & HULL_JUNCTIONS)    ? "more than 256 junctions on one hull"
                           : (d & HULL_JOBS)         ? "more misorientations on one hull than the element build holds"
                           : (d & HULL_INDEX)        ? "a hull's neighbour -> elements index beyond its capacity"
                           : (d & HULL_TABLE)        ? "a hull's element, ID or segment table beyond its capacity"
                                                     : "hull or interfacial-element capacity exceeded";
        return fail(ctx, GG_ERR_POOL_EXHAUSTED, "%s: %s (diag %d)", where, what, d);
    }
    if (e & ERR_TIMEOUT) return fail(ctx, GG_ERR_CUDA, "%s: a bounded tensor-core pipeline wait timed out", where);
    if (e & ERR_BOUNDS) return fail(ctx, GG_ERR_CUDA, "%s: a kernel bounds check failed (access skipped)", where);
    return GG_OK;
}

template <typename T>
Arena<T> arena(gg_ctx* c, int a) {
    return Arena<T>{reinterpret_cast<T*>(c->d_arena[a]), c->d_box[a], c->d_off[a]};
}

int plan(gg_ctx* ctx, const int* box, int only_existing, long long* off, long long* spec_off, int* toff_n,
         int* toff_slab, int* toff_one, long long* total_voxels = nullptr) {
    PlanArgs a{};
    a.G = ctx->G;
    a.present = ctx->d_present;
    a.exists = ctx->d_exists;
    a.box = box;
    a.only_existing = only_existing;
    a.off = off;
    a.capacity = ctx->pool_voxels;
    a.spec_off = spec_off;
    a.spec_capacity = ctx->spec_capacity;
    a.toff_n = toff_n;
    a.toff_slab = toff_slab;
    a.slab = ctx->slab;
    a.row_tile = ctx->fp64 ? 0 : kUmmaRows;
    // mixed path: boxes up to the tensor-core kernel's side in row tiles, larger ones in slices
    a.class_side = ctx->fp64 ? 0 : kUmmaMaxSide;
    a.toff_big = (!ctx->fp64 && toff_slab) ? ctx->d_toff_big : nullptr;
    a.toff_one = toff_one;
    a.total_voxels = total_voxels;
    a.err = ctx->d_err;
    launch_plan(a, ctx->stream);
    ctx->launches += 1;
    return GG_OK;
}

int read_counts(gg_ctx* ctx, const int* box) {
    launch_count(ctx->G, ctx->d_present, ctx->d_exists, box, ctx->d_count3, ctx->stream);
    ctx->launches += 1;
    CK(cudaMemcpyAsync(ctx->h_count3, ctx->d_count3, 3 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_total_vox, ctx->d_total_vox, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->grain_count = ctx->h_count3[0];
    ctx->live = ctx->h_count3[1];
    return GG_OK;
}

int side_check(gg_ctx* ctx, int side) {
    if (side > ctx->side_limit)
        return fail(ctx, GG_ERR_UNSUPPORTED, "box side %d exceeds the supported maximum %d", side, ctx->side_limit);
    return GG_OK;
}

template <typename T>
int redistance(gg_ctx* ctx, int in_a, int out_a, const int* toff, int side, bool classes = false) {
    RedistArgs<T> r{};
    r.G = ctx->G;
    r.geo = ctx->geo;
    r.toff = toff;
    r.exists = ctx->d_exists;
    r.in = arena<T>(ctx, in_a);
    r.out = arena<T>(ctx, out_a);
    r.err = ctx->d_err;
    if (classes) {  // per size class of the output boxes (their tiles from toff)
        launch_redist_classes(ctx->G, toff, ctx->d_box[out_a], ctx->d_toff_rcls, ctx->stream);
        launch_redistance<T>(r, stage_grid(ctx, ST_REDIST), side, ctx->d_toff_rcls, ctx->stream);
        int nc = 0;
        for (int c = 0; c < kRedistClasses && (c == 0 || redist_side(c - 1) < side); c++) nc++;
        ctx->launches += 1 + 2 * nc;
    } else {
        launch_redistance<T>(r, stage_grid(ctx, ST_REDIST), side, nullptr, ctx->stream);
        ctx->launches += 2;
    }
    CK(cudaGetLastError());
    return GG_OK;
}

template <typename T>
int load_state_t(gg_ctx* ctx, const uint32_t* labels) {
    const int G = ctx->G;
    // initial layout in arena 0, mirrored to arena 1 and the first IDLocal arena
    plan(ctx, ctx->d_box[0], 1, ctx->d_off[0], nullptr, ctx->d_toff_n, nullptr, nullptr);
    launch_copy_layout(G, ctx->d_present, ctx->d_box[0], ctx->d_off[0], ctx->d_box[1], ctx->d_off[1], ctx->stream);
    ctx->launches += 1;
    launch_copy_layout(G, ctx->d_present, ctx->d_box[0], ctx->d_off[0], ctx->d_idbox[0], ctx->d_idoff[0], ctx->stream);
    ctx->launches += 1;
    CK(cudaMemsetAsync(ctx->d_idarena[0], 0, sizeof(uint32_t) * ctx->pool_voxels, ctx->stream));
    int rc = check_err(ctx, "gg_load_state");
    if (rc) return rc;
    uint32_t* d_labels = nullptr;
    const size_t nl = (size_t)ctx->N * ctx->N * ctx->N;
    CK(dalloc(&d_labels, nl));
    CK(cudaMemcpyAsync(d_labels, labels, nl * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    InitArgs<T> ia{};
    ia.G = G;
    ia.geo = ctx->geo;
    ia.toff = ctx->d_toff_n;
    ia.present = ctx->d_present;
    ia.dst = arena<T>(ctx, 0);
    ia.labels = d_labels;
    launch_init_sdf<T>(ia, ctx->grid, ctx->stream);
    CK(cudaGetLastError());
    // calculateDistanceFunction ends with executeRedistancing (box.cpp:396): arena 0 -> arena 1
    rc = redistance<T>(ctx, 0, 1, ctx->d_toff_n, ctx->side_max);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(d_labels));
    ctx->p = 0;   // m_inputDistance = +-h field, m_outputDistance = initial SDF
    ctx->q = 0;
    return check_err(ctx, "gg_load_state");
}

// The convolution correction (box.cpp:426-535) on the convolved boxes of arena p ^ 1,
// from the input in arena p and the IDLocal of the last comparison (arena q).
template <typename T>
int correct_convolution(gg_ctx* ctx) {
    if (!ctx->correction || ctx->loop == 0) return GG_OK;
    const int p = ctx->p;
    CorrectionArgs<T> c{};
    c.G = ctx->G;
    c.geo = ctx->geo;
    c.toff = ctx->d_toff_one;
    c.present = ctx->d_present;
    c.box = ctx->d_box[p];
    c.in = reinterpret_cast<const T*>(ctx->d_arena[p]);
    c.in_off = ctx->d_off[p];
    c.out = reinterpret_cast<T*>(ctx->d_arena[p ^ 1]);
    c.out_off = ctx->d_off[p ^ 1];
    c.id_old = ctx->d_idarena[ctx->q];
    c.idbox_old = ctx->d_idbox[ctx->q];
    c.idoff_old = ctx->d_idoff[ctx->q];
    c.el = ctx->el;
    c.ph = physics(ctx);
    c.err = ctx->d_err;
    launch_work_order(ctx->work, ctx->G, ctx->d_toff_one, ctx->d_box[p], correction_item_voxels(), ctx->stream);
    c.order = ctx->work.order;
    c.item_off = ctx->work.item_off;
    c.queue = ctx->work.queue;
    launch_correction<T>(c, stage_grid(ctx, ST_CONV), ctx->stream);
    ctx->launches += 5;
    CK(cudaGetLastError());
    return GG_OK;
}

template <typename T>
int coarsen_t(gg_ctx* ctx, int new_size);
int coarsening_size(const gg_ctx* ctx);

template <typename T>
int stage_convolution_t(gg_ctx* ctx) {
    // gridCoarsement (grainhdl.cpp:1446-1498): re-grid, or switchDistancebuffer (:1496)
    if (const int new_size = coarsening_size(ctx)) {
        const int rc = coarsen_t<T>(ctx, new_size);
        if (rc) return rc;
    }
    ctx->p ^= 1;
    const int p = ctx->p;
    plan(ctx, ctx->d_box[p], 1, nullptr, sizeof(T) == 8 ? ctx->d_spec_off : nullptr, ctx->d_toff_n,
         ctx->d_toff_slab, ctx->d_toff_one, ctx->d_total_vox);
    // IDLocal follows the output box (resizeIDLocalToDistanceBuffer, box.cpp:426)
    launch_copy_layout(ctx->G, ctx->d_present, ctx->d_box[p], ctx->d_off[p], ctx->d_idbox[ctx->q ^ 1],
                       ctx->d_idoff[ctx->q ^ 1], ctx->stream);
    ctx->launches += 1;
    if (sizeof(T) == 8) {
        ConvArgs a{};
        a.G = ctx->G;
        a.toff = ctx->d_toff_n;
        a.in = reinterpret_cast<const double*>(ctx->d_arena[p]);
        a.in_box = ctx->d_box[p];
        a.in_off = ctx->d_off[p];
        a.out = reinterpret_cast<double*>(ctx->d_arena[p ^ 1]);
        a.out_off = ctx->d_off[p ^ 1];
        a.spec = ctx->d_spec;
        a.spec_off = ctx->d_spec_off;
        a.tw = ctx->d_tw;
        a.tw_off = ctx->d_tw_off;
        a.gtab = ctx->d_gtab;
        a.g_off = ctx->d_g_off;
        launch_conv_f64(a, stage_grid(ctx, ST_CONV), conv_f64_smem_bytes(ctx->side_max), ctx->stream);
        ctx->launches += 3;
    } else {
        // two size classes in one step: sides up to kUmmaMaxSide on the tensor cores, larger
        // boxes (when any) on the FP32 SIMT kernels; each launch walks only its class's tiles
        const int small_side = std::min(ctx->side_max, kUmmaMaxSide);
        if (!umma_supported(small_side)) return fail(ctx, GG_ERR_UNSUPPORTED, "tensor-core convolution unavailable");
        // The middle pass needs a buffer in out's layout.  Without the correction nothing
        // reads the input after the convolution (the comparison overwrites its arena), so
        // the input arena serves, and the large boxes, which read the input, go first.
        float* scratch = ctx->d_cscr;
        if (!scratch) {
            if (ctx->correction) return fail(ctx, GG_ERR_INVALID, "convolution scratch missing");
            scratch = reinterpret_cast<float*>(ctx->d_arena[p]);
        }
        const bool big = ctx->side_max > kUmmaMaxSide;
        auto large_boxes = [&]() {
            ConvTCArgs a{};
            a.G = ctx->G;
            a.toff = ctx->d_toff_big;
            a.in = reinterpret_cast<const float*>(ctx->d_arena[p]);
            a.box = ctx->d_box[p];
            a.in_off = ctx->d_off[p];
            a.out = reinterpret_cast<float*>(ctx->d_arena[p ^ 1]);
            a.out_off = ctx->d_off[p ^ 1];
            a.circ = ctx->d_circ;
            a.circ_off = ctx->d_circ_off;
            a.err = ctx->d_err;
            launch_conv_tc(a, ctx->num_sms, ctx->side_max, ctx->stream);
            ctx->launches += 2;
        };
        if (big) large_boxes();
        UmmaConvArgs u{};
        u.G = ctx->G;
        u.toff = ctx->d_toff_slab;
        u.box = ctx->d_box[p];
        u.in = reinterpret_cast<const float*>(ctx->d_arena[p]);
        u.in_off = ctx->d_off[p];
        u.out = reinterpret_cast<float*>(ctx->d_arena[p ^ 1]);
        u.out_off = ctx->d_off[p ^ 1];
        u.scratch = scratch;
        u.bmat = ctx->d_bmat;
        u.boff = ctx->d_boff;
        u.err = ctx->d_err;
        launch_conv_umma(u, ctx->num_sms, small_side, ctx->stream);
        ctx->launches += 3;
        CK(cudaGetLastError());
    }
    CK(cudaGetLastError());
    return correct_convolution<T>(ctx);
}

// Make room for the list update's cell entries of the current layout.
int ensure_list_bins(gg_ctx* ctx) {
    const int n = ctx->M / kListCell + 1;
    if ((long long)n * n * n > ctx->lbins_cells) return fail(ctx, GG_ERR_INVALID, "list cells exceed their arrays");
    ctx->lbins.ntx = ctx->lbins.nty = ctx->lbins.ntz = n;
    const long long need = list_bin_capacity(ctx->G, ctx->side_max);
    if (need <= ctx->lbins.capacity) return GG_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->lbins.entries) CK(cudaFree(ctx->lbins.entries));
    ctx->lbins.capacity = need + need / 4;
    CK(dalloc(&ctx->lbins.entries, ctx->lbins.capacity));
    return GG_OK;
}

int stage_update_lists_t(gg_ctx* ctx) {
    ctx->p ^= 1;  // switchDistancebuffer, grainhdl.cpp:852
    int rc = ensure_list_bins(ctx);
    if (rc) return rc;
    // position tables of the previous lists (every present grain: the lists of grains
    // whose hull vanished last step are walked too), and the candidate cells
    PosTableArgs pt{};
    pt.G = ctx->G;
    pt.present = ctx->d_present;
    pt.cmp = ctx->d_son;
    pt.n_cmp = ctx->d_nson;
    pt.list_cap = ctx->list_cap;
    pt.table = ctx->d_pt;
    pt.pos_cap = ctx->pos_cap;
    pt.err = ctx->d_err;
    launch_pos_tables(pt, ctx->grid, ctx->stream);
    launch_list_bins(ctx->lbins, ctx->G, ctx->d_exists, ctx->d_box[ctx->p], ctx->d_err, ctx->stream);
    ctx->launches += 4;
    ListArgs a{};
    a.G = ctx->G;
    a.toff = ctx->d_toff_one;
    a.exists = ctx->d_exists;
    a.box = ctx->d_box[ctx->p];
    a.son = ctx->d_son;
    a.n_son = ctx->d_nson;
    a.cmp = ctx->d_cmp;
    a.n_cmp = ctx->d_ncmp;
    a.list_cap = ctx->list_cap;
    a.cells = ctx->lbins;
    a.pos = ctx->d_pt;
    a.pos_cap = ctx->pos_cap;
    a.err = ctx->d_err;
    launch_update_lists(a, stage_grid(ctx, ST_LISTS), ctx->stream);
    // m_secondOrderNeighbours = m_comparisonList (box.cpp:895), once every list is rebuilt
    ListCopyArgs sl{};
    sl.G = ctx->G;
    sl.toff = ctx->d_toff_one;
    sl.cmp = ctx->d_cmp;
    sl.n_cmp = ctx->d_ncmp;
    sl.son = ctx->d_son;
    sl.n_son = ctx->d_nson;
    sl.list_cap = ctx->list_cap;
    launch_copy_lists(sl, stage_grid(ctx, ST_LISTS), ctx->stream);
    ctx->launches += 2;
    CK(cudaGetLastError());
    return GG_OK;
}

// Make room for the tile-to-grain entries of the current layout.
int ensure_bins(gg_ctx* ctx) {
    const long long need = bin_capacity(ctx->G, ctx->side_max);
    if (need <= ctx->bins.capacity) return GG_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->bins.entries) CK(cudaFree(ctx->bins.entries));
    ctx->bins.capacity = need + need / 4;
    CK(dalloc(&ctx->bins.entries, ctx->bins.capacity));
    return GG_OK;
}

// executeComparison (+ executeSetComparison when set_comparison) of every grain: the
// neighbours' fields in arena `in_a`, the result into arena `out_a`, IDLocal from arena
// q into q ^ 1.  After a grid coarsening (set_comparison 0) every present grain's field
// takes part as a neighbour: comparison lists may still name a grain whose hull vanished
// in the last step, and the reference has re-gridded it too.
template <typename T>
int compare_t(gg_ctx* ctx, int in_a, int out_a, int set_comparison) {
    const int q = ctx->q;
    int rc = ensure_bins(ctx);
    if (rc) return rc;
    if (set_comparison)
        launch_newbox_init(ctx->G, ctx->d_present, ctx->d_exists, ctx->d_box[out_a], ctx->d_newbox, ctx->stream);
    PosTableArgs pt{};
    pt.G = ctx->G;
    pt.toff = ctx->d_toff_one;
    pt.cmp = ctx->d_cmp;
    pt.n_cmp = ctx->d_ncmp;
    pt.list_cap = ctx->list_cap;
    pt.table = ctx->d_pt;
    pt.pos_cap = ctx->pos_cap;
    pt.err = ctx->d_err;
    launch_pos_tables(pt, ctx->grid, ctx->stream);
    ctx->launches += 1;
    launch_bin(ctx->bins, ctx->G, set_comparison ? ctx->d_exists : ctx->d_present, ctx->d_box[in_a], ctx->d_err,
               ctx->stream);
    ctx->launches += 5;
    CK(cudaMemcpyAsync(ctx->h_maxcount, ctx->bins.max_count, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    rc = check_err(ctx, "comparison binning");  // nothing may read past the tile entries
    if (rc) return rc;
    const int mcap = std::max(1, *ctx->h_maxcount);
    if (mcap > 254 || compare_smem_bytes(mcap, sizeof(T) == 8) > 227 * 1024)
        return fail(ctx, GG_ERR_UNSUPPORTED, "%d grain boxes reach one comparison tile (at most 254 supported)", mcap);
    CompareArgs<T> a{};
    a.geo = ctx->geo;
    a.bins = ctx->bins;
    a.mcap = mcap;
    a.in = arena<T>(ctx, in_a);
    a.out = arena<T>(ctx, out_a);
    a.id_old = ctx->d_idarena[q];
    a.idbox_old = ctx->d_idbox[q];
    a.idoff_old = ctx->d_idoff[q];
    a.id_new = ctx->d_idarena[q ^ 1];
    a.idoff_new = ctx->d_idoff[q ^ 1];
    a.cmp = ctx->d_cmp;
    a.n_cmp = ctx->d_ncmp;
    a.list_cap = ctx->list_cap;
    a.pos_table = ctx->d_pt;
    a.pos_cap = ctx->pos_cap;
    a.newbox = ctx->d_newbox;
    a.err = ctx->d_err;
    a.set_comparison = set_comparison;
    a.exists = ctx->d_exists;
    if (set_comparison) cudaEventRecord(ctx->ev[6], ctx->stream);
    launch_compare<T>(a, stage_grid(ctx, ST_COMPARE), ctx->stream);
    if (set_comparison) cudaEventRecord(ctx->ev[7], ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    ctx->q ^= 1;
    return GG_OK;
}

template <typename T>
int stage_comparison_t(gg_ctx* ctx) {
    const int rc = compare_t<T>(ctx, ctx->p, ctx->p ^ 1, 1);
    if (rc) return rc;
    ctx->p ^= 1;  // switchDistancebuffer, grainhdl.cpp:865
    return GG_OK;
}

// extractContour of every present grain on the field in arena p (the new box of the
// grains that exist goes to arena p ^ 1), then computeSurfaceElements.  regrid: the
// extractContour that follows a grid coarsening (see MCArgs).
template <typename T>
int level_set_t(gg_ctx* ctx, int p, int regrid) {
    plan(ctx, ctx->d_box[p], 0, nullptr, nullptr, nullptr, nullptr, ctx->d_toff_mc);
    MCArgs<T> a{};
    a.G = ctx->G;
    a.geo = ctx->geo;
    a.toff = ctx->d_toff_mc;
    a.present = ctx->d_present;
    a.exists = ctx->d_exists;
    a.in = arena<T>(ctx, p);
    a.idl = ctx->d_idarena[ctx->q];
    a.idoff = ctx->d_idoff[ctx->q];
    a.newbox = ctx->d_newbox;
    a.out_box = ctx->d_box[p ^ 1];
    a.volume = ctx->d_volume;
    a.surface = ctx->d_surface;
    a.nb = ctx->d_nb;
    a.n_nb = ctx->d_nnb;
    a.nb_cap = kNbCap;
    a.err = ctx->d_err;
    a.regrid = regrid;
    if (ctx->elements) a.hull = ctx->hull;
    launch_work_order(ctx->work, ctx->G, ctx->d_toff_mc, ctx->d_box[p], 0, ctx->stream);
    a.order = ctx->work.order;
    a.item_off = ctx->work.item_off;
    a.queue = ctx->work.queue;
    launch_mc<T>(a, stage_grid(ctx, ST_LEVELSET), ctx->side_max, ctx->stream);
    ctx->launches += 5;
    CK(cudaGetLastError());
    if (ctx->elements) {  // computeSurfaceElements, box.cpp:1175-1180
        ElementArgs e{};
        e.G = ctx->G;
        e.toff = ctx->d_toff_mc;
        e.exists = ctx->d_exists;
        e.cap = ctx->hull;
        e.el = ctx->el;
        e.ph = physics(ctx);
        e.scratch = ctx->d_elscr;
        e.scratch_ctas = ctx->elscr_ctas;
        e.order = ctx->work.order;
        e.item_off = ctx->work.item_off;
        e.queue = ctx->work.queue + 1;
        e.err = ctx->d_err;
        launch_elements(e, ctx->elscr_ctas, ctx->stream);
        ctx->launches += 1;
        CK(cudaGetLastError());
    }
    return GG_OK;
}

template <typename T>
int stage_level_set_t(gg_ctx* ctx) {
    return level_set_t<T>(ctx, ctx->p, 0);
}

// grainhdl::gridCoarsement (grainhdl.cpp:1446-1498) when it re-grids: the geometry and
// time variables of the new size (updateGridAndTimeVariables, grainhdl.cpp:1419-1443) and
// their tables, LSbox::resizeGrid of every present grain (box.cpp:2595-2694), then
// recalculateIDLocal (box.cpp:2697-2700) and extractContour of every present grain.
// The last redistancing's result (arena p ^ 1, the reference's m_outputDistance) is
// re-sampled into arena p, which the convolution then reads without the usual
// switchDistancebuffer: p is left pointing at the other arena so that the convolution
// stage's switch lands on the re-sampled field.
template <typename T>
int coarsen_t(gg_ctx* ctx, int new_size) {
    const int src = ctx->p ^ 1, dst = ctx->p;
    const double h_old = ctx->geo.h;
    ctx->N = new_size;
    ctx->M = ctx->N + 2 * ctx->gb;
    ctx->geo = Geometry{ctx->N, ctx->gb, ctx->M, 1 / (double)ctx->N, ctx->gb / double(ctx->N), ctx->P.time_step};
    int rc = upload_tables(ctx);
    if (rc) return rc;
    ctx->bins.ntx = (ctx->M + kTX - 1) / kTX;  // fewer tiles than the arrays hold
    ctx->bins.nty = (ctx->M + kTY - 1) / kTY;
    ctx->bins.ntz = (ctx->M + kTZ - 1) / kTZ;
    RegridBoxArgs rb{};
    rb.G = ctx->G;
    rb.present = ctx->d_present;
    rb.old_box = ctx->d_box[src];
    rb.scaled = ctx->d_newbox;
    rb.new_box = ctx->d_box[dst];
    rb.ratio = h_old / ctx->geo.h;  // h / hn of resizeGrid
    rb.gb = ctx->gb;
    rb.M_new = ctx->M;
    rb.err = ctx->d_err;
    launch_regrid_boxes(rb, ctx->stream);
    ctx->launches += 1;
    plan(ctx, ctx->d_box[dst], 0, ctx->d_off[dst], nullptr, ctx->d_toff_n, nullptr, nullptr);
    rc = check_err(ctx, "grid coarsening");
    if (rc) return rc;
    ResampleArgs<T> rs{};
    rs.G = ctx->G;
    rs.toff = ctx->d_toff_n;
    rs.src = Arena<const T>{reinterpret_cast<const T*>(ctx->d_arena[src]), ctx->d_box[src], ctx->d_off[src]};
    rs.dst = arena<T>(ctx, dst);
    rs.ratio_inv = ctx->geo.h / h_old;  // hn / h
    rs.gb = ctx->gb;
    rs.delta_new = ctx->geo.delta;
    launch_resample<T>(rs, ctx->grid, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    // m_outputDistance->resize(the input's box); IDLocal follows it (resizeIDLocalToDistanceBuffer)
    launch_copy_layout(ctx->G, ctx->d_present, ctx->d_box[dst], ctx->d_off[dst], ctx->d_box[src], ctx->d_off[src],
                       ctx->stream);
    launch_copy_layout(ctx->G, ctx->d_present, ctx->d_box[dst], ctx->d_off[dst], ctx->d_idbox[ctx->q ^ 1],
                       ctx->d_idoff[ctx->q ^ 1], ctx->stream);
    IdResizeArgs ir{};
    ir.G = ctx->G;
    ir.present = ctx->d_present;
    ir.exists = ctx->d_exists;
    ir.id_old = ctx->d_idarena[ctx->q];
    ir.idbox_old = ctx->d_idbox[ctx->q];
    ir.idoff_old = ctx->d_idoff[ctx->q];
    ir.id_new = ctx->d_idarena[ctx->q ^ 1];
    ir.idbox_new = ctx->d_idbox[ctx->q ^ 1];
    ir.idoff_new = ctx->d_idoff[ctx->q ^ 1];
    launch_id_resize(ir, ctx->grid, ctx->stream);
    ctx->launches += 3;
    CK(cudaGetLastError());
    ctx->coarse_ref = ctx->grain_count;  // ngrains = currentNrGrains
    rc = compare_t<T>(ctx, dst, src, 0);
    if (rc) return rc;
    rc = level_set_t<T>(ctx, dst, 1);
    if (rc) return rc;
    ctx->p = src;
    return check_err(ctx, "grid coarsening");
}

// The size gridCoarsement would re-grid to now, or 0 when it keeps the grid
// (grainhdl.cpp:1447-1451).
int coarsening_size(const gg_ctx* ctx) {
    if (!ctx->P.grid_coarsening || ctx->loop == 0) return 0;
    const int cur = ctx->grain_count;  // currentNrGrains: countGrains of the last loop
    const int new_size = (int)(std::pow((double)cur, 1 / 3.0) * std::pow(kPi * 4 / 3, 1. / 3) / 2 *
                               ctx->points_per_grain);
    const double gradient = ctx->P.coarsening_gradient > 0 ? ctx->P.coarsening_gradient : 0.95;
    if ((double)cur / (double)ctx->coarse_ref < gradient && new_size < ctx->N) return new_size;
    return 0;
}

template <typename T>
int stage_redistancing_t(gg_ctx* ctx) {
    const int p = ctx->p;
    // new packing of the resized output boxes
    plan(ctx, ctx->d_box[p ^ 1], 1, ctx->d_off[p ^ 1], nullptr, ctx->d_toff_red, nullptr, nullptr);
    int rc = read_counts(ctx, ctx->d_box[p ^ 1]);
    if (rc) return rc;
    const int side_new = ctx->h_count3[2];
    rc = side_check(ctx, side_new);
    if (rc) return rc;
    rc = check_err(ctx, "redistancing plan");
    if (rc) return rc;
    rc = redistance<T>(ctx, p, p ^ 1, ctx->d_toff_red, std::max(side_new, ctx->side_max), true);
    if (rc) return rc;
    // in.resize(out dims), box.cpp:2581-2584
    launch_copy_layout(ctx->G, ctx->d_present, ctx->d_box[p ^ 1], ctx->d_off[p ^ 1], ctx->d_box[p], ctx->d_off[p],
                       ctx->stream);
    ctx->launches += 1;
    ctx->side_max = side_new;
    return GG_OK;
}

template <typename T>
int step_t(gg_ctx* ctx, gg_step_stats* st) {
    const long long launches0 = ctx->launches;
    // the autotuner: loops 1 .. kNumTune (loop 0 has no correction) each run one candidate
    const bool tuning = ctx->tune_next >= 0 && ctx->loop >= 1;
    if (tuning)
        for (int s = 0; s < 5; s++) ctx->mult[s] = kTuneCand[ctx->tune_next];
    cudaEventRecord(ctx->ev[0], ctx->stream);
    int rc = stage_convolution_t<T>(ctx);
    if (rc) return rc;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    if ((rc = stage_update_lists_t(ctx))) return rc;
    cudaEventRecord(ctx->ev[2], ctx->stream);
    if ((rc = stage_comparison_t<T>(ctx))) return rc;
    cudaEventRecord(ctx->ev[3], ctx->stream);
    if ((rc = stage_level_set_t<T>(ctx))) return rc;
    cudaEventRecord(ctx->ev[4], ctx->stream);
    if ((rc = stage_redistancing_t<T>(ctx))) return rc;
    cudaEventRecord(ctx->ev[5], ctx->stream);
    CK(cudaEventSynchronize(ctx->ev[5]));
    rc = check_err(ctx, "gg_step");
    if (rc) return rc;
    if (tuning) {  // device time per voxel-update of each stage under this candidate
        const double vox = (double)std::max(1LL, *ctx->h_total_vox);
        for (int s = 0; s < 5; s++) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->ev[s], ctx->ev[s + 1]);
            ctx->tune_cost[s][ctx->tune_next] = ms / vox;
        }
        if (++ctx->tune_next == kNumTune) {
            for (int s = 0; s < 5; s++) {
                int best = 0;
                for (int c = 1; c < kNumTune; c++)
                    if (ctx->tune_cost[s][c] < ctx->tune_cost[s][best]) best = c;
                ctx->mult[s] = kTuneCand[best];
            }
            ctx->tune_next = -1;
        }
    }
    if (st) {
        st->loop = ctx->loop;
        st->grain_count = ctx->grain_count;
        st->live_grains = ctx->live;
        st->kernel_launches = (int32_t)(ctx->launches - launches0);
        st->voxel_updates = *ctx->h_total_vox;
        float* f[5] = {&st->ms_convolution, &st->ms_lists, &st->ms_comparison, &st->ms_levelset, &st->ms_redistancing};
        for (int i = 0; i < 5; i++) cudaEventElapsedTime(f[i], ctx->ev[i], ctx->ev[i + 1]);
        cudaEventElapsedTime(&st->ms_total, ctx->ev[0], ctx->ev[5]);
        cudaEventElapsedTime(&st->ms_compare_kernel, ctx->ev[6], ctx->ev[7]);
        st->compare_voxels = *ctx->h_total_vox;
    }
    ctx->loop++;
    return GG_OK;
}

template <typename T>
int voxel_container_t(gg_ctx* ctx, uint32_t* d_labels) {
    const int a = ctx->p ^ 1;  // m_outputDistance
    // n tiles per existing grain of the current layout
    plan(ctx, ctx->d_box[a], 1, nullptr, nullptr, ctx->d_toff_n, nullptr, nullptr);
    ContainerArgs<T> c{};
    c.G = ctx->G;
    c.geo = ctx->geo;
    c.toff = ctx->d_toff_n;
    c.src = Arena<const T>{reinterpret_cast<const T*>(ctx->d_arena[a]), ctx->d_box[a], ctx->d_off[a]};
    c.labels = d_labels;
    launch_container<T>(c, ctx->grid, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return GG_OK;
}
}  // namespace

namespace {
int stage_grid(const gg_ctx* c, int s) { return c->num_sms * c->mult[s]; }
}  // namespace

// ===================================================================================
// C ABI
// ===================================================================================
namespace {

// Box of the mode-4 LSbox constructor (box.cpp:239-304) followed by resizeToCube.
Box initial_box(const int32_t* e, int gb, int M) {
    int xmin = e[0], xmax = e[1], ymin = e[2], ymax = e[3], zmin = e[4], zmax = e[5];
    xmax += 2 * gb;
    ymax += 2 * gb;
    zmax += 2 * gb;
    if (ymax > M) ymax = M;
    if (xmax > M) xmax = M;
    if (zmax > M) zmax = M;
    if (ymin < 0) ymin = 0;
    if (xmin < 0) xmin = 0;
    if (zmin < 0) zmin = 0;
    // DimensionalBuffer::resizeToCube, dimensionalBuffer.h:139-219
    return resize_to_cube(Box{xmin, xmax, ymin, ymax, zmin, zmax}, M);
}

int supported_side(bool fp64) {
    const size_t lim = 227 * 1024;
    int n = 8;
    for (;;) {
        const int m = n + 1;
        bool ok = redist_smem_bytes(m, fp64) <= lim && mc_slab_bytes(m) + 40 * 1024 <= lim;
        if (fp64) ok = ok && conv_f64_smem_bytes(m) <= lim;
        else ok = ok && 3 * (size_t)m * (m | 1) * 4 <= lim;
        if (!ok || m > 4096) return n;
        n = m;
    }
}

void free_all(gg_ctx* c) {
    void* ptrs[] = {c->d_present, c->d_exists, c->d_newbox, c->d_nnb, c->d_volume, c->d_surface, c->d_nb, c->d_cmp,
                    c->d_son, c->d_ncmp, c->d_nson, c->d_pt, c->d_arena[0], c->d_arena[1], c->d_box[0], c->d_box[1],
                    c->d_off[0], c->d_off[1], c->d_idarena[0], c->d_idarena[1], c->d_idbox[0], c->d_idbox[1],
                    c->d_idoff[0], c->d_idoff[1], c->d_spec, c->d_spec_off, c->d_toff_n, c->d_toff_slab,
                    c->d_toff_one, c->d_toff_mc, c->d_toff_red, c->d_toff_big, c->d_tw, c->d_tw_off, c->d_gtab, c->d_g_off,
                    c->d_circ, c->d_circ_off, c->d_bmat, c->d_boff, c->d_cscr, c->d_elscr, c->d_quat, c->d_see,
                    c->hull.rec_list, c->hull.rec_ntri, c->hull.bary, c->hull.tarea, c->hull.diag, c->el.earea, c->el.ebf, c->el.eidx, c->el.n_flat, c->el.eorg, c->hull.n_rec, c->hull.n_tri, c->el.n_elem,
                    c->el.elem, c->el.ids, c->el.segs, c->el.ebary, c->el.n_idx, c->el.idx_key, c->el.idx_rng,
                    c->el.idx_elem, c->d_err, c->d_total_vox, c->d_count3, c->bins.count, c->work.keys,
                    c->d_toff_rcls, c->work.keys_out, c->work.vals, c->work.order, c->work.item_off, c->work.temp, c->work.queue,
                    c->bins.off, c->bins.cursor, c->bins.entries, c->bins.max_count, c->bins.temp, c->lbins.count,
                    c->lbins.off, c->lbins.cursor, c->lbins.entries};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->h_maxcount) cudaFreeHost(c->h_maxcount);
    if (c->h_count3) cudaFreeHost(c->h_count3);
    if (c->h_total_vox) cudaFreeHost(c->h_total_vox);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
}

}  // namespace

extern "C" {

int gg_create(const gg_params* params, gg_ctx** out) {
    gg_ctx* ctx = nullptr;
    if (!params || !out) return GG_ERR_INVALID;
    *out = nullptr;
    ctx = new gg_ctx();
    ctx->P = *params;
    const gg_params& P = ctx->P;
    int rc = GG_OK;
    if (P.domain_size < 2 || P.border < 0 || P.n_grains < 1 || !(P.time_step > 0))
        rc = fail(ctx, GG_ERR_INVALID, "invalid geometry (domain_size=%d border=%d n_grains=%d)", P.domain_size,
                  P.border, P.n_grains);
    else if (P.precision != GG_PRECISION_FP64 && P.precision != GG_PRECISION_MIXED)
        rc = fail(ctx, GG_ERR_INVALID, "unknown precision mode %d", P.precision);
    else if (list_smem_bytes(P.n_grains) > 227 * 1024)
        rc = fail(ctx, GG_ERR_UNSUPPORTED, "%d grains: the list update's ID bitmaps exceed shared memory",
                  P.n_grains);

    if (rc) {
        *out = ctx;  // keep the message readable through gg_last_error
        return rc;
    }
    ctx->G = P.n_grains;
    ctx->N = P.domain_size;
    ctx->gb = P.border;
    ctx->M = ctx->N + 2 * ctx->gb;
    ctx->fp64 = P.precision == GG_PRECISION_FP64;
    ctx->esz = ctx->fp64 ? 8 : 4;
    ctx->geo = Geometry{ctx->N, ctx->gb, ctx->M, 1 / (double)ctx->N, ctx->gb / double(ctx->N), P.time_step};
    ctx->list_cap = P.list_capacity > 0 ? P.list_capacity : 4096;
    ctx->correction = !P.disable_correction;
    ctx->elements = ctx->correction || P.keep_elements;
    ctx->side_limit = supported_side(ctx->fp64);
    // NumberOfPointsPerGrain as the mode-4 reader sets it (grainhdl.cpp:221); ngrains
    ctx->points_per_grain = P.points_per_grain > 0 ? P.points_per_grain
                                                   : (int)(ctx->N / std::pow(ctx->G, 1 / 3.0) + 0.5);
    ctx->coarse_ref = ctx->G;
    ctx->tune_next = P.autotune ? 0 : -1;
    *out = ctx;
#undef CK_RET
    cudaError_t e = cudaSetDevice(P.device);
    if (e != cudaSuccess) return fail(ctx, GG_ERR_CUDA, "cudaSetDevice(%d): %s", P.device, cudaGetErrorString(e));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, P.device));
    ctx->grid = ctx->num_sms * 8;
    for (auto& ev : ctx->ev) CK(cudaEventCreate(&ev));
    const size_t G1 = (size_t)ctx->G + 1;
    CK(dalloc(&ctx->d_present, G1));
    CK(dalloc(&ctx->d_exists, G1));
    CK(dalloc(&ctx->d_newbox, 6 * G1));
    CK(dalloc(&ctx->d_nnb, G1));
    CK(dalloc(&ctx->d_volume, G1));
    CK(dalloc(&ctx->d_surface, G1));
    CK(dalloc(&ctx->d_nb, (size_t)kNbCap * G1));
    CK(dalloc(&ctx->d_cmp, (size_t)ctx->list_cap * G1));
    ctx->pos_cap = 64;
    while (ctx->pos_cap < 2 * ctx->list_cap) ctx->pos_cap <<= 1;  // load factor <= 1/2 at full lists
    CK(dalloc(&ctx->d_pt, (size_t)ctx->pos_cap * G1));
    CK(dalloc(&ctx->d_son, (size_t)ctx->list_cap * G1));
    CK(dalloc(&ctx->d_ncmp, G1));
    CK(dalloc(&ctx->d_nson, G1));
    for (int a = 0; a < 2; a++) {
        CK(dalloc(&ctx->d_box[a], 6 * G1));
        CK(dalloc(&ctx->d_off[a], G1));
        CK(dalloc(&ctx->d_idbox[a], 6 * G1));
        CK(dalloc(&ctx->d_idoff[a], G1));
    }
    CK(dalloc(&ctx->d_spec_off, G1));
    CK(dalloc(&ctx->d_toff_n, G1 + 1));
    CK(dalloc(&ctx->d_toff_slab, G1 + 1));
    CK(dalloc(&ctx->d_toff_one, G1 + 1));
    CK(dalloc(&ctx->d_toff_mc, G1 + 1));
    CK(dalloc(&ctx->d_toff_red, G1 + 1));
    CK(dalloc(&ctx->d_toff_big, G1 + 1));
    CK(dalloc(&ctx->d_toff_rcls, (size_t)kRedistClasses * (G1 + 1)));
    CK(dalloc(&ctx->work.keys, G1));
    CK(dalloc(&ctx->work.keys_out, G1));
    CK(dalloc(&ctx->work.vals, G1));
    CK(dalloc(&ctx->work.order, G1));
    CK(dalloc(&ctx->work.item_off, G1 + 1));
    CK(dalloc(&ctx->work.queue, kQueues));
    ctx->work.temp_bytes = work_order_temp_bytes(ctx->G);
    CK(cudaMalloc(&ctx->work.temp, ctx->work.temp_bytes ? ctx->work.temp_bytes : 1));
    CK(dalloc(&ctx->d_err, 1));
    CK(dalloc(&ctx->d_total_vox, 1));
    CK(dalloc(&ctx->d_count3, 3));
    {
        std::vector<double4> q(G1, euler_to_quat(0, 0, 0));
        q[0] = euler_to_quat(0, 35 * (kPi / 180), 0);  // the boundary grain, grainhdl.cpp:86
        std::vector<double> see(G1, 0.0);
        CK(dalloc(&ctx->d_quat, G1));
        CK(dalloc(&ctx->d_see, G1));
        CK(cudaMemcpy(ctx->d_quat, q.data(), sizeof(double4) * G1, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->d_see, see.data(), sizeof(double) * G1, cudaMemcpyHostToDevice));
    }
    ctx->bins.ntx = (ctx->M + kTX - 1) / kTX;
    ctx->bins.nty = (ctx->M + kTY - 1) / kTY;
    ctx->bins.ntz = (ctx->M + kTZ - 1) / kTZ;
    const size_t n_tiles = (size_t)ctx->bins.ntx * ctx->bins.nty * ctx->bins.ntz;
    CK(dalloc(&ctx->bins.count, n_tiles + 1));
    CK(dalloc(&ctx->bins.off, n_tiles + 1));
    CK(dalloc(&ctx->bins.cursor, n_tiles + 1));
    CK(dalloc(&ctx->bins.max_count, 1));
    ctx->bins.temp_bytes = exclusive_scan_temp_bytes((int)n_tiles + 1);
    CK(cudaMalloc(&ctx->bins.temp, ctx->bins.temp_bytes ? ctx->bins.temp_bytes : 1));
    {
        const int n = ctx->M / kListCell + 1;
        ctx->lbins_cells = n * n * n;
        CK(dalloc(&ctx->lbins.count, (size_t)ctx->lbins_cells + 1));
        CK(dalloc(&ctx->lbins.off, (size_t)ctx->lbins_cells + 1));
        CK(dalloc(&ctx->lbins.cursor, (size_t)ctx->lbins_cells + 1));
    }
    CK(cudaMallocHost((void**)&ctx->h_maxcount, sizeof(int)));
    CK(cudaMallocHost((void**)&ctx->h_count3, 3 * sizeof(int)));
    CK(cudaMallocHost((void**)&ctx->h_total_vox, sizeof(long long)));
    CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
    CK(cudaMemset(ctx->d_total_vox, 0, sizeof(long long)));
    CK(cudaMemset(ctx->d_present, 0, sizeof(int) * G1));
    CK(cudaMemset(ctx->d_exists, 0, sizeof(int) * G1));
    CK(cudaMemset(ctx->d_nnb, 0, sizeof(int) * G1));
    CK(cudaMemset(ctx->d_ncmp, 0, sizeof(int) * G1));
    CK(cudaMemset(ctx->d_nson, 0, sizeof(int) * G1));
    CK(cudaMemset(ctx->d_volume, 0, sizeof(double) * G1));
    CK(cudaMemset(ctx->d_surface, 0, sizeof(double) * G1));
    for (int a = 0; a < 2; a++) {
        CK(cudaMemset(ctx->d_box[a], 0, sizeof(int) * 6 * G1));
        CK(cudaMemset(ctx->d_off[a], 0, sizeof(long long) * G1));
        CK(cudaMemset(ctx->d_idbox[a], 0, sizeof(int) * 6 * G1));
        CK(cudaMemset(ctx->d_idoff[a], 0, sizeof(long long) * G1));
    }
    return upload_tables(ctx);
}

int gg_destroy(gg_ctx* ctx) {
    if (!ctx) return GG_OK;
    free_all(ctx);
    delete ctx;
    return GG_OK;
}

const char* gg_last_error(const gg_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int gg_load_state(gg_ctx* ctx, const uint32_t* labels, const int32_t* extents, const int64_t* counts) {
    if (!ctx || !labels || !extents || !counts) return GG_ERR_INVALID;
    if (ctx->loaded) return fail(ctx, GG_ERR_INVALID, "state already loaded");
    const int G = ctx->G, gb = ctx->gb, M = ctx->M;
    std::vector<int> present(G + 1, 0), box(6 * (G + 1), 0);
    long long need = 0;
    int side = 0;
    for (int g = 1; g <= G; g++) {
        if (counts[g - 1] <= 0) continue;  // the reference skips empty grains, grainhdl.cpp:492-497
        const Box b = initial_box(extents + 6 * (g - 1), gb, M);
        if (b.x0 < 0 || b.y0 < 0 || b.z0 < 0 || b.nx() <= 0 || b.nx() != b.ny() || b.nx() != b.nz())
            return fail(ctx, GG_ERR_INVALID, "grain %d: invalid initial box", g);
        present[g] = 1;
        store_box(&box[6 * g], b);
        need += (b.count() + 31) / 32 * 32;
        side = std::max(side, b.nx());
    }
    int rc = side_check(ctx, side);
    if (rc) return rc;
    ctx->side_max = side;
    ctx->pool_voxels = ctx->P.pool_voxels > 0 ? ctx->P.pool_voxels : 2 * need + 4096;
    if (need > ctx->pool_voxels)
        return fail(ctx, GG_ERR_POOL_EXHAUSTED, "initial boxes need %lld voxels, pool holds %lld", need,
                    ctx->pool_voxels);
    ctx->spec_capacity = ctx->fp64 ? (ctx->pool_voxels * 6) / 10 + 32LL * (G + 1) : 0;
    for (int a = 0; a < 2; a++) {
        CK(cudaMalloc(&ctx->d_arena[a], ctx->esz * ctx->pool_voxels));
        CK(dalloc(&ctx->d_idarena[a], ctx->pool_voxels));
    }
    if (ctx->fp64) CK(dalloc(&ctx->d_spec, ctx->spec_capacity));
    else if (ctx->correction) CK(dalloc(&ctx->d_cscr, ctx->pool_voxels));
    if (ctx->elements) {
        const long long cap = ctx->P.hull_capacity > 0 ? ctx->P.hull_capacity : 16LL * side * side + 2048;
        const size_t G1h = (size_t)G + 1;
        ctx->hull.cap = (int)cap;
        CK(dalloc(&ctx->hull.rec_list, 8 * cap * G1h));
        CK(dalloc(&ctx->hull.rec_ntri, cap * G1h));
        CK(dalloc(&ctx->hull.bary, 3 * cap * G1h));
        CK(dalloc(&ctx->hull.tarea, cap * G1h));
        CK(dalloc(&ctx->hull.diag, 1));
        CK(cudaMemset(ctx->hull.diag, 0, sizeof(int)));
        CK(dalloc(&ctx->hull.n_rec, G1h));
        CK(dalloc(&ctx->hull.n_tri, G1h));
        ctx->el.elem_cap = 512;
        ctx->el.id_cap = 4096;
        ctx->el.seg_cap = 1024;
        ctx->el.bary_cap = (int)cap;
        CK(dalloc(&ctx->el.n_elem, G1h));
        CK(dalloc(&ctx->el.elem, (size_t)ctx->el.elem_cap * G1h));
        CK(dalloc(&ctx->el.ids, (size_t)ctx->el.id_cap * G1h));
        CK(dalloc(&ctx->el.segs, (size_t)ctx->el.seg_cap * G1h));
        CK(dalloc(&ctx->el.ebary, 3 * cap * G1h));
        CK(dalloc(&ctx->el.earea, cap * G1h));
        ctx->el.flat_cap = (int)((cap + ctx->el.elem_cap + 1) & ~1LL);
        CK(dalloc(&ctx->el.ebf, (size_t)ctx->el.flat_cap * G1h));
        CK(dalloc(&ctx->el.eidx, (size_t)ctx->el.flat_cap * G1h));
        CK(dalloc(&ctx->el.n_flat, G1h));
        CK(cudaMemset(ctx->el.n_flat, 0, sizeof(int) * G1h));
        CK(dalloc(&ctx->el.eorg, G1h));
        CK(cudaMemset(ctx->el.eorg, 0, sizeof(float4) * G1h));
        ctx->el.idx_cap = 256;
        ctx->el.pair_cap = 2048;
        CK(dalloc(&ctx->el.n_idx, G1h));
        CK(dalloc(&ctx->el.idx_key, (size_t)ctx->el.idx_cap * G1h));
        CK(dalloc(&ctx->el.idx_rng, (size_t)ctx->el.idx_cap * G1h));
        CK(dalloc(&ctx->el.idx_elem, (size_t)ctx->el.pair_cap * G1h));
        ctx->elscr_ctas = ctx->num_sms * 16;
        CK(dalloc(&ctx->d_elscr, elements_scratch_per_cta() * ctx->elscr_ctas));
        CK(cudaMemset(ctx->el.n_elem, 0, sizeof(int) * G1h));
        CK(cudaMemset(ctx->el.n_idx, 0, sizeof(int) * G1h));
        CK(cudaMemset(ctx->hull.n_rec, 0, sizeof(int) * G1h));
        CK(cudaMemset(ctx->hull.n_tri, 0, sizeof(int) * G1h));
    }
    const size_t G1 = (size_t)G + 1;
    CK(cudaMemcpy(ctx->d_present, present.data(), sizeof(int) * G1, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_exists, present.data(), sizeof(int) * G1, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_box[0], box.data(), sizeof(int) * 6 * G1, cudaMemcpyHostToDevice));
    rc = ctx->fp64 ? load_state_t<double>(ctx, labels) : load_state_t<float>(ctx, labels);
    if (rc) return rc;
    rc = read_counts(ctx, ctx->d_box[1]);
    if (rc) return rc;
    ctx->loaded = true;
    ctx->loop = 0;
    return GG_OK;
}

int gg_set_lists(gg_ctx* ctx, const int64_t* offsets, const uint32_t* ids) {
    if (!ctx || !offsets || (!ids && offsets[ctx->G + 1] > 0)) return GG_ERR_INVALID;
    const int G = ctx->G, cap = ctx->list_cap;
    for (int g = 1; g <= G; g++) {
        const int64_t len = offsets[g + 1] - offsets[g];
        if (len < 0 || len > cap) return fail(ctx, GG_ERR_LIST_OVERFLOW, "list of grain %d has %lld entries", g, (long long)len);
        for (int64_t k = 0; k < len; k++) {
            const uint32_t v = ids[offsets[g] + k];
            if (v < 1 || v > (uint32_t)G) return fail(ctx, GG_ERR_INVALID, "list of grain %d names grain %u", g, v);
        }
    }
    // the packed lists cross once; a kernel spreads them over the fixed-capacity rows
    const int64_t total = offsets[G + 1];
    int64_t* d_off = nullptr;
    uint32_t* d_ids = nullptr;
    CK(dalloc(&d_off, (size_t)G + 2));
    CK(dalloc(&d_ids, (size_t)(total > 0 ? total : 1)));
    CK(cudaMemcpyAsync(d_off, offsets, sizeof(int64_t) * (G + 2), cudaMemcpyHostToDevice, ctx->stream));
    if (total > 0) CK(cudaMemcpyAsync(d_ids, ids, sizeof(uint32_t) * total, cudaMemcpyHostToDevice, ctx->stream));
    launch_scatter_lists(G, d_off, d_ids, ctx->d_cmp, ctx->d_ncmp, ctx->d_son, ctx->d_nson, cap, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(d_off));
    CK(cudaFree(d_ids));
    return GG_OK;
}

int gg_default_lists(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    DefaultListArgs a{};
    a.G = ctx->G;
    a.present = ctx->d_present;
    a.box = ctx->d_box[ctx->p ^ 1];
    a.cmp = ctx->d_cmp;
    a.n_cmp = ctx->d_ncmp;
    a.son = ctx->d_son;
    a.n_son = ctx->d_nson;
    a.list_cap = ctx->list_cap;
    a.err = ctx->d_err;
    launch_default_lists(a, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return check_err(ctx, "gg_default_lists");
}

int gg_rtree_lists(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    const size_t G1 = (size_t)ctx->G + 1;
    std::vector<int32_t> boxes(6 * G1);
    std::vector<int> present(G1), exists(G1);
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(boxes.data(), ctx->d_box[ctx->p ^ 1], sizeof(int32_t) * 6 * G1, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(present.data(), ctx->d_present, sizeof(int) * G1, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(exists.data(), ctx->d_exists, sizeof(int) * G1, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> valid(G1, 0);
    for (size_t g = 1; g < G1; g++) valid[g] = (uint8_t)(present[g] && exists[g]);
    std::vector<int64_t> off(G1 + 1, 0);
    const int64_t total = gg_rtree_lists_from_boxes(ctx->G, boxes.data(), valid.data(), off.data(), nullptr, 0);
    if (total < 0) return fail(ctx, (int)total, "R-tree lists: invalid boxes");
    std::vector<uint32_t> ids(total > 0 ? total : 1);
    gg_rtree_lists_from_boxes(ctx->G, boxes.data(), valid.data(), off.data(), ids.data(), total);
    return gg_set_lists(ctx, off.data(), ids.data());
}

int gg_stage_convolution(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    int rc = ctx->fp64 ? stage_convolution_t<double>(ctx) : stage_convolution_t<float>(ctx);
    return rc ? rc : check_err(ctx, "convolution");
}
int gg_stage_update_lists(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    int rc = stage_update_lists_t(ctx);
    return rc ? rc : check_err(ctx, "update lists");
}
int gg_stage_comparison(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    int rc = ctx->fp64 ? stage_comparison_t<double>(ctx) : stage_comparison_t<float>(ctx);
    return rc ? rc : check_err(ctx, "comparison");
}
int gg_stage_level_set(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    int rc = ctx->fp64 ? stage_level_set_t<double>(ctx) : stage_level_set_t<float>(ctx);
    return rc ? rc : check_err(ctx, "level set");
}
int gg_stage_redistancing(gg_ctx* ctx) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    int rc = ctx->fp64 ? stage_redistancing_t<double>(ctx) : stage_redistancing_t<float>(ctx);
    if (rc) return rc;
    rc = check_err(ctx, "redistancing");
    if (rc) return rc;
    ctx->loop++;
    return GG_OK;
}

int gg_step(gg_ctx* ctx, gg_step_stats* stats) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    return ctx->fp64 ? step_t<double>(ctx, stats) : step_t<float>(ctx, stats);
}

int gg_get_grain_stats(gg_ctx* ctx, uint8_t* exists, double* volume, double* surface, int32_t* boxes,
                       int32_t* n_neighbors) {
    if (!ctx || !ctx->loaded) return GG_ERR_INVALID;
    const size_t G1 = (size_t)ctx->G + 1;
    CK(cudaStreamSynchronize(ctx->stream));
    if (exists) {
        std::vector<int> pr(G1), ex(G1);
        CK(cudaMemcpy(pr.data(), ctx->d_present, sizeof(int) * G1, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ex.data(), ctx->d_exists, sizeof(int) * G1, cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < G1; g++) exists[g] = (uint8_t)(g > 0 && pr[g] && ex[g]);
    }
    if (volume) CK(cudaMemcpy(volume, ctx->d_volume, sizeof(double) * G1, cudaMemcpyDeviceToHost));
    if (surface) CK(cudaMemcpy(surface, ctx->d_surface, sizeof(double) * G1, cudaMemcpyDeviceToHost));
    if (boxes) CK(cudaMemcpy(boxes, ctx->d_box[ctx->p ^ 1], sizeof(int) * 6 * G1, cudaMemcpyDeviceToHost));
    if (n_neighbors) CK(cudaMemcpy(n_neighbors, ctx->d_nnb, sizeof(int) * G1, cudaMemcpyDeviceToHost));
    return GG_OK;
}

int gg_get_neighbors(gg_ctx* ctx, int32_t id, uint32_t* out, int32_t cap) {
    if (!ctx || id < 1 || id > ctx->G) return GG_ERR_INVALID;
    int n = 0;
    CK(cudaMemcpy(&n, ctx->d_nnb + id, sizeof(int), cudaMemcpyDeviceToHost));
    const int k = std::min(std::min(n, cap), kNbCap);
    if (out && k > 0)
        CK(cudaMemcpy(out, ctx->d_nb + (size_t)id * kNbCap, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost));
    return n;
}

int gg_get_list(gg_ctx* ctx, int32_t id, uint32_t* out, int32_t cap) {
    if (!ctx || id < 1 || id > ctx->G) return GG_ERR_INVALID;
    int n = 0;
    CK(cudaMemcpy(&n, ctx->d_ncmp + id, sizeof(int), cudaMemcpyDeviceToHost));
    const int k = std::min(n, cap);
    if (out && k > 0)
        CK(cudaMemcpy(out, ctx->d_cmp + (size_t)id * ctx->list_cap, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost));
    return n;
}

int64_t gg_get_sdf(gg_ctx* ctx, int32_t id, int32_t which, int32_t box[6], double* out, int64_t cap) {
    if (!ctx || !ctx->loaded || id < 1 || id > ctx->G || !box) return GG_ERR_INVALID;
    const int a = which == 0 ? ctx->p : ctx->p ^ 1;
    long long off = 0;
    CK(cudaMemcpy(box, ctx->d_box[a] + 6 * id, sizeof(int) * 6, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&off, ctx->d_off[a] + id, sizeof(long long), cudaMemcpyDeviceToHost));
    const Box b = load_box(box);
    const long long n = b.count();
    if (out && n > 0) {
        const long long k = std::min((long long)cap, n);
        if (ctx->fp64) {
            CK(cudaMemcpy(out, (double*)ctx->d_arena[a] + off, sizeof(double) * k, cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> tmp(k);
            CK(cudaMemcpy(tmp.data(), (float*)ctx->d_arena[a] + off, sizeof(float) * k, cudaMemcpyDeviceToHost));
            for (long long i = 0; i < k; i++) out[i] = tmp[i];
        }
    }
    return n;
}

int64_t gg_get_idlocal(gg_ctx* ctx, int32_t id, int32_t box[6], uint32_t* out, int64_t cap) {
    if (!ctx || !ctx->loaded || id < 1 || id > ctx->G || !box) return GG_ERR_INVALID;
    long long off = 0;
    CK(cudaMemcpy(box, ctx->d_idbox[ctx->q] + 6 * id, sizeof(int) * 6, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&off, ctx->d_idoff[ctx->q] + id, sizeof(long long), cudaMemcpyDeviceToHost));
    const long long n = load_box(box).count();
    if (out && n > 0)
        CK(cudaMemcpy(out, ctx->d_idarena[ctx->q] + off, sizeof(uint32_t) * std::min((long long)cap, n),
                      cudaMemcpyDeviceToHost));
    return n;
}

int gg_grain_count(gg_ctx* ctx) { return ctx ? ctx->grain_count : GG_ERR_INVALID; }
int gg_domain_size(gg_ctx* ctx) { return ctx ? ctx->N : GG_ERR_INVALID; }

int gg_launch_config(gg_ctx* ctx, int32_t ctas_per_sm[5]) {
    if (!ctx || !ctas_per_sm) return GG_ERR_INVALID;
    for (int s = 0; s < 5; s++) ctas_per_sm[s] = ctx->mult[s];
    return ctx->tune_next >= 0 ? 0 : 1;
}
int gg_loop(gg_ctx* ctx) { return ctx ? ctx->loop : GG_ERR_INVALID; }

int gg_voxel_container(gg_ctx* ctx, uint32_t* labels) {
    if (!ctx || !labels || !ctx->loaded) return GG_ERR_INVALID;
    const size_t n = (size_t)ctx->N * ctx->N * ctx->N;
    uint32_t* d = nullptr;
    CK(dalloc(&d, n));
    CK(cudaMemsetAsync(d, 0, sizeof(uint32_t) * n, ctx->stream));
    int rc = ctx->fp64 ? voxel_container_t<double>(ctx, d) : voxel_container_t<float>(ctx, d);
    if (rc == GG_OK) {
        CK(cudaMemcpyAsync(labels, d, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    CK(cudaFree(d));
    return rc == GG_OK ? check_err(ctx, "gg_voxel_container") : rc;
}

int64_t gg_get_faces(gg_ctx* ctx, double* area, uint32_t* grain_a, uint32_t* grain_b, int64_t cap) {
    if (!ctx || !ctx->loaded || cap < 0 || (cap > 0 && (!area || !grain_a || !grain_b))) return GG_ERR_INVALID;
    if (!ctx->elements)
        return fail(ctx, GG_ERR_UNSUPPORTED, "gg_get_faces needs the interfacial elements (correction or keep_elements)");
    const int G = ctx->G;
    int* d_count = nullptr;
    long long* d_off = nullptr;
    CK(dalloc(&d_count, (size_t)G + 1));
    CK(dalloc(&d_off, (size_t)G + 1));
    CK(cudaMemsetAsync(d_count, 0, sizeof(int) * (G + 1), ctx->stream));
    launch_faces(G, ctx->d_exists, ctx->el, ctx->geo.h, nullptr, d_count, nullptr, nullptr, nullptr, ctx->stream);
    std::vector<int> count(G + 1);
    std::vector<long long> off(G + 1, 0);
    CK(cudaMemcpyAsync(count.data(), d_count, sizeof(int) * (G + 1), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    long long total = 0;
    for (int g = 1; g <= G; g++) {
        off[g] = total;
        total += count[g];
    }
    double* d_area = nullptr;
    uint32_t *d_a = nullptr, *d_b = nullptr;
    CK(dalloc(&d_area, (size_t)(total > 0 ? total : 1)));
    CK(dalloc(&d_a, (size_t)(total > 0 ? total : 1)));
    CK(dalloc(&d_b, (size_t)(total > 0 ? total : 1)));
    CK(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * (G + 1), cudaMemcpyHostToDevice, ctx->stream));
    launch_faces(G, ctx->d_exists, ctx->el, ctx->geo.h, d_off, d_count, d_area, d_a, d_b, ctx->stream);
    ctx->launches += 2;
    CK(cudaGetLastError());
    const long long n = std::min<long long>(total, cap);
    if (n > 0) {
        CK(cudaMemcpyAsync(area, d_area, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(grain_a, d_a, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(grain_b, d_b, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    for (void* p : {(void*)d_count, (void*)d_off, (void*)d_area, (void*)d_a, (void*)d_b}) CK(cudaFree(p));
    return total;
}

int gg_set_orientations(gg_ctx* ctx, const double* euler) {
    if (!ctx || !euler) return GG_ERR_INVALID;
    const size_t G1 = (size_t)ctx->G + 1;
    std::vector<double4> q(G1);
    q[0] = euler_to_quat(0, 35 * (kPi / 180), 0);
    for (int g = 1; g <= ctx->G; g++)
        q[g] = euler_to_quat(euler[3 * (g - 1)], euler[3 * (g - 1) + 1], euler[3 * (g - 1) + 2]);
    CK(cudaMemcpy(ctx->d_quat, q.data(), sizeof(double4) * G1, cudaMemcpyHostToDevice));
    return GG_OK;
}

int gg_set_stored_energy(gg_ctx* ctx, const double* see) {
    if (!ctx || !see) return GG_ERR_INVALID;
    std::vector<double> v((size_t)ctx->G + 1, 0.0);
    for (int g = 1; g <= ctx->G; g++) v[g] = see[g - 1];
    CK(cudaMemcpy(ctx->d_see, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
    return GG_OK;
}

int gg_get_elements(gg_ctx* ctx, int32_t id, int32_t counts[4]) {
    if (!ctx || !ctx->loaded || id < 1 || id > ctx->G || !counts) return GG_ERR_INVALID;
    counts[0] = counts[1] = counts[2] = counts[3] = 0;
    if (!ctx->elements) return GG_OK;
    int ne = 0;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(&ne, ctx->el.n_elem + id, sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<HullElem> e(ne > 0 ? ne : 1);
    if (ne > 0)
        CK(cudaMemcpy(e.data(), ctx->el.elem + (size_t)id * ctx->el.elem_cap, sizeof(HullElem) * ne,
                      cudaMemcpyDeviceToHost));
    for (int i = 0; i < ne; i++)
        if (e[i].type >= 1 && e[i].type <= 4) counts[e[i].type - 1]++;
    return GG_OK;
}

int gg_convolve_boxes_f64(const double* d_in, double* d_out, const int32_t* sides, const int64_t* offs,
                          int32_t n_boxes, int32_t domain_size, double time_step) {
    gg_ctx* ctx = nullptr;  // for CK: no context to carry a message
    if (!d_in || !d_out || !sides || !offs || n_boxes < 1 || domain_size < 1) return GG_ERR_INVALID;
    int nmax = 0;
    for (int b = 0; b < n_boxes; b++) nmax = std::max(nmax, (int)sides[b]);
    int dev = 0, sms = 0, optin = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (nmax < 1 || conv_f64_smem_bytes(nmax) > (size_t)optin) return GG_ERR_UNSUPPORTED;
    std::vector<double2> tw;
    std::vector<long long> tw_off(nmax + 2, 0), g_off(nmax + 2, 0);
    std::vector<double> gt;
    for (int n = 1; n <= nmax; n++) {
        tw_off[n] = (long long)tw.size();
        twiddle_table(n, tw);
        g_off[n] = (long long)gt.size();
        gaussian_table(n, domain_size, time_step, gt);
    }
    // grains 1..n_boxes, box b at (0, n, 0, n, 0, n)
    std::vector<int> box(6 * (n_boxes + 1), 0);
    std::vector<long long> off(n_boxes + 1, 0), spec_off(n_boxes + 1, 0);
    std::vector<int> toff(n_boxes + 2, 0);
    long long spec_total = 0;
    for (int b = 0; b < n_boxes; b++) {
        const int n = sides[b];
        int* bb = &box[6 * (b + 1)];
        bb[1] = bb[3] = bb[5] = n;
        off[b + 1] = offs[b];
        spec_off[b + 1] = spec_total;
        spec_total += (long long)n * n * (n / 2 + 1);
        toff[b + 2] = toff[b + 1] + n;
    }
    double2 *d_tw = nullptr, *d_spec = nullptr;
    double* d_gt = nullptr;
    long long *d_tw_off = nullptr, *d_g_off = nullptr, *d_off = nullptr, *d_spec_off = nullptr;
    int *d_box = nullptr, *d_toff = nullptr;
    CK(dalloc(&d_tw, tw.size()));
    CK(dalloc(&d_gt, gt.size()));
    CK(dalloc(&d_tw_off, tw_off.size()));
    CK(dalloc(&d_g_off, g_off.size()));
    CK(dalloc(&d_spec, spec_total));
    CK(dalloc(&d_box, box.size()));
    CK(dalloc(&d_off, off.size()));
    CK(dalloc(&d_spec_off, spec_off.size()));
    CK(dalloc(&d_toff, toff.size()));
    CK(cudaMemcpy(d_tw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_gt, gt.data(), sizeof(double) * gt.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_tw_off, tw_off.data(), sizeof(long long) * tw_off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_g_off, g_off.data(), sizeof(long long) * g_off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_box, box.data(), sizeof(int) * box.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_spec_off, spec_off.data(), sizeof(long long) * spec_off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_toff, toff.data(), sizeof(int) * toff.size(), cudaMemcpyHostToDevice));
    ConvArgs a{};
    a.G = n_boxes;
    a.toff = d_toff;
    a.in = d_in;
    a.in_box = d_box;
    a.in_off = d_off;
    a.out = d_out;
    a.out_off = d_off;
    a.spec = d_spec;
    a.spec_off = d_spec_off;
    a.tw = d_tw;
    a.tw_off = d_tw_off;
    a.gtab = d_gt;
    a.g_off = d_g_off;
    launch_conv_f64(a, (sms > 0 ? sms : 148) * 8, conv_f64_smem_bytes(nmax), 0);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    void* ptrs[] = {d_tw, d_gt, d_tw_off, d_g_off, d_spec, d_box, d_off, d_spec_off, d_toff};
    for (void* p : ptrs) cudaFree(p);
    return GG_OK;
}

int gg_convolve_boxes_mixed(const float* d_in, float* d_out, const int32_t* sides, const int64_t* offs,
                            int32_t n_boxes, int32_t domain_size, double time_step) {
    gg_ctx* ctx = nullptr;  // for CK: no context to carry a message
    if (!d_in || !d_out || !sides || !offs || n_boxes < 1 || domain_size < 1) return GG_ERR_INVALID;
    int nmax = 0;
    long long span = 0;
    for (int b = 0; b < n_boxes; b++) {
        if (sides[b] < 1 || offs[b] < 0 || offs[b] % 4) return GG_ERR_INVALID;
        nmax = std::max(nmax, (int)sides[b]);
        span = std::max(span, (long long)offs[b] + (long long)sides[b] * sides[b] * sides[b]);
    }
    const bool tc = umma_supported(nmax);
    if (!tc && 3 * (size_t)nmax * (nmax | 1) * sizeof(float) > 227 * 1024) return GG_ERR_UNSUPPORTED;
    std::vector<int> box(6 * (n_boxes + 1), 0);
    std::vector<long long> off(n_boxes + 1, 0);
    std::vector<int> toff(n_boxes + 2, 0);
    for (int b = 0; b < n_boxes; b++) {
        const int n = sides[b];
        int* bb = &box[6 * (b + 1)];
        bb[1] = bb[3] = bb[5] = n;
        off[b + 1] = offs[b];
        toff[b + 2] = toff[b + 1] + (tc ? (n * n + kUmmaRows - 1) / kUmmaRows : n);
    }
    std::vector<float> tab;
    std::vector<uint16_t> tab16;
    std::vector<long long> tab_off;
    if (tc) {
        umma_tables(domain_size, time_step, nmax, tab16, tab_off);
    } else {
        tab_off.assign(nmax + 2, 0);
        for (int n = 1; n <= nmax; n++) {
            tab_off[n] = (long long)tab.size();
            circulant_matrix(n, domain_size, time_step, tab);
        }
    }
    float *d_tab = nullptr, *d_scr = nullptr;
    uint16_t* d_tab16 = nullptr;
    long long *d_tab_off = nullptr, *d_off = nullptr;
    int *d_box = nullptr, *d_toff = nullptr, *d_err = nullptr;
    CK(dalloc(&d_tab, tab.size()));
    CK(dalloc(&d_tab16, tab16.size()));
    CK(dalloc(&d_tab_off, tab_off.size()));
    CK(dalloc(&d_box, box.size()));
    CK(dalloc(&d_off, off.size()));
    CK(dalloc(&d_toff, toff.size()));
    CK(dalloc(&d_err, 1));
    if (tc) CK(dalloc(&d_scr, (size_t)(span + 4) / 4 * 4));
    if (!tab.empty()) CK(cudaMemcpy(d_tab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice));
    if (!tab16.empty())
        CK(cudaMemcpy(d_tab16, tab16.data(), sizeof(uint16_t) * tab16.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_tab_off, tab_off.data(), sizeof(long long) * tab_off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_box, box.data(), sizeof(int) * box.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_toff, toff.data(), sizeof(int) * toff.size(), cudaMemcpyHostToDevice));
    CK(cudaMemset(d_err, 0, sizeof(int)));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (tc) {
        UmmaConvArgs u{};
        u.G = n_boxes;
        u.toff = d_toff;
        u.box = d_box;
        u.in = d_in;
        u.in_off = d_off;
        u.out = d_out;
        u.out_off = d_off;
        u.scratch = d_scr;
        u.bmat = d_tab16;
        u.boff = d_tab_off;
        u.err = d_err;
        launch_conv_umma(u, sms, nmax, 0);
    } else {
        ConvTCArgs a{};
        a.G = n_boxes;
        a.toff = d_toff;
        a.in = d_in;
        a.box = d_box;
        a.in_off = d_off;
        a.out = d_out;
        a.out_off = d_off;
        a.circ = d_tab;
        a.circ_off = d_tab_off;
        a.err = d_err;
        launch_conv_tc(a, sms, nmax, 0);
    }
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    int e = 0;
    CK(cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    void* ptrs[] = {d_tab, d_tab16, d_tab_off, d_box, d_off, d_toff, d_err, d_scr};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (e & ERR_TIMEOUT) return GG_ERR_CUDA;
    if (e) return GG_ERR_UNSUPPORTED;
    return GG_OK;
}

}  // extern "C"

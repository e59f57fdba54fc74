/*
 * gg_b200.h -- C ABI of the B200-native GraGLeS_3D level-set timestep.
 *
 * The reference drives its per-timestep loop from grainhdl::run_sim
 * (grainhdl.cpp:821-919) through OpenMP loops over LSbox methods (box.h:111-190).
 * This library replaces that loop with device-resident state on one GPU: every
 * grain box lives in a pool in HBM, every stage is a batched CUDA kernel over all
 * boxes, and the host only sequences calls.  Each entry point below names the
 * reference method (file:line) it stands in for.
 *
 * Conventions: every function returns GG_OK (0) or a negative GG_ERR_* code and
 * never throws; gg_last_error() gives the message.  One context = one GPU, one
 * CUDA stream, one host thread.  Boxes are int32[6] = {xmin, xmax, ymin, ymax,
 * zmin, zmax} in absolute grid coordinates (border included), maxima exclusive,
 * and box buffers are flat [z][y][x] with x fastest (dimensionalBuffer.h:71-76).
 * Grain IDs run 1..n_grains; ID 0 is the domain-boundary grain.
 */
#ifndef GG_B200_H
#define GG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GG_OK 0
#define GG_ERR_INVALID (-1)          /* bad argument or call order */
#define GG_ERR_CUDA (-2)             /* a CUDA call failed */
#define GG_ERR_POOL_EXHAUSTED (-3)   /* box pool or scratch capacity exceeded */
#define GG_ERR_LIST_OVERFLOW (-4)    /* a comparison or neighbour list exceeded its capacity */
#define GG_ERR_UNSUPPORTED (-5)      /* option not implemented on this path */

#define GG_PRECISION_FP64 0          /* FP64 storage and arithmetic, bit-exact with the oracle */
#define GG_PRECISION_MIXED 1         /* FP32 storage, tensor-core convolution, FP64 tallies */

typedef struct gg_ctx gg_ctx;

/* The Settings fields the loop reads (Settings.h:63-119, grainhdl.cpp:1419-1442). */
typedef struct {
    int32_t domain_size;        /* realDomainSize N (NX of the mode-4 header) */
    int32_t border;             /* DomainBorderSize (grid_blowup) */
    double time_step;           /* TimeStepSize */
    int32_t n_grains;           /* NumberOfParticles */
    int32_t precision;          /* GG_PRECISION_* */
    int32_t disable_correction; /* DisableConvolutionCorrection (0 = the correction, box.cpp:426-535) */
    int32_t list_capacity;      /* comparison-list capacity per grain (0 = 4096) */
    int64_t pool_voxels;        /* voxels per SDF arena (0 = 2x the initial total) */
    int32_t device;             /* CUDA device ordinal */
    int32_t unique_gb_energies; /* UniqueGBEnergies (correction only) */
    int32_t mobility_model;     /* UseMobilityFactor -> Settings::UseMobilityModel (correction only) */
    int32_t use_stored_energy;  /* UseStoredElasticEnergy (correction only) */
    double triple_line_drag;    /* TripleLineDrag (correction only) */
    int32_t hull_capacity;      /* triangles kept per hull for the correction (0 = 16 side^2 + 2048) */
    int32_t keep_elements;      /* build the interfacial elements every step even without the
                                   correction (computeSurfaceElements, box.cpp:1175-1180), for gg_get_faces */
    int32_t grid_coarsening;    /* GridCoarsement (grainhdl::gridCoarsement, grainhdl.cpp:1446-1498) */
    int32_t points_per_grain;   /* NumberOfPointsPerGrain (0 = the mode-4 reader's rule,
                                   (int)(N / n_grains^(1/3) + 0.5), grainhdl.cpp:221) */
    double coarsening_gradient; /* GridCoarsementGradient (0 = 0.95, the Settings default) */
    int32_t autotune;           /* 1: loops 1..5 each time one launch configuration (2, 4, 8, 16 and 32
                                   CTAs per SM for the grid-stride kernels of every stage) and the
                                   rest run each stage with its fastest; results do not depend on it */
} gg_params;

/* Per-step report (the reference prints the same stage times, grainhdl.cpp:920-933). */
typedef struct {
    int32_t loop;               /* loop index of the step just run */
    int32_t grain_count;        /* currentNrGrains after the step (countGrains) */
    int32_t live_grains;        /* grains whose hull is non-empty after the step */
    int32_t kernel_launches;    /* kernels this library launched for the step */
    int64_t voxel_updates;      /* sum of n^3 over the boxes convolved this step */
    float ms_convolution, ms_lists, ms_comparison, ms_levelset, ms_redistancing, ms_total;
    float ms_compare_kernel;    /* the comparison kernel alone (device time) */
    int64_t compare_voxels;     /* box voxels that kernel compared */
} gg_step_stats;

/* grainhdl::grainhdl + initializeSimulation (grainhdl.cpp:50-128): allocate the
 * context, the box pool and the per-size DFT / Gaussian tables on the device. */
int gg_create(const gg_params* params, gg_ctx** out);
int gg_destroy(gg_ctx* ctx);
const char* gg_last_error(const gg_ctx* ctx);

/* read_voxelized_microstructure + buildBoxVectors + distanceInitialisation
 * (grainhdl.cpp:404-578, 1220-1254, 580-596; box.cpp:227-304, 374-397):
 * labels = N^3 grain IDs [z][y][x] (host memory, IDs 1..n_grains), extents =
 * n_grains x 6 inclusive domain extents {xmin,xmax,ymin,ymax,zmin,zmax}, counts =
 * voxels per grain (0 = no such grain).  Builds the boxes and the initial SDFs on
 * the device. */
int gg_load_state(gg_ctx* ctx, const uint32_t* labels, const int32_t* extents, const int64_t* counts);

/* find_neighbors (grainhdl.cpp:1029-1054, box.cpp:2871-2887): initial comparison
 * lists as CSR (offsets[n_grains + 2], row = grain ID).  The reference fills them
 * from an R-tree search; the order of each row sets the comparison tie-break. */
int gg_set_lists(gg_ctx* ctx, const int64_t* offsets, const uint32_t* ids);
/* The same membership (inclusive box overlap) in grain-ID order, built on the device. */
int gg_default_lists(gg_ctx* ctx);
/* The lists in the reference's own order: find_neighbors' R-tree over the loaded boxes
 * (grainhdl.cpp:1029-1054, box.cpp:2871-2887; RTree.h: quadratic split, 8/4 branches
 * per node, spherical volumes in float), built on the host from the device's initial
 * boxes and uploaded as gg_set_lists does.  A run from these lists is bit-exact with the
 * reference's from its first comparison on. */
int gg_rtree_lists(gg_ctx* ctx);
/* The same R-tree search on caller boxes, without a context (host only): boxes =
 * (n_grains + 1) x 6 in box order, valid[g] != 0 for the grains inserted.  Writes
 * offsets[n_grains + 2] (CSR by grain ID) and up to cap IDs; returns the total ID count
 * or a negative GG_ERR_*. */
int64_t gg_rtree_lists_from_boxes(int32_t n_grains, const int32_t* boxes, const uint8_t* valid, int64_t* offsets,
                                  uint32_t* ids, int64_t cap);

/* One loop iteration of grainhdl::run_sim (grainhdl.cpp:837-917).  With grid_coarsening
 * set, the iteration starts with grainhdl::gridCoarsement (grainhdl.cpp:1446-1498): when
 * the grain count has fallen below coarsening_gradient of its count at the last
 * coarsening, the domain is re-gridded to the smaller size the reference computes
 * (LSbox::resizeGrid trilinear re-sampling, then recalculateIDLocal and extractContour,
 * box.cpp:2595-2702, 1144-1161) before the convolution. */
int gg_step(gg_ctx* ctx, gg_step_stats* stats);

/* grainhdl::realDomainSize: the current grid size N (smaller than the initial one after
 * a grid coarsening). */
int gg_domain_size(gg_ctx* ctx);

/* The launch configuration in use: CTAs per SM of the grid-stride kernels of each stage
 * (convolution with the correction, lists, comparison, level set, redistancing).  No
 * counterpart in the reference (its parallel loops are OpenMP over grains).  Returns 1
 * once the autotuner has chosen them (or when it is off), 0 while it is still trying. */
int gg_launch_config(gg_ctx* ctx, int32_t ctas_per_sm[5]);

/* The stages of one iteration, for stage-level testing, in the order gg_step runs
 * them.  Each stands in for the grainhdl method named. */
int gg_stage_convolution(gg_ctx* ctx);       /* switchDistancebuffer + convolution, :839-849 */
int gg_stage_update_lists(gg_ctx* ctx);      /* switchDistancebuffer + updateSecondOrderNeighbors, :852-853 */
int gg_stage_comparison(gg_ctx* ctx);        /* comparison_box + switchDistancebuffer, :858-868 */
int gg_stage_level_set(gg_ctx* ctx);         /* level_set, :875 */
int gg_stage_redistancing(gg_ctx* ctx);      /* redistancing + countGrains, :881-886 */

/* Host mirror of per-grain state (LSbox getters, box.h:211-250): arrays of
 * n_grains + 1 entries indexed by grain ID (entry 0 unused); any pointer may be NULL. */
int gg_get_grain_stats(gg_ctx* ctx, uint8_t* exists, double* volume, double* surface, int32_t* boxes,
                       int32_t* n_neighbors);
/* Distinct grain IDs of the last hull in first-seen order (GrainHull::getAllNeighbors). */
int gg_get_neighbors(gg_ctx* ctx, int32_t id, uint32_t* out, int32_t cap);
/* Current comparison list (LSbox::m_comparisonList). */
int gg_get_list(gg_ctx* ctx, int32_t id, uint32_t* out, int32_t cap);
/* One of the grain's two SDF buffers as FP64: which = 0 -> m_inputDistance,
 * 1 -> m_outputDistance (after a full step that is the redistanced field).
 * Returns the voxel count; out may be NULL to query the box only. */
int64_t gg_get_sdf(gg_ctx* ctx, int32_t id, int32_t which, int32_t box[6], double* out, int64_t cap);
/* The grain's IDLocal buffer; returns voxels. */
int64_t gg_get_idlocal(gg_ctx* ctx, int32_t id, int32_t box[6], uint32_t* out, int64_t cap);
int gg_grain_count(gg_ctx* ctx);
int gg_loop(gg_ctx* ctx);

/* The voxel container of the current network (grainhdl::saveNetworkAsVoxelContainer with
 * LSbox::copyDataToContainer, grainhdl.cpp:1074-1095, box.cpp:3008-3032): labels =
 * N^3 grain IDs [z][y][x] (host memory), the largest ID of the grains whose current SDF
 * (m_outputDistance) is >= 0 at the voxel -- the reference's last writer in ascending
 * ID order -- and 0 where there is none.  Grains whose hull vanished in the last step
 * are left out (their buffer is not kept; in the reference it holds no voxel >= 0 then). */
int gg_voxel_container(gg_ctx* ctx, uint32_t* labels);

/* GrainHull::get_Faces of every existing grain (grainHull.cpp:1330-1339), as save_Texture
 * writes them to Faces_<loop>.bin (grainhdl.cpp:753-775): per grain in ascending ID order,
 * its grain-boundary elements toward lower IDs in element order, each with its area
 * (GrainBoundary::computeArea, InterfacialElement.cpp:81-91).  Fills at most cap faces and
 * returns the total; needs the elements (the correction on, or keep_elements). */
int64_t gg_get_faces(gg_ctx* ctx, double* area, uint32_t* grain_a, uint32_t* grain_b, int64_t cap);

/* Grain orientations for the convolution correction's boundary energies and
 * mobilities: Bunge Euler angles phi1, PHI, phi2 in radians, 3 per grain for IDs
 * 1..n_grains (the .uds columns read at grainhdl.cpp:480-504, turned into
 * quaternions as myQuaternion::euler2Quaternion, myQuaternion.cpp:168-191).  The
 * boundary grain 0 has (0, 35 deg, 0) (grainhdl.cpp:86).  Default: all (0, 0, 0). */
int gg_set_orientations(gg_ctx* ctx, const double* euler);
/* m_StoredElasticEnergy per grain for IDs 1..n_grains (box.cpp:232-233 computes it from
 * the .uds column as DislocEnPerM * value / HAGB_Energy * Physical_Domain_Size).
 * The boundary grain's, indeterminate in the reference, is 0. */
int gg_set_stored_energy(gg_ctx* ctx, const double* see);
/* Interfacial elements of the grain's last hull (computeSurfaceElements,
 * box.cpp:1175-1180) as counts {GB, TL, QJ, HJ}; only kept with the correction on. */
int gg_get_elements(gg_ctx* ctx, int32_t id, int32_t counts[4]);

/* Single-box stage kernels on caller-owned device memory (stream 0 of the current
 * device), for testing each kernel against the oracle on arbitrary inputs.
 * n_boxes cubic boxes of sides sides[b] packed at element offsets offs[b]. */
int gg_convolve_boxes_f64(const double* d_in, double* d_out, const int32_t* sides, const int64_t* offs,
                          int32_t n_boxes, int32_t domain_size, double time_step);

/* The mixed-precision convolution of GG_PRECISION_MIXED on FP32 boxes: three per-axis
 * contractions with the circulant C_n on the tcgen05 tensor cores (operands split into
 * FP16 hi + lo, three MMAs per K-step, FP32 accumulation in TMEM) when every side is
 * within the tensor-core kernel's limit, on the FP32 SIMT kernels otherwise.  Same packing
 * and stream as gg_convolve_boxes_f64, except that the offsets must be multiples of 4
 * elements and the buffers must extend to a multiple of 4 elements past the last box
 * (boxes are read as 16-byte aligned spans); allocates its scratch.  Replaces the same
 * call site (LSbox::convolutionGeneratorMKL, box.cpp:685-795) as the FP64 entry. */
int gg_convolve_boxes_mixed(const float* d_in, float* d_out, const int32_t* sides, const int64_t* offs,
                            int32_t n_boxes, int32_t domain_size, double time_step);

/* The same FP64 convolution, bit for bit, without allocating any device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- programs that give all device memory to their own pool at start-up,
 * or that keep their device footprint fixed after start-up.  Its scratch (32 MiB
 * half-spectrum) and tables live in fixed device arrays that every GPU loading the
 * library holds until exit.  Limits: n_boxes <= 256, sides <= 96, sum of
 * n*n*(n/2+1) <= 2^21; beyond them it returns GG_ERR_UNSUPPORTED.  The first call on a
 * device looks up the arrays and uploads the twiddles.  Synchronous: it ends with
 * cudaDeviceSynchronize, so it waits for all work on the device.  Calls from one
 * process share the arrays and are therefore serialised by a lock, one at a time. */
int gg_convolve_boxes_f64_noalloc(const double* d_in, double* d_out, const int32_t* sides, const int64_t* offs,
                                  int32_t n_boxes, int32_t domain_size, double time_step);

#ifdef __cplusplus
}
#endif
#endif

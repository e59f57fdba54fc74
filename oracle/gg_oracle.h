/*
 * gg_oracle.h -- CPU restatement of the reference's per-timestep level-set loop.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg as the checker.  The product path never links it.
 *
 * Boxes are int[6] = {xmin, xmax, ymin, ymax, zmin, zmax} in absolute grid
 * coordinates with exclusive maxima (DimensionalBuffer semantics,
 * dimensionalBuffer.h:71-131); box buffers are flat [z][y][x], x fastest.
 */
#ifndef GG_ORACLE_H
#define GG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ggo_sim ggo_sim;

/* ---- whole-loop restatement (grainhdl::run_sim, grainhdl.cpp:821-919) ---- */

/* N = realDomainSize, border = DomainBorderSize, time_step = TimeStepSize. */
ggo_sim* ggo_create(int N, int border, double time_step, int n_grains);
void ggo_destroy(ggo_sim* s);

/* Mode-4 state: labels N^3 uint32 [z][y][x] with grain IDs 1..n_grains; per grain
 * (row g = ID g+1) inclusive domain extents {xmin,xmax,ymin,ymax,zmin,zmax} and the
 * voxel count (0 = no grain, as grainhdl.cpp:492-497).  Builds the boxes
 * (box.cpp:227-304) and the initial SDF (distanceInitialisation, box.cpp:374-397). */
int ggo_load(ggo_sim* s, const uint32_t* labels, const int32_t* extents, const int64_t* counts);

/* Initial comparison lists as CSR over grain IDs 0..n_grains (row 0 unused); this is
 * what find_neighbors (grainhdl.cpp:1029-1054) leaves in m_secondOrderNeighbours. */
int ggo_set_lists(ggo_sim* s, const int64_t* offsets, const uint32_t* ids);

/* Lists by inclusive box overlap in ID order (same members as the reference's
 * R-tree search; the order of members differs). */
int ggo_default_lists(ggo_sim* s);

/* The convolution correction (box.cpp:426-535; off unless set) with its settings:
 * UniqueGBEnergies, UseMobilityModel, TripleLineDrag, UseStoredElasticEnergy. */
void ggo_set_physics(ggo_sim* s, int correction, int unique_gb_energies, int mobility_model,
                     double triple_line_drag, int use_stored_energy);
/* Bunge Euler angles (3 per grain, rows 1..G of a (G+1) x 3 array). */
void ggo_set_orientations(ggo_sim* s, const double* euler);
/* m_StoredElasticEnergy per grain (entries 1..G of a G+1 array). */
void ggo_set_stored_energy(ggo_sim* s, const double* see);
/* Interfacial elements of the grain's last hull: GB, TL, QJ, HJ counts. */
int ggo_grain_elements(const ggo_sim* s, int id, int counts[4]);

/* One loop iteration (grainhdl.cpp:837-917).  Returns currentNrGrains
 * (countGrains, grainhdl.cpp:936-943) or a negative error. */
int ggo_step(ggo_sim* s);

int ggo_loop(const ggo_sim* s);
/* Per grain: exists flag after the last extractContour, box of the live SDF
 * (the redistanced buffer), volume, surface, neighbour count. */
int ggo_grain_info(const ggo_sim* s, int id, int* exists, int32_t box[6], double* volume,
                   double* surface, int* n_neighbors);
/* Distinct grain IDs of the last hull, in the reference's first-seen order. */
int ggo_grain_neighbors(const ggo_sim* s, int id, uint32_t* out, int cap);
/* Current comparison list. */
int ggo_grain_list(const ggo_sim* s, int id, uint32_t* out, int cap);
/* Live SDF box (the buffer redistancing wrote) and its values; returns count. */
int64_t ggo_grain_sdf(const ggo_sim* s, int id, int32_t box[6], double* out, int64_t cap);
/* IDLocal box and values. */
int64_t ggo_grain_idlocal(const ggo_sim* s, int id, int32_t box[6], uint32_t* out, int64_t cap);
/* Sum over live grains of n^3 at the last convolution (voxel-updates of that step). */
int64_t ggo_last_voxels(const ggo_sim* s);

/* ---- single-box stage functions ---- */

/* LSbox::convolutionGeneratorMKL (box.cpp:685-795) with the specified DFT. */
void ggo_convolve_box(int n, int N, double time_step, const double* in, double* out);

/* LSbox::executeRedistancing (box.cpp:2322-2586): in on in_box, out on out_box. */
void ggo_redistance_box(const int32_t in_box[6], const double* in, const int32_t out_box[6],
                        double* out, double h, double delta);

/* Marching cubes + hull statistics (marchingCubes.cpp:364-618, grainHull.cpp:40-155)
 * on one box: returns the triangle count; volume/surface as computeGrainVolume /
 * computeSurfaceArea; distinct IDs in first-seen order (count in *n_nbrs). */
int64_t ggo_mc_box(const int32_t box[6], const double* sdf, const uint32_t* idlocal, uint32_t own_id,
                   double h, double* volume, double* surface, uint32_t* nbrs, int* n_nbrs, int cap);

/* LSbox::executeComparison + boundaryCondition (box.cpp:891-1088) for one grain with
 * box `box` against K neighbour boxes, in list order.  out and idl are on `box`;
 * idl must hold the grain's IDLocal before the stage (stale IDs survive). */
void ggo_compare_box(const int32_t box[6], int K, const int32_t* nb_boxes, const uint32_t* nb_ids,
                     const double* const* nb_sdf, double* out, uint32_t* idl, int M, int border,
                     double h);

/* LSbox::executeSetComparison (box.cpp:814-878): returns the new bbox in newbox. */
void ggo_set_compare_box(const int32_t box[6], const double* in, double* out, double delta, int M,
                         int border, int32_t newbox[6]);

/* DimensionalBuffer::resizeToCube (dimensionalBuffer.h:139-219) applied to box. */
void ggo_resize_to_cube(int32_t box[6], int M);

#ifdef __cplusplus
}
#endif
#endif

/*
 * gg_oracle.c -- CPU restatement of GraGLeS_3D's per-timestep level-set loop
 * (TEST INFRASTRUCTURE; see gg_oracle.h).
 *
 * Scope: the isotropic path (DisableConvolutionCorrection=1, GridCoarsement=0,
 * DecoupleGrains=0, ConvolutionMode=2).  Every function names the reference lines
 * it restates.  Arithmetic follows the reference expression by expression with no
 * floating-point contraction (compile with -ffp-contract=off), so results are
 * bit-identical to the reference compiled with the specified DFT (oracle/gg_dft.c).
 */
#include "gg_oracle.h"
#include "gg_oracle_gb.h"
#include "gg_dft.h"
#include "gg_mc_tables.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GGO_PI 3.14159265358979323846 /* ggLS.h:25 */

typedef struct { int x0, x1, y0, y1, z0, z1; } box_t;

static box_t box_from(const int32_t b[6]) { box_t r = {b[0], b[1], b[2], b[3], b[4], b[5]}; return r; }
static void box_to(box_t b, int32_t o[6]) { o[0] = b.x0; o[1] = b.x1; o[2] = b.y0; o[3] = b.y1; o[4] = b.z0; o[5] = b.z1; }
static size_t box_count(box_t b) {
    return (size_t)((unsigned)(b.x1 - b.x0) * (unsigned)(b.y1 - b.y0) * (unsigned)(b.z1 - b.z0));
}
/* getValueAt(row=i (y), column=j (x), depth=k (z)), dimensionalBuffer.h:71-76 */
static size_t at(box_t b, int i, int j, int k) {
    return (size_t)(k - b.z0) * (size_t)(b.x1 - b.x0) * (size_t)(b.y1 - b.y0) +
           (size_t)(i - b.y0) * (size_t)(b.x1 - b.x0) + (size_t)(j - b.x0);
}

/* A DimensionalBuffer: a box and a std::vector-like store whose resize keeps the
 * flat prefix and zero-fills the tail (dimensionalBuffer.h:120-131). */
typedef struct { box_t b; void* v; size_t size, cap, esz; } buf_t;

static void buf_resize(buf_t* B, box_t nb) {
    size_t n = box_count(nb);
    if (n > B->cap) {
        size_t cap = n;
        B->v = realloc(B->v, cap * B->esz);
        B->cap = cap;
    }
    if (n > B->size) memset((char*)B->v + B->size * B->esz, 0, (n - B->size) * B->esz);
    B->size = n;
    B->b = nb;
}
#define D(B) ((double*)(B)->v)
#define U(B) ((uint32_t*)(B)->v)

/* dimensionalBuffer.h:139-219 */
static box_t resize_to_cube(box_t b, int maximumLength) {
    int grid_size = maximumLength - 1;
    unsigned height = (unsigned)(b.y1 - b.y0), width = (unsigned)(b.x1 - b.x0), depth = (unsigned)(b.z1 - b.z0);
    if (width == height && width == depth) return b;
    int ref = width > height ? (int)width : (int)height;
    if (ref < (int)depth) ref = (int)depth;
    if (ref > (int)width) { int d = ref - (int)width; b.x0 -= d / 2; b.x1 += d / 2 + d % 2; }
    if (ref > (int)height) { int d = ref - (int)height; b.y0 -= d / 2; b.y1 += d / 2 + d % 2; }
    if (ref > (int)depth) { int d = ref - (int)depth; b.z0 -= d / 2; b.z1 += d / 2 + d % 2; }
    if (b.x0 < 0) { int d = -b.x0; b.x1 += d; b.x0 += d; }
    else if (b.x1 > grid_size) { int d = grid_size - b.x1; b.x1 += d; b.x0 += d; }
    if (b.y0 < 0) { int d = -b.y0; b.y1 += d; b.y0 += d; }
    else if (b.y1 > grid_size) { int d = grid_size - b.y1; b.y1 += d; b.y0 += d; }
    if (b.z0 < 0) { int d = -b.z0; b.z1 += d; b.z0 += d; }
    else if (b.z1 > grid_size) { int d = grid_size - b.z1; b.z1 += d; b.z0 += d; }
    return b;
}

void ggo_resize_to_cube(int32_t box[6], int M) { box_to(resize_to_cube(box_from(box), M), box); }

static int sgn(double v) { return (0.0 < v) - (v < 0.0); } /* utilities.h:27-30 */

/* ------------------------------------------------------------------ */
/* Convolution: box.cpp:685-795 (MKL path) with the specified DFT.     */
/* ------------------------------------------------------------------ */
void ggo_convolve_box(int n, int N, double time_step, const double* in, double* out) {
    const int n2 = n / 2 + 1;
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n * n * n2);
    ggdft_forward_r2c_3d(n, in, tmp);
    const double dt = time_step / (double)(N * N);   /* grainhdl.cpp:1431 */
    const double nsq = (double)(N * N);
    const double local_nsq = (double)(n * n);
    for (int k = 0; k < n; k++) {
        int k2 = k < n - k ? k : n - k;
        for (int i = 0; i < n; i++) {
            int i2 = i < n - i ? i : n - i;
            for (int j = 0; j < n2; j++) {
                int j2 = j < n - j ? j : n - j;
                double G = exp(-sqrt(2 / GGO_PI) * (i2 * i2 + j2 * j2 + k2 * k2) * 4.0 * dt * nsq / local_nsq *
                               GGO_PI * GGO_PI) / (local_nsq * n);
                size_t q = (size_t)j + (size_t)n2 * ((size_t)i + (size_t)n * k);
                tmp[2 * q] = tmp[2 * q] * G;
                tmp[2 * q + 1] = tmp[2 * q + 1] * G;
            }
        }
    }
    ggdft_backward_c2r_3d(n, tmp, out);
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* Redistancing: box.cpp:2322-2586.                                     */
/* ------------------------------------------------------------------ */
static void redistance(box_t ib, const double* in, box_t ob, double* out, size_t out_size, double h,
                       double delta) {
#define IN(i, j, k) in[at(ib, i, j, k)]
#define OUT(i, j, k) out[at(ob, i, j, k)]
    double candidate, i_slope, distToZero;
    for (size_t q = 0; q < out_size; q++) out[q] = -1.0;
    int ixmin = ib.x0 < ob.x0 ? ob.x0 : ib.x0;
    int iymin = ib.y0 < ob.y0 ? ob.y0 : ib.y0;
    int izmin = ib.z0 < ob.z0 ? ob.z0 : ib.z0;
    int ixmax = ib.x1 < ob.x1 ? ib.x1 : ob.x1;
    int iymax = ib.y1 < ob.y1 ? ib.y1 : ob.y1;
    int izmax = ib.z1 < ob.z1 ? ib.z1 : ob.z1;
    for (int k = izmin; k < izmax - 1; k++) {
        for (int i = iymin; i < ob.y1; i++) { /* x forward, box.cpp:2367-2401 */
            for (int j = ixmin; j < ob.x1 - 1; j++) {
                if (j < ixmax - 1 && i < iymax) {
                    if (IN(i, j, k) * IN(i, j + 1, k) <= 0.0) {
                        i_slope = (IN(i, j + 1, k) - IN(i, j, k)) / h;
                        distToZero = -IN(i, j, k) / i_slope;
                        if (fabs(OUT(i, j, k)) > fabs(distToZero)) OUT(i, j, k) = -distToZero * sgn(i_slope);
                    }
                    candidate = OUT(i, j, k) + (sgn(IN(i, j + 1, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j + 1, k))) OUT(i, j + 1, k) = candidate;
                } else {
                    candidate = OUT(i, j, k) + (sgn(OUT(i, j + 1, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j + 1, k))) OUT(i, j + 1, k) = candidate;
                }
            }
        }
        for (int i = iymin; i < ob.y1; i++) { /* x backward, box.cpp:2403-2435 */
            for (int j = ixmax - 1; j > ob.x0; j--) {
                if (j > ixmin && i < iymax) {
                    candidate = OUT(i, j, k) + (sgn(IN(i, j - 1, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j - 1, k))) OUT(i, j - 1, k) = candidate;
                } else {
                    candidate = OUT(i, j, k) + sgn(OUT(i, j - 1, k)) * h;
                    if (fabs(candidate) < fabs(OUT(i, j - 1, k))) OUT(i, j - 1, k) = candidate;
                }
            }
        }
        for (int j = ixmin; j < ob.x1; j++) { /* y forward, box.cpp:2437-2472 */
            for (int i = iymin; i < ob.y1 - 1; i++) {
                if (j < ixmax && i < iymax - 1) {
                    if (IN(i, j, k) * IN(i + 1, j, k) <= 0.0) {
                        i_slope = (IN(i + 1, j, k) - IN(i, j, k)) / h;
                        distToZero = -IN(i, j, k) / i_slope;
                        if (fabs(OUT(i, j, k)) > fabs(distToZero)) OUT(i, j, k) = -distToZero * sgn(i_slope);
                    }
                    candidate = OUT(i, j, k) + (sgn(IN(i + 1, j, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i + 1, j, k))) OUT(i + 1, j, k) = candidate;
                } else {
                    candidate = OUT(i, j, k) + (sgn(OUT(i + 1, j, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i + 1, j, k))) OUT(i + 1, j, k) = candidate;
                }
            }
        }
        for (int j = ixmin; j < ob.x1; j++) { /* y backward, box.cpp:2474-2496 */
            for (int i = iymax - 1; i > ob.y0; i--) {
                if (j < ixmax && i > iymin) {
                    candidate = OUT(i, j, k) + (sgn(IN(i - 1, j, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i - 1, j, k))) OUT(i - 1, j, k) = candidate;
                } else {
                    candidate = OUT(i, j, k) + (sgn(OUT(i - 1, j, k)) * h);
                    if (fabs(candidate) < fabs(OUT(i - 1, j, k))) OUT(i - 1, j, k) = candidate;
                }
            }
        }
    }
    for (int k = izmin; k < ob.z1 - 1; k++) { /* z forward, box.cpp:2501-2538 */
        for (int i = iymin; i < ob.y1; i++) {
            for (int j = ixmin; j < ob.x1; j++) {
                if (k < izmax - 1 && i < iymax && j < ixmax) {
                    if (IN(i, j, k) * IN(i, j, k + 1) <= 0.0) {
                        i_slope = (IN(i, j, k + 1) - IN(i, j, k)) / h;
                        distToZero = -IN(i, j, k) / i_slope;
                        if (fabs(OUT(i, j, k)) > fabs(distToZero)) OUT(i, j, k) = -distToZero * sgn(i_slope);
                    }
                    candidate = OUT(i, j, k) + (sgn(IN(i, j, k + 1)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j, k + 1))) OUT(i, j, k + 1) = candidate;
                } else {
                    candidate = OUT(i, j, k) + (sgn(OUT(i, j, k + 1)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j, k + 1))) OUT(i, j, k + 1) = candidate;
                }
            }
        }
    }
    for (int k = izmax - 1; k > ob.z0; k--) { /* z backward, box.cpp:2539-2576 */
        for (int i = iymin; i < ob.y1; i++) {
            for (int j = ixmin; j < ob.x1; j++) {
                if (k > izmin && i < iymax && j < ixmax) {
                    if (IN(i, j, k) * IN(i, j, k - 1) <= 0.0) {
                        i_slope = (IN(i, j, k - 1) - IN(i, j, k)) / h;
                        distToZero = -IN(i, j, k) / i_slope;
                        if (fabs(OUT(i, j, k)) > fabs(distToZero)) OUT(i, j, k) = -distToZero * sgn(i_slope);
                    }
                    candidate = OUT(i, j, k) + (sgn(IN(i, j, k - 1)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j, k - 1))) OUT(i, j, k - 1) = candidate;
                } else {
                    candidate = OUT(i, j, k) + (sgn(OUT(i, j, k - 1)) * h);
                    if (fabs(candidate) < fabs(OUT(i, j, k - 1))) OUT(i, j, k - 1) = candidate;
                }
            }
        }
    }
    for (size_t q = 0; q < out_size; q++) { /* clampValues, dimensionalBufferReal.h:44-57 */
        if (out[q] < -delta) { out[q] = -delta; continue; }
        if (out[q] > delta) { out[q] = delta; continue; }
    }
#undef IN
#undef OUT
}

void ggo_redistance_box(const int32_t in_box[6], const double* in, const int32_t out_box[6], double* out,
                        double h, double delta) {
    box_t ob = box_from(out_box);
    redistance(box_from(in_box), in, ob, out, box_count(ob), h, delta);
}

/* ------------------------------------------------------------------ */
/* Marching cubes + volume/area: marchingCubes.cpp:364-618,            */
/* grainHull.cpp:40-55, 120-131, 146-155.                              */
/* ------------------------------------------------------------------ */
typedef struct { double x, y, z; } v3;

/* marchingCubes.cpp:484-499 */
static v3 vinterp(v3 p1, v3 p2, double v1, double v2) {
    if (fabs(v1) < 0.00001) return p1;
    if (fabs(v2) < 0.00001) return p2;
    if (fabs(v1 - v2) < 0.00001) return p1;
    double mu = v1 / (v1 - v2);
    v3 p = {p1.x + mu * (p2.x - p1.x), p1.y + mu * (p2.y - p1.y), p1.z + mu * (p2.z - p1.z)};
    return p;
}

/* cubeindex bit b <-> corner offset (dx,dy,dz), marchingCubes.cpp:376-385 */
static const int CORNER[8][3] = {{0, 0, 1}, {1, 0, 1}, {1, 0, 0}, {0, 0, 0}, {0, 1, 1}, {1, 1, 1}, {1, 1, 0}, {0, 1, 0}};
/* edge e joins corners (a,b) in the VertexInterp argument order, marchingCubes.cpp:392-469 */
static const int EDGE[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
/* neighbour-list corner order, marchingCubes.cpp:505-553: (x,y,z),(x+1,y,z),(x+1,y+1,z),(x,y+1,z), then z+1 */
static const int NBC[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

/* Optional outputs of the hull for the interfacial elements: the distinct neighbour
 * lists in first-seen order (insertNeighborList, marchingCubes.cpp:605-618), and per
 * triangle its list key and barycenter (Triangle::computeBarycenter, triangle.h:12-18). */
typedef struct {
    uint32_t* lists; /* 8 per list */
    int nlists, caplists;
    int* key;
    double* bary;
    int ntri, captri;
} mc_out_t;

static int mc_list_index(mc_out_t* o, const uint32_t* nl) {
    for (int i = 0; i < o->nlists; i++)
        if (memcmp(o->lists + 8 * i, nl, 8 * sizeof(uint32_t)) == 0) return i;
    if (o->nlists == o->caplists) {
        o->caplists = o->caplists ? 2 * o->caplists : 32;
        o->lists = (uint32_t*)realloc(o->lists, sizeof(uint32_t) * 8 * o->caplists);
    }
    memcpy(o->lists + 8 * o->nlists, nl, 8 * sizeof(uint32_t));
    return o->nlists++;
}

static void mc_push_tri(mc_out_t* o, int key, v3 p0, v3 p1, v3 p2) {
    if (o->ntri == o->captri) {
        o->captri = o->captri ? 2 * o->captri : 256;
        o->key = (int*)realloc(o->key, sizeof(int) * o->captri);
        o->bary = (double*)realloc(o->bary, sizeof(double) * 3 * o->captri);
    }
    o->key[o->ntri] = key;
    o->bary[3 * o->ntri + 0] = (p0.x + p1.x + p2.x) / 3;
    o->bary[3 * o->ntri + 1] = (p0.y + p1.y + p2.y) / 3;
    o->bary[3 * o->ntri + 2] = (p0.z + p1.z + p2.z) / 3;
    o->ntri++;
}

static int64_t mc_core(const int32_t box6[6], const double* sdf, const uint32_t* idl, uint32_t own, double h,
                       double* volume_out, double* surface_out, uint32_t* nbrs, int* n_nbrs, int cap,
                       mc_out_t* col) {
    box_t b = box_from(box6);
    double volume = 0.0, surface = 0.0;
    int64_t ntri = 0;
    int nd = 0;
    for (int z = b.z0; z < b.z1 - 1; z++)
        for (int y = b.y0; y < b.y1 - 1; y++)
            for (int x = b.x0; x < b.x1 - 1; x++) {
                double val[8];
                unsigned ci = 0;
                for (int c = 0; c < 8; c++) {
                    val[c] = sdf[at(b, y + CORNER[c][1], x + CORNER[c][0], z + CORNER[c][2])];
                    if (val[c] >= 0) ci |= 1u << c;
                }
                int et = gg_mc_edge_table[ci];
                if (et == 0) continue;
                v3 vl[12];
                for (int e = 0; e < 12; e++) {
                    if (!(et & (1 << e))) continue;
                    int a = EDGE[e][0], c2 = EDGE[e][1];
                    v3 p1 = {x + CORNER[a][0], y + CORNER[a][1], z + CORNER[a][2]};
                    v3 p2 = {x + CORNER[c2][0], y + CORNER[c2][1], z + CORNER[c2][2]};
                    vl[e] = vinterp(p1, p2, val[a], val[c2]);
                }
                /* generateAdditionalInformation: sorted distinct IDs of the 8 corners */
                uint32_t lst[8];
                int cnt = 0;
                for (int c = 0; c < 8; c++) {
                    int xx = x + NBC[c][0], yy = y + NBC[c][1], zz = z + NBC[c][2];
                    uint32_t id = sdf[at(b, yy, xx, zz)] >= 0 ? own : idl[at(b, yy, xx, zz)];
                    int found = 0;
                    for (int q = 0; q < cnt; q++) if (lst[q] == id) { found = 1; break; }
                    if (!found) { /* insertDistinctInteger, marchingCubes.cpp:559-583 */
                        for (int q = 0; q < cnt; q++)
                            if (id < lst[q]) { uint32_t t = lst[q]; lst[q] = id; id = t; }
                        lst[cnt++] = id;
                    }
                }
                int key = -1;
                if (col) {
                    uint32_t nl[8];
                    for (int q = 0; q < 8; q++) nl[q] = q < cnt ? lst[q] : 0xFFFFFFFFu;
                    key = mc_list_index(col, nl);
                }
                for (int q = 0; q < cnt; q++) { /* recordNewGrains, marchingCubes.cpp:585-603 */
                    if (lst[q] == 0xFFFFFFFFu) continue;
                    int found = 0;
                    for (int r = 0; r < nd; r++) if (nbrs[r] == lst[q]) { found = 1; break; }
                    if (!found) { if (nd < cap) nbrs[nd] = lst[q]; nd++; }
                }
                for (int t = 0; gg_mc_tri_table[ci][t] != -1; t += 3) {
                    v3 p0 = vl[gg_mc_tri_table[ci][t]], p1 = vl[gg_mc_tri_table[ci][t + 1]],
                       p2 = vl[gg_mc_tri_table[ci][t + 2]];
                    /* computeGrainVolume, grainHull.cpp:42-51 */
                    double v321 = p2.x * p1.y * p0.z;
                    double v231 = p1.x * p2.y * p0.z;
                    double v312 = p2.x * p0.y * p1.z;
                    double v132 = p0.x * p2.y * p1.z;
                    double v213 = p1.x * p0.y * p2.z;
                    double v123 = p0.x * p1.y * p2.z;
                    volume += (double)(1.0f / 6.0f) * (-v321 + v231 + v312 - v132 - v213 + v123);
                    /* computeSurfaceArea, grainHull.cpp:122-127 */
                    double abx = p0.x - p1.x, aby = p0.y - p1.y, abz = p0.z - p1.z;
                    double bcx = p0.x - p2.x, bcy = p0.y - p2.y, bcz = p0.z - p2.z;
                    double cx = aby * bcz - abz * bcy, cy = abz * bcx - abx * bcz, cz = abx * bcy - aby * bcx;
                    surface += sqrt(cx * cx + (cy * cy + cz * cz)) / 2.0; /* Eigen's unrolled redux: c0 + (c1 + c2) */
                    if (col) mc_push_tri(col, key, p0, p1, p2);
                    ntri++;
                }
            }
    *volume_out = fabs(volume) * h * h * h;
    *surface_out = surface * h * h;
    *n_nbrs = nd;
    return ntri;
}

int64_t ggo_mc_box(const int32_t box6[6], const double* sdf, const uint32_t* idl, uint32_t own, double h,
                   double* volume_out, double* surface_out, uint32_t* nbrs, int* n_nbrs, int cap) {
    return mc_core(box6, sdf, idl, own, h, volume_out, surface_out, nbrs, n_nbrs, cap, NULL);
}

/* ------------------------------------------------------------------ */
/* Comparison: box.cpp:891-1088; set comparison: box.cpp:814-878.      */
/* ------------------------------------------------------------------ */
static void boundary_condition(box_t ib, box_t ob, double* out, box_t idb, uint32_t* idl, int m, int grid_blowup,
                               double h) {
    double distZMin, distZMax, distXMin, distXMax, distX, distYMin, distYMax, distY, distZ;
    double dist = 0; /* carried across voxels when no branch assigns it, box.cpp:1001 */
    for (int k = ib.z0; k < ib.z1; k++)
        for (int i = ib.y0; i < ib.y1; i++)
            for (int j = ib.x0; j < ib.x1; j++) {
                distXMax = (j - (m - 1 - grid_blowup));
                distYMax = (i - (m - 1 - grid_blowup));
                distZMax = (k - (m - 1 - grid_blowup));
                distXMin = -(j - grid_blowup + 1);
                distYMin = -(i - grid_blowup + 1);
                distZMin = -(k - grid_blowup + 1);
                distX = fabs(distXMin) < fabs(distXMax) ? distXMin : distXMax;
                distY = fabs(distYMin) < fabs(distYMax) ? distYMin : distYMax;
                distZ = fabs(distZMin) < fabs(distZMax) ? distZMin : distZMax;
                if (distX > 0 && distY > 0 && distZ > 0)
                    dist = sqrt((double)distX * distX + distY * distY + distZ * distZ);
                else if (distX < 0 && distY < 0 && distZ < 0) {
                    dist = distX > distY ? distX : distY;
                    dist = dist > distZ ? dist : distZ;
                } else if (distX >= 0) {
                    if (distY < 0 && distZ < 0) dist = distX;
                    else if (distY < 0 && distZ >= 0) dist = sqrt((double)distX * distX + distZ * distZ);
                    else if (distY >= 0 && distZ < 0) dist = sqrt((double)distX * distX + distY * distY);
                } else if (distY >= 0) {
                    if (distZ < 0 && distX < 0) dist = distY;
                    else if (distX < 0 && distZ >= 0) dist = sqrt((double)distY * distY + distZ * distZ);
                } else if (distZ >= 0) {
                    if (distY < 0 && distX < 0) dist = distZ;
                } else if (distX == 0 || distY == 0 || distZ == 0)
                    dist = 0;
                if (dist > -grid_blowup)
                    if (dist * h > out[at(ob, i, j, k)]) {
                        out[at(ob, i, j, k)] = dist * h;
                        idl[at(idb, i, j, k)] = 0;
                    }
            }
}

/* LSbox::BoundaryIntersection, box.cpp:968-990 (BoundaryGrainTube pinned to 0) */
static int boundary_intersection(box_t ob, int M, int gb) {
    int lo = gb + 0, hi = M - gb - 0;
    if (ob.x0 > lo && ob.x1 < hi && ob.y0 > lo && ob.y1 < hi && ob.z0 > lo && ob.z1 < hi) return 0;
    return 1;
}

void ggo_compare_box(const int32_t box6[6], int K, const int32_t* nb_boxes, const uint32_t* nb_ids,
                     const double* const* nb_sdf, double* out, uint32_t* idl, int M, int border, double h) {
    box_t b = box_from(box6);
    size_t cnt = box_count(b);
    for (size_t q = 0; q < cnt; q++) out[q] = -1.0;
    for (int n = 0; n < K; n++) {
        box_t nb = box_from(nb_boxes + 6 * n);
        int x0 = b.x0 < nb.x0 ? nb.x0 : b.x0, x1 = b.x1 > nb.x1 ? nb.x1 : b.x1;
        int y0 = b.y0 < nb.y0 ? nb.y0 : b.y0, y1 = b.y1 > nb.y1 ? nb.y1 : b.y1;
        int z0 = b.z0 < nb.z0 ? nb.z0 : b.z0, z1 = b.z1 > nb.z1 ? nb.z1 : b.z1;
        for (int k = z0; k < z1; k++)
            for (int i = y0; i < y1; i++)
                for (int j = x0; j < x1; j++) {
                    double dist = nb_sdf[n][at(nb, i, j, k)];
                    size_t q = at(b, i, j, k);
                    if (dist > out[q]) { out[q] = dist; idl[q] = nb_ids[n]; }
                }
    }
    if (boundary_intersection(b, M, border)) boundary_condition(b, b, out, b, idl, M, border, h);
}

void ggo_set_compare_box(const int32_t box6[6], const double* in, double* out, double delta, int M, int border,
                         int32_t newbox[6]) {
    box_t b = box_from(box6);
    int nx0 = b.x1, nx1 = b.x0, ny0 = b.y1, ny1 = b.y0, nz0 = b.z1, nz1 = b.z0;
    for (int k = b.z0; k < b.z1; k++)
        for (int i = b.y0; i < b.y1; i++)
            for (int j = b.x0; j < b.x1; j++) {
                size_t q = at(b, i, j, k);
                if (fabs(in[q]) < 0.7 * delta) out[q] = 0.5 * (in[q] - out[q]);
                else out[q] = in[q];
                if (out[q] >= 0) {
                    if (i < ny0) ny0 = i;
                    if (i > ny1) ny1 = i;
                    if (j < nx0) nx0 = j;
                    if (j > nx1) nx1 = j;
                    if (k < nz0) nz0 = k;
                    if (k > nz1) nz1 = k;
                }
            }
    nx0 -= border; nx1 += border; ny0 -= border; ny1 += border; nz0 -= border; nz1 += border;
    if (nx0 < 0) nx0 = 0;
    if (ny0 < 0) ny0 = 0;
    if (nz0 < 0) nz0 = 0;
    if (nx1 >= M) nx1 = M - 1;
    if (ny1 >= M) ny1 = M - 1;
    if (nz1 >= M) nz1 = M - 1;
    newbox[0] = nx0; newbox[1] = nx1; newbox[2] = ny0; newbox[3] = ny1; newbox[4] = nz0; newbox[5] = nz1;
}

/* ------------------------------------------------------------------ */
/* Whole loop                                                           */
/* ------------------------------------------------------------------ */
typedef struct {
    int present;   /* grains[id] != NULL */
    int exists;    /* m_exists */
    buf_t in, out; /* m_inputDistance / m_outputDistance (swapped by switchInNOut) */
    buf_t idl;     /* m_IDLocal */
    uint32_t *cmp, *son; /* m_comparisonList, m_secondOrderNeighbours */
    int ncmp, nson, capcmp, capson;
    int32_t newbox[6];
    double volume, surface;
    uint32_t* nb;
    int nnb, capnb;
    hull_t hull;   /* interfacial elements of the last hull (m_explicitHull) */
} grain_t;

struct ggo_sim {
    int N, gb, M, G, loop;
    double h, delta, dt, time_step;
    grain_t* g; /* index 0 = boundary grain (never processed) */
    int64_t last_voxels;
    /* convolution correction (box.cpp:426-539) */
    int correction, use_see;
    gbphys_t ph;
    quat_t* quats;  /* G + 1, [0] = boundary grain (0, 35 deg, 0), grainhdl.cpp:86 */
    double* see;    /* m_StoredElasticEnergy, G + 1; the boundary grain's is pinned to 0 */
    mc_out_t mc;    /* scratch of the hull extraction */
};

static void push(uint32_t** v, int* n, int* cap, uint32_t x) {
    if (*n == *cap) { *cap = *cap ? 2 * *cap : 16; *v = (uint32_t*)realloc(*v, sizeof(uint32_t) * *cap); }
    (*v)[(*n)++] = x;
}

ggo_sim* ggo_create(int N, int border, double time_step, int n_grains) {
    ggo_sim* s = (ggo_sim*)calloc(1, sizeof(ggo_sim));
    s->N = N; s->gb = border; s->M = N + 2 * border; s->G = n_grains; s->loop = 0;
    s->time_step = time_step;
    s->dt = time_step / (double)(N * N);            /* grainhdl.cpp:1431 */
    s->delta = (double)border / (double)N;           /* grainhdl.cpp:1439 */
    s->h = 1 / (double)N;                            /* grainhdl.h:182 */
    s->g = (grain_t*)calloc((size_t)n_grains + 1, sizeof(grain_t));
    s->quats = (quat_t*)calloc((size_t)n_grains + 1, sizeof(quat_t));
    s->see = (double*)calloc((size_t)n_grains + 1, sizeof(double));
    const double bnd[3] = {0, 35 * (3.14159265358979323846 / 180), 0};
    for (int i = 0; i <= n_grains; i++) s->quats[i] = ggo_euler_to_quat(bnd);
    s->ph.unique_gb = 1;
    s->ph.mobility_model = 0;
    s->ph.tl_drag = 0.0;
    s->ph.ds = 1 / (double)N;
    s->ph.quats = s->quats;
    for (int i = 0; i <= n_grains; i++) {
        s->g[i].in.esz = s->g[i].out.esz = sizeof(double);
        s->g[i].idl.esz = sizeof(uint32_t);
    }
    return s;
}

void ggo_destroy(ggo_sim* s) {
    if (!s) return;
    for (int i = 0; i <= s->G; i++) {
        free(s->g[i].in.v); free(s->g[i].out.v); free(s->g[i].idl.v);
        free(s->g[i].cmp); free(s->g[i].son); free(s->g[i].nb);
        ggo_hull_free(&s->g[i].hull);
    }
    free(s->g);
    free(s->quats);
    free(s->see);
    free(s->mc.lists); free(s->mc.key); free(s->mc.bary);
    free(s);
}

int ggo_load(ggo_sim* s, const uint32_t* labels, const int32_t* ext, const int64_t* counts) {
    const int N = s->N, gb = s->gb, M = s->M;
    for (int id = 1; id <= s->G; id++) {
        grain_t* G = &s->g[id];
        if (counts[id - 1] == 0) { G->present = 0; continue; } /* grainhdl.cpp:492-497 */
        const int32_t* e = ext + 6 * (id - 1);
        /* LSSbox mode-4 constructor, box.cpp:239-304 */
        int xmin = e[0], xmax = e[1], ymin = e[2], ymax = e[3], zmin = e[4], zmax = e[5];
        xmax += 2 * gb; ymax += 2 * gb; zmax += 2 * gb;
        if (ymax > M) ymax = M;
        if (xmax > M) xmax = M;
        if (zmax > M) zmax = M;
        if (ymin < 0) ymin = 0;
        if (xmin < 0) xmin = 0;
        if (zmin < 0) zmin = 0;
        box_t b = {xmin, xmax, ymin, ymax, zmin, zmax};
        b = resize_to_cube(b, M);
        G->present = 1; G->exists = 1;
        buf_resize(&G->in, b);
        buf_resize(&G->out, b);
        buf_resize(&G->idl, b);
        /* calculateDistanceFunction, box.cpp:374-397 */
        const double h = s->h;
        int lo = gb, hi = M - gb - 1;
        for (int k = b.z0; k < b.z1; k++)
            for (int i = b.y0; i < b.y1; i++)
                for (int j = b.x0; j < b.x1; j++) {
                    double v;
                    if (i < lo || i > hi || j < lo || j > hi || k < lo || k > hi) v = -h;
                    else {
                        uint32_t lab = labels[((size_t)(k - gb) * N + (i - gb)) * N + (j - gb)];
                        v = (lab == (uint32_t)id) ? h : -h;
                    }
                    D(&G->in)[at(b, i, j, k)] = v;
                }
        redistance(G->in.b, D(&G->in), G->out.b, D(&G->out), G->out.size, h, s->delta);
        buf_resize(&G->in, G->out.b);
    }
    return 0;
}

static int boxes_touch(box_t a, box_t b) { /* inclusive overlap, as LSbox::checkIntersection */
    return !(a.x0 > b.x1 || a.x1 < b.x0 || a.y0 > b.y1 || a.y1 < b.y0 || a.z0 > b.z1 || a.z1 < b.z0);
}

int ggo_set_lists(ggo_sim* s, const int64_t* off, const uint32_t* ids) {
    for (int id = 1; id <= s->G; id++) {
        grain_t* G = &s->g[id];
        G->nson = 0;
        for (int64_t q = off[id]; q < off[id + 1]; q++) push(&G->son, &G->nson, &G->capson, ids[q]);
    }
    return 0;
}

int ggo_default_lists(ggo_sim* s) {
    for (int a = 1; a <= s->G; a++) {
        grain_t* A = &s->g[a];
        A->nson = 0;
        if (!A->present || !A->exists) continue;
        for (int b = 1; b <= s->G; b++) {
            if (b == a || !s->g[b].present || !s->g[b].exists) continue;
            if (boxes_touch(A->out.b, s->g[b].out.b)) push(&A->son, &A->nson, &A->capson, (uint32_t)b);
        }
    }
    return 0;
}

static void switch_in_out(grain_t* G) { buf_t t = G->in; G->in = G->out; G->out = t; }

/* LSbox::computeSecondOrderNeighbours, box.cpp:1090-1134 */
static void update_lists(ggo_sim* s, int id, uint32_t** cand, int* ncand, int* capcand) {
    grain_t* A = &s->g[id];
    if (!A->exists) return;
    A->ncmp = 0;
    *ncand = 0;
    for (int i = 0; i < A->nson; i++) {
        grain_t* C = &s->g[A->son[i]];
        if (C->exists) push(&A->cmp, &A->ncmp, &A->capcmp, A->son[i]);
        for (int j = 0; j < C->nson; j++) {
            grain_t* H = &s->g[C->son[j]];
            if (H->exists && boxes_touch(A->in.b, H->in.b)) push(cand, ncand, capcand, C->son[j]);
        }
    }
    for (int i = 0; i < *ncand; i++) {
        uint32_t c = (*cand)[i];
        if (c == (uint32_t)id || c == 0) continue;
        int just_in = 0;
        for (int j = 0; j < A->ncmp; j++) if (A->cmp[j] == c) { just_in = 1; break; }
        if (!just_in) push(&A->cmp, &A->ncmp, &A->capcmp, c);
    }
}

/* The convolution correction of LSbox::executeConvolution (box.cpp:426-535): every
 * voxel of the output box with |input| < delta moves by the energy x mobility of the
 * nearest interfacial element towards its IDLocal neighbour, minus the stored-energy
 * difference when UseStoredElasticEnergy is on.  The point is Vector3d(i, j, k), i.e.
 * (y, x, z), while the barycenters are (x, y, z) (sic). */
static void convolution_correction(ggo_sim* s, int id) {
    grain_t* A = &s->g[id];
    const box_t ob = A->out.b;
    const double delta = s->delta;
    const double ts = 1 / 1.21; /* TimeSlope, grainhdl.cpp:1432 */
    for (int k = ob.z0; k < ob.z1; k++)
        for (int i = ob.y0; i < ob.y1; i++)
            for (int j = ob.x0; j < ob.x1; j++) {
                const double val = D(&A->in)[at(A->in.b, i, j, k)];
                if (!(fabs(val) < delta)) continue;
                const double point[3] = {(double)i, (double)j, (double)k};
                const uint32_t nb = U(&A->idl)[at(A->idl.b, i, j, k)];
                double fe, fm;
                ggo_hull_project(&A->hull, point, nb, &fe, &fm);
                const size_t q = at(ob, i, j, k);
                D(&A->out)[q] = val + (D(&A->out)[q] - val) * fe * fm * 1.0;
                if (s->use_see) {
                    double f = 0;
                    const int alive = nb == 0 || (nb <= (uint32_t)s->G && s->g[nb].present);
                    if (alive) f = (s->see[id] - s->see[nb]) * fm * s->dt / (ts * ts);
                    D(&A->out)[q] = D(&A->out)[q] - f;
                }
            }
}

void ggo_set_physics(ggo_sim* s, int correction, int unique_gb_energies, int mobility_model, double triple_line_drag,
                     int use_stored_energy) {
    s->correction = correction;
    s->ph.unique_gb = unique_gb_energies;
    s->ph.mobility_model = mobility_model;
    s->ph.tl_drag = triple_line_drag;
    s->use_see = use_stored_energy;
}

void ggo_set_orientations(ggo_sim* s, const double* euler) {
    for (int g = 1; g <= s->G; g++) s->quats[g] = ggo_euler_to_quat(euler + 3 * g);
}

void ggo_set_stored_energy(ggo_sim* s, const double* see) {
    for (int g = 1; g <= s->G; g++) s->see[g] = see[g];
}

int ggo_grain_elements(const ggo_sim* s, int id, int counts[4]) {
    if (id < 1 || id > s->G) return -1;
    const hull_t* H = &s->g[id].hull;
    counts[0] = H->gb.n;
    counts[1] = H->tl.n;
    counts[2] = H->qj.n;
    counts[3] = H->hj.n;
    return 0;
}

int ggo_step(ggo_sim* s) {
    const int G = s->G, M = s->M, gb = s->gb;
    const double h = s->h, delta = s->delta;
    /* 1. gridCoarsement (off) -> switchDistancebuffer, grainhdl.cpp:1496 */
    for (int id = 1; id <= G; id++) if (s->g[id].present) switch_in_out(&s->g[id]);
    /* 2. convolution, grainhdl.cpp:621-652 / box.cpp:414-539 */
    s->last_voxels = 0;
    for (int id = 1; id <= G; id++) {
        grain_t* A = &s->g[id];
        if (!A->present || !A->exists) continue;
        int n = A->out.b.x1 - A->out.b.x0;
        ggo_convolve_box(n, s->N, s->time_step, D(&A->in), D(&A->out));
        s->last_voxels += (int64_t)n * n * n;
        buf_resize(&A->idl, A->out.b); /* resizeIDLocalToDistanceBuffer, box.cpp:426 */
        if (s->correction && s->loop != 0) convolution_correction(s, id);
    }
    /* 3. switchDistancebuffer + updateSecondOrderNeighbors, grainhdl.cpp:852-853 */
    for (int id = 1; id <= G; id++) if (s->g[id].present) switch_in_out(&s->g[id]);
    uint32_t* cand = NULL;
    int ncand = 0, capcand = 0;
    for (int id = 1; id <= G; id++) if (s->g[id].present) update_lists(s, id, &cand, &ncand, &capcand);
    free(cand);
    /* 4. comparison_box, grainhdl.cpp:654-667 */
    for (int id = 1; id <= G; id++) {
        grain_t* A = &s->g[id];
        if (!A->present || !A->exists) continue;
        /* executeComparison, box.cpp:891-966 */
        size_t cnt = A->out.size;
        for (size_t q = 0; q < cnt; q++) D(&A->out)[q] = -1.0;
        A->nson = 0;
        for (int i = 0; i < A->ncmp; i++) push(&A->son, &A->nson, &A->capson, A->cmp[i]);
        box_t b = A->in.b;
        for (int n = 0; n < A->nson; n++) {
            grain_t* B = &s->g[A->son[n]];
            box_t nb = B->in.b;
            int x0 = b.x0 < nb.x0 ? nb.x0 : b.x0, x1 = b.x1 > nb.x1 ? nb.x1 : b.x1;
            int y0 = b.y0 < nb.y0 ? nb.y0 : b.y0, y1 = b.y1 > nb.y1 ? nb.y1 : b.y1;
            int z0 = b.z0 < nb.z0 ? nb.z0 : b.z0, z1 = b.z1 > nb.z1 ? nb.z1 : b.z1;
            for (int k = z0; k < z1; k++)
                for (int i = y0; i < y1; i++)
                    for (int j = x0; j < x1; j++) {
                        double dist = D(&B->in)[at(nb, i, j, k)];
                        size_t qo = at(A->out.b, i, j, k);
                        if (dist > D(&A->out)[qo]) {
                            D(&A->out)[qo] = dist;
                            U(&A->idl)[at(A->idl.b, i, j, k)] = A->son[n];
                        }
                    }
        }
        if (boundary_intersection(A->out.b, M, gb))
            boundary_condition(A->in.b, A->out.b, D(&A->out), A->idl.b, U(&A->idl), M, gb, h);
        /* executeSetComparison, box.cpp:814-878 */
        ggo_set_compare_box((int32_t[6]){A->out.b.x0, A->out.b.x1, A->out.b.y0, A->out.b.y1, A->out.b.z0,
                                         A->out.b.z1},
                            D(&A->in), D(&A->out), delta, M, gb, A->newbox);
    }
    /* 5. switchDistancebuffer, grainhdl.cpp:865 */
    for (int id = 1; id <= G; id++) if (s->g[id].present) switch_in_out(&s->g[id]);
    /* 6. level_set, grainhdl.cpp:669-718 */
    for (int id = 1; id <= G; id++) {
        grain_t* A = &s->g[id];
        if (!A->present) continue;
        if (!A->exists) { A->present = 0; continue; } /* deleted, grainhdl.cpp:678-680 */
        /* extractContour, box.cpp:1144-1161 */
        int32_t ib[6] = {A->in.b.x0, A->in.b.x1, A->in.b.y0, A->in.b.y1, A->in.b.z0, A->in.b.z1};
        int cap = A->capnb < 64 ? 64 : A->capnb;
        for (;;) {
            if (A->capnb < cap) { A->nb = (uint32_t*)realloc(A->nb, sizeof(uint32_t) * cap); A->capnb = cap; }
            int nn = 0;
            s->mc.nlists = 0;
            s->mc.ntri = 0;
            int64_t ntri = mc_core(ib, D(&A->in), U(&A->idl), (uint32_t)id, h, &A->volume, &A->surface, A->nb,
                                   &nn, A->capnb, s->correction ? &s->mc : NULL);
            if (nn > A->capnb) { cap = nn; continue; }
            A->nnb = nn;
            A->exists = ntri > 0;
            break;
        }
        /* computeSurfaceElements, box.cpp:1175-1180 (only the correction reads them) */
        if (A->exists && s->correction)
            ggo_hull_build(&A->hull, (uint32_t)id, s->mc.nlists, s->mc.lists, s->mc.ntri, s->mc.bary, s->mc.key,
                           &s->ph);
        if (!A->exists) continue;
        box_t nb = {A->newbox[0], A->newbox[1], A->newbox[2], A->newbox[3], A->newbox[4], A->newbox[5]};
        buf_resize(&A->out, nb);
        buf_resize(&A->out, resize_to_cube(nb, M));
    }
    /* 7. redistancing, grainhdl.cpp:720-748 */
    for (int id = 1; id <= G; id++) {
        grain_t* A = &s->g[id];
        if (!A->present || !A->exists) continue;
        redistance(A->in.b, D(&A->in), A->out.b, D(&A->out), A->out.size, h, delta);
        buf_resize(&A->in, A->out.b);
    }
    /* 8. countGrains, grainhdl.cpp:936-943 */
    int count = 0;
    for (int id = 1; id <= G; id++) count += s->g[id].present;
    s->loop++;
    return count;
}

int ggo_loop(const ggo_sim* s) { return s->loop; }

int ggo_grain_info(const ggo_sim* s, int id, int* exists, int32_t box[6], double* volume, double* surface,
                   int* n_neighbors) {
    if (id < 1 || id > s->G) return -1;
    const grain_t* A = &s->g[id];
    *exists = A->present && A->exists;
    box_t b = A->out.b;
    box_to(b, box);
    *volume = A->volume;
    *surface = A->surface;
    *n_neighbors = A->nnb;
    return A->present;
}

int ggo_grain_neighbors(const ggo_sim* s, int id, uint32_t* out, int cap) {
    if (id < 1 || id > s->G) return -1;
    const grain_t* A = &s->g[id];
    for (int i = 0; i < A->nnb && i < cap; i++) out[i] = A->nb[i];
    return A->nnb;
}

int ggo_grain_list(const ggo_sim* s, int id, uint32_t* out, int cap) {
    if (id < 1 || id > s->G) return -1;
    const grain_t* A = &s->g[id];
    for (int i = 0; i < A->ncmp && i < cap; i++) out[i] = A->cmp[i];
    return A->ncmp;
}

int64_t ggo_grain_sdf(const ggo_sim* s, int id, int32_t box[6], double* out, int64_t cap) {
    if (id < 1 || id > s->G) return -1;
    const grain_t* A = &s->g[id];
    box_to(A->out.b, box);
    int64_t n = (int64_t)A->out.size;
    if (out) memcpy(out, A->out.v, sizeof(double) * (size_t)(n < cap ? n : cap));
    return n;
}

int64_t ggo_grain_idlocal(const ggo_sim* s, int id, int32_t box[6], uint32_t* out, int64_t cap) {
    if (id < 1 || id > s->G) return -1;
    const grain_t* A = &s->g[id];
    box_to(A->idl.b, box);
    int64_t n = (int64_t)A->idl.size;
    if (out) memcpy(out, A->idl.v, sizeof(uint32_t) * (size_t)(n < cap ? n : cap));
    return n;
}

int64_t ggo_last_voxels(const ggo_sim* s) { return s->last_voxels; }

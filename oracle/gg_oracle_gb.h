/*
 * gg_oracle_gb.h -- TEST INFRASTRUCTURE: interfacial elements of a grain hull and the
 * convolution correction's projection (CPU restatement; see gg_oracle_gb.c).
 */
#ifndef GG_ORACLE_GB_H
#define GG_ORACLE_GB_H

#include <stdint.h>

typedef struct {
    double q0, q1, q2, q3;
} quat_t;

typedef struct {
    int unique_gb;        /* Settings::UniqueGBEnergies */
    int mobility_model;   /* Settings::UseMobilityModel */
    double tl_drag;       /* Settings::TripleLineDrag */
    double ds;            /* grainhdl::get_ds() = 1 / realDomainSize */
    const quat_t* quats;  /* orientation of grain ID 0..G (0 = the boundary grain) */
} gbphys_t;

typedef struct {
    int type; /* 1 GB, 2 TL, 3 QJ, 4 HJ */
    int key;  /* neighbour-list key it was made from */
    uint32_t* ids;
    int nids, capids;
    double energy, mobility; /* m_energy, m_mobility */
    double pos[3];
    double* bary; /* 3 per triangle, in triangle order */
    int nb, capb;
} elem_t;

typedef struct {
    elem_t* e;
    int n, cap;
} elist_t;

typedef struct {
    elist_t hj, qj, tl, gb;
} hull_t;

quat_t ggo_euler_to_quat(const double euler[3]);
double ggo_misorientation(quat_t self, quat_t other);

/* The element mesh of one hull: nlists distinct neighbour lists (8 IDs each, first-seen
 * order = key), ntri triangle barycenters (3 doubles each) with their list keys. */
void ggo_hull_build(hull_t* H, uint32_t own, int nlists, const uint32_t* lists, int ntri, const double* bary,
                    const int* tri_key, const gbphys_t* ph);
void ggo_hull_free(hull_t* H);

/* GBInfo of the nearest element holding `id` (fields as the reference returns them). */
void ggo_hull_project(const hull_t* H, const double p[3], uint32_t id, double* f_energy, double* f_mobility);

#endif

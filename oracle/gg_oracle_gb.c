/*
 * gg_oracle_gb.c -- TEST INFRASTRUCTURE: CPU restatement of the interfacial-element
 * mesh of a grain hull and of the convolution correction's projection onto it.
 * Used only as the checker (tests/, smoke(), the CPU baseline); the product never
 * links it.
 *
 * Follows, statement by statement:
 *   myQuaternion::euler2Quaternion (myQuaternion.cpp:168-191), Inverse / operator*
 *   (myQuaternion.cpp:54-70), misorientationCubicQxQ (myQuaternion.cpp:309-367);
 *   LSbox::computeMisorientation (box.cpp:2704-2719);
 *   InterfacialElement::computeMobilityMisori / computeReadShockleyEnergy and the
 *   GrainBoundary / TripleLine / QuadrupleJunction / HighOrderJunction constructors,
 *   energies, mobilities, positions and merges (InterfacialElement.cpp:23-456);
 *   GrainHull::computeGrainBoundaryElements, subDivideTrianglesToInterfacialElements,
 *   computeJunctionPosition, mergeJunction, projectPointToGrainBoundary
 *   (grainHull.cpp:187-275, 483-531, 570-660); Triangle::computeBarycenter
 *   (triangle.h:12-18).
 */
#include "gg_oracle_gb.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GGO_PI 3.14159265358979323846 /* ggLS.h:25 */

quat_t ggo_euler_to_quat(const double e[3]) {
    const double p1 = e[0], t = e[1], p2 = e[2];
    const double co1 = cos(t / 2), s1 = sin(t / 2);
    quat_t q;
    q.q0 = co1 * cos((p1 + p2) / 2);
    q.q1 = s1 * cos((p1 - p2) / 2);
    q.q2 = s1 * sin((p1 - p2) / 2);
    q.q3 = co1 * sin((p1 + p2) / 2);
    return q;
}

/* (this)^-1 * p, then the smallest rotation angle over the 24 cubic symmetries */
static double misorientation_cubic(quat_t self, quat_t p) {
    const quat_t m = {self.q0, -self.q1, -self.q2, -self.q3}; /* Inverse */
    quat_t r;                                                  /* operator* */
    r.q0 = +m.q0 * p.q0 - m.q1 * p.q1 - m.q2 * p.q2 - m.q3 * p.q3;
    r.q1 = +m.q1 * p.q0 + m.q0 * p.q1 - m.q3 * p.q2 + m.q2 * p.q3;
    r.q2 = +m.q2 * p.q0 + m.q3 * p.q1 + m.q0 * p.q2 - m.q1 * p.q3;
    r.q3 = +m.q3 * p.q0 - m.q2 * p.q1 + m.q1 * p.q2 + m.q0 * p.q3;
    const double a = r.q0, b = r.q1, c = r.q2, d = r.q3;
    const double fac = 1.0 / sqrt(2.0);
    double r0[6][4];
    r0[0][0] = (a + b) * fac; r0[0][1] = (a - b) * fac; r0[0][2] = (c + d) * fac; r0[0][3] = (c - d) * fac;
    r0[1][0] = (a + c) * fac; r0[1][1] = (a - c) * fac; r0[1][2] = (b + d) * fac; r0[1][3] = (b - d) * fac;
    r0[2][0] = (a + d) * fac; r0[2][1] = (a - d) * fac; r0[2][2] = (b + c) * fac; r0[2][3] = (b - c) * fac;
    r0[3][0] = (a + b + c + d) * 0.5; r0[3][1] = (a + b - c - d) * 0.5;
    r0[3][2] = (a - b + c - d) * 0.5; r0[3][3] = (a - b - c + d) * 0.5;
    r0[4][0] = (a + b + c - d) * 0.5; r0[4][1] = (a + b - c + d) * 0.5;
    r0[4][2] = (a - b + c + d) * 0.5; r0[4][3] = (a - b - c - d) * 0.5;
    r0[5][0] = a; r0[5][1] = b; r0[5][2] = c; r0[5][3] = d;
    double omega = 0.0;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 4; j++)
            if (fabs(r0[i][j]) > omega) omega = fabs(r0[i][j]);
    if (omega > 1.0) omega = (double)(int)omega;
    omega = 2 * acos(omega);
    return omega;
}

double ggo_misorientation(quat_t self, quat_t p) {
    const double result = misorientation_cubic(self, p);
    if (result > 1 * GGO_PI / 180.0) return result;
    return 1 * GGO_PI / 180.0;
}

static double mobility_misori(const gbphys_t* ph, double misori) {
    if (ph->mobility_model == 0) return 1.0;
    const double mob = 1.0 - (0.99 * exp(-5. * (pow(misori / (15 * GGO_PI / 180), 9.))));
    return mob < 0.1 ? 0.1 : mob;
}

static double read_shockley(const gbphys_t* ph, double misori) {
    if (ph->unique_gb == 1) return 1.0;
    const double gamma_hagb = 1.0;
    const double theta_ref = 15 * GGO_PI / 180;
    if (misori > theta_ref) return gamma_hagb;
    return gamma_hagb * (misori / theta_ref) * (1.0 - log(misori / theta_ref));
}

static double misori_ids(const gbphys_t* ph, uint32_t a, uint32_t b) {
    return ggo_misorientation(ph->quats[a], ph->quats[b]);
}

/* TripleLine energy and mobility of (me, n0, n1), InterfacialElement.cpp:119-170 */
static void triple_line(const gbphys_t* ph, uint32_t me, uint32_t n0, uint32_t n1, double* energy,
                        double* mobility) {
    double avg = 0;
    avg += mobility_misori(ph, misori_ids(ph, me, n0));
    avg += mobility_misori(ph, misori_ids(ph, n0, n1));
    avg += mobility_misori(ph, misori_ids(ph, me, n1));
    avg /= 3;
    const double ds = 3 * sqrt(3 * ph->ds * ph->ds);
    *mobility = 1. / ((1. / (ds * ph->tl_drag)) + 1. / avg);
    double gamma[3];
    gamma[0] = read_shockley(ph, misori_ids(ph, me, n0));
    gamma[1] = read_shockley(ph, misori_ids(ph, n0, n1));
    gamma[2] = read_shockley(ph, misori_ids(ph, me, n1));
    double sigma = gamma[0] - gamma[1] + gamma[2];
    if (sigma < 0.01) sigma = 0.01;
    if (sigma > 1.0) sigma = 1.0;
    *energy = sigma;
}

static void push_id(elem_t* e, uint32_t id) {
    if (e->nids == e->capids) {
        e->capids = e->capids ? 2 * e->capids : 8;
        e->ids = (uint32_t*)realloc(e->ids, sizeof(uint32_t) * e->capids);
    }
    e->ids[e->nids++] = id;
}
static void push_bary(elem_t* e, const double* b) {
    if (e->nb == e->capb) {
        e->capb = e->capb ? 2 * e->capb : 16;
        e->bary = (double*)realloc(e->bary, sizeof(double) * 3 * e->capb);
    }
    memcpy(e->bary + 3 * e->nb, b, 3 * sizeof(double));
    e->nb++;
}
static elem_t* add_elem(elist_t* L) {
    if (L->n == L->cap) {
        L->cap = L->cap ? 2 * L->cap : 8;
        L->e = (elem_t*)realloc(L->e, sizeof(elem_t) * L->cap);
    }
    elem_t* e = &L->e[L->n++];
    memset(e, 0, sizeof(*e));
    return e;
}
static void free_elem(elem_t* e) { free(e->ids); free(e->bary); }
static void erase_elem(elist_t* L, int i) {
    free_elem(&L->e[i]);
    memmove(&L->e[i], &L->e[i + 1], sizeof(elem_t) * (L->n - i - 1));
    L->n--;
}

void ggo_hull_free(hull_t* H) {
    elist_t* lists[4] = {&H->hj, &H->qj, &H->tl, &H->gb};
    for (int t = 0; t < 4; t++) {
        for (int i = 0; i < lists[t]->n; i++) free_elem(&lists[t]->e[i]);
        free(lists[t]->e);
        lists[t]->e = NULL;
        lists[t]->n = lists[t]->cap = 0;
    }
}

/* Vector3d squaredNorm / norm of a - b: Eigen's unrolled redux, c0 + (c1 + c2) */
static double sqdist(const double* a, const double* b) {
    const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return d0 * d0 + (d1 * d1 + d2 * d2);
}

/* QuadrupleJunction / HighOrderJunction::computePosition */
static void junction_position(elem_t* e) {
    double p[3] = {0, 0, 0};
    for (int i = 0; i < e->nb; i++) {
        p[0] += e->bary[3 * i];
        p[1] += e->bary[3 * i + 1];
        p[2] += e->bary[3 * i + 2];
    }
    const double n = (double)e->nb;
    e->pos[0] = p[0] / n;
    e->pos[1] = p[1] / n;
    e->pos[2] = p[2] / n;
}

/* HighOrderJunction(A, B): A's three IDs, then those of B's that A already has (sic) */
static void hj_from_pair(elem_t* h, const elem_t* A, const elem_t* B) {
    h->type = 4;
    h->key = A->key;
    for (int i = 0; i < 3; i++) push_id(h, A->ids[i]);
    for (int i = 0; i < A->nb; i++) push_bary(h, A->bary + 3 * i);
    for (int i = 0; i < B->nb; i++) push_bary(h, B->bary + 3 * i);
    for (int b = 0; b < 3; b++) {
        int neighbor = 0;
        for (int i = 0; i < 3; i++)
            if (h->ids[i] == B->ids[b]) neighbor = 1;
        if (neighbor) push_id(h, B->ids[b]);
    }
    junction_position(h);
    h->energy = 1.0;
    h->mobility = 1.0;
}

/* HighOrderJunction::mergeWith: all of B's barycenters, then all of B's IDs (sic) */
static void hj_merge(elem_t* h, const elem_t* B) {
    for (int i = 0; i < B->nb; i++) push_bary(h, B->bary + 3 * i);
    for (int i = 0; i < B->nids; i++) push_id(h, B->ids[i]);
    junction_position(h);
    h->energy = 1.0;
    h->mobility = 1.0;
}

static int find_key(const elist_t* L, int key) {
    for (int i = 0; i < L->n; i++)
        if (L->e[i].key == key) return i;
    return -1;
}

void ggo_hull_build(hull_t* H, uint32_t own, int nlists, const uint32_t* lists, int ntri, const double* bary,
                    const int* tri_key, const gbphys_t* ph) {
    ggo_hull_free(H);
    /* computeGrainBoundaryElements: one element per distinct neighbour list, in key order */
    for (int key = 0; key < nlists; key++) {
        const uint32_t* nl = lists + 8 * key;
        int count = 0;
        for (int j = 0; j < 8; j++) count += nl[j] == 0xFFFFFFFFu ? 0 : 1;
        elem_t* e;
        switch (count) {
            case 2: {
                e = add_elem(&H->gb);
                e->type = 1;
                push_id(e, own != nl[0] ? nl[0] : nl[1]);
                const double m = misori_ids(ph, own, e->ids[0]);
                e->mobility = mobility_misori(ph, m);
                e->energy = read_shockley(ph, m);
                break;
            }
            case 3: {
                e = add_elem(&H->tl);
                e->type = 2;
                for (int i = 0; i < 3; i++)
                    if (own != nl[i]) push_id(e, nl[i]);
                triple_line(ph, own, e->ids[0], e->ids[1], &e->energy, &e->mobility);
                break;
            }
            case 4: {
                e = add_elem(&H->qj);
                e->type = 3;
                for (int i = 0; i < 4; i++)
                    if (own != nl[i]) push_id(e, nl[i]);
                double E1, M1, E2, M2, E3, M3;
                triple_line(ph, own, e->ids[0], e->ids[1], &E1, &M1);
                triple_line(ph, own, e->ids[1], e->ids[2], &E2, &M2);
                triple_line(ph, own, e->ids[0], e->ids[2], &E3, &M3);
                e->mobility = (M1 + M2 + M3) / 3.0;
                e->energy = (E1 + E2 + E3) / 3.0;
                break;
            }
            default: {
                e = add_elem(&H->hj);
                e->type = 4;
                for (int i = 0; i < count; i++)
                    if (own != nl[i]) push_id(e, nl[i]);
                e->mobility = 1.0;
                e->energy = 1.0;
                break;
            }
        }
        e->key = key;
    }
    /* subDivideTrianglesToInterfacialElements: barycenters in triangle order */
    for (int t = 0; t < ntri; t++) {
        const int key = tri_key[t];
        const uint32_t* nl = lists + 8 * key;
        int count = 0;
        for (int j = 0; j < 8; j++) count += nl[j] == 0xFFFFFFFFu ? 0 : 1;
        elist_t* L = count == 2 ? &H->gb : count == 3 ? &H->tl : count == 4 ? &H->qj : &H->hj;
        push_bary(&L->e[find_key(L, key)], bary + 3 * t);
    }
    /* computeJunctionPosition + mergeJunction */
    for (int i = 0; i < H->qj.n; i++) junction_position(&H->qj.e[i]);
    for (int i = 0; i < H->hj.n; i++) junction_position(&H->hj.e[i]);
    for (int i = 0; i < H->qj.n; i++) {
        for (int j = i + 1; j < H->qj.n; j++) {
            if (sqrt(sqdist(H->qj.e[i].pos, H->qj.e[j].pos)) < 2) {
                elem_t tmp;
                memset(&tmp, 0, sizeof(tmp));
                hj_from_pair(&tmp, &H->qj.e[i], &H->qj.e[j]);
                erase_elem(&H->qj, i);
                erase_elem(&H->qj, j - 1);
                i--;
                j--;
                *add_elem(&H->hj) = tmp;
                break;
            }
        }
    }
    for (int k = 0; k < H->hj.n; k++)
        for (int i = 0; i < H->qj.n; i++)
            if (sqrt(sqdist(H->qj.e[i].pos, H->hj.e[k].pos)) < 2) {
                hj_merge(&H->hj.e[k], &H->qj.e[i]);
                erase_elem(&H->qj, i);
                i--;
            }
    for (int i = 0; i < H->hj.n; i++)
        for (int k = i + 1; k < H->hj.n; k++)
            if (sqrt(sqdist(H->hj.e[i].pos, H->hj.e[k].pos)) < 2) {
                hj_merge(&H->hj.e[i], &H->hj.e[k]);
                erase_elem(&H->hj, k);
                k--;
            }
}

/* projectPointToGrainBoundary: nearest barycenter over the elements that hold `id`,
 * searched HJ, QJ, TL, GB with strict <.  Returns GBInfo(m_energy, m_mobility) through
 * the constructor GBInfo(_mobility, _energy): field energy = m_mobility, field mobility =
 * m_energy (InterfacialElement.h:24-35, 70-72). */
void ggo_hull_project(const hull_t* H, const double p[3], uint32_t id, double* f_energy, double* f_mobility) {
    double minimal = 10000000.0;
    double E = 1., Mo = 1.; /* GBInfo weight(1., 1.) */
    const elist_t* lists[4] = {&H->hj, &H->qj, &H->tl, &H->gb};
    const int nchk[4] = {-1, 3, 2, 1}; /* IDs compared: all for HJ, else the first 3, 2, 1 */
    for (int t = 0; t < 4; t++) {
        const elist_t* L = lists[t];
        for (int j = 0; j < L->n; j++) {
            const elem_t* e = &L->e[j];
            const int nc = nchk[t] < 0 ? e->nids : nchk[t];
            int found = 0;
            for (int i = 0; i < nc; i++)
                if (e->ids[i] == id) found = 1;
            if (!found) continue;
            for (int i = 0; i < e->nb; i++) {
                const double d = sqdist(p, e->bary + 3 * i);
                if (d < minimal) {
                    minimal = d;
                    E = e->energy;
                    Mo = e->mobility;
                }
            }
        }
    }
    *f_energy = Mo;
    *f_mobility = E;
}

/*
 * ref_hooks.cpp -- observation hooks for the compiled reference (TEST INFRASTRUCTURE).
 *
 * Linked into oracle/_ref/ggls_ref with `-Wl,--wrap=<symbol>` for LSbox methods
 * that grainhdl.cpp calls across translation units, so the reference sources are
 * compiled unmodified.  Each wrapper calls the real method and, when the
 * environment asks for it, appends binary records to a dump file:
 *
 *   GG_REF_DUMP=<path>          enable; records are appended to <path>
 *   GG_REF_DUMP_STATS=1         per-step per-grain records (STATS, NEIGHBORS, LIST)
 *                               plus the initial state (INIT_SDF, INIT_LIST)
 *   GG_REF_DUMP_GRAINS=a,b,...  grains whose box buffers are dumped around every
 *                               stage ("all" for every grain; default none)
 *   GG_REF_DUMP_LOOPS=a,b,...   timesteps for those buffer dumps (default all)
 *
 * One documented deviation from the reference's behaviour is made here:
 * grainhdl::BoundaryGrainTube (grainhdl.h:87) is never assigned by the reference
 * and lives in malloc'd memory, so its value is indeterminate; the wrapper of
 * grainhdl::initializeSimulation pins it to 0 before the simulation starts.
 *
 * Record layout (little endian): u32 magic 'GGDR', i32 kind, i32 loop, i32 grain,
 * i32 box[6] = {xmin,xmax,ymin,ymax,zmin,zmax}, i32 dtype (0 f64, 1 u32),
 * i64 count, then count elements.
 */
// Standard and third-party headers first, so that the access override below
// only touches the reference's own classes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <sys/time.h>
#include <omp.h>
#include "Eigen/Dense"

#define private public
#define protected public
#include "box.h"
#include "grainhdl.h"
#include "Settings.h"
#undef private
#undef protected

namespace {

enum Kind {
    K_INIT_SDF = 1, K_INIT_LIST = 2, K_STATS = 3, K_NEIGHBORS = 4, K_CONV_IN = 5, K_CONV_OUT = 6,
    K_LIST = 7, K_CMP_OUT = 8, K_CMP_ID = 9, K_SETCMP_OUT = 10, K_REDIST_IN = 11, K_REDIST_OUT = 12,
    K_MC_ID = 13, K_MC_IN = 14, K_LOOP_TIME = 15
};

struct Dumper {
    FILE* f = nullptr;
    bool stats = false;
    bool init = true;  // GG_REF_DUMP_INIT=0: no initial SDF and list records (large domains)
    bool all_grains = false;
    std::set<int> grains;
    bool all_loops = true;
    std::set<int> loops;
    std::mutex mu;

    static void parse_list(const char* s, bool& all, std::set<int>& out) {
        if (!s) return;
        if (std::strcmp(s, "all") == 0) { all = true; return; }
        all = false;
        std::string cur;
        for (const char* p = s;; ++p) {
            if (*p == ',' || *p == 0) {
                if (!cur.empty()) out.insert(std::atoi(cur.c_str()));
                cur.clear();
                if (*p == 0) break;
            } else {
                cur += *p;
            }
        }
    }

    Dumper() {
        const char* path = std::getenv("GG_REF_DUMP");
        if (!path) return;
        f = std::fopen(path, "wb");
        const char* st = std::getenv("GG_REF_DUMP_STATS");
        stats = st && st[0] == '1';
        const char* in = std::getenv("GG_REF_DUMP_INIT");
        init = !(in && in[0] == '0');
        parse_list(std::getenv("GG_REF_DUMP_GRAINS"), all_grains, grains);
        parse_list(std::getenv("GG_REF_DUMP_LOOPS"), all_loops, loops);
    }
    ~Dumper() { if (f) std::fclose(f); }

    bool want_buffers(int grain, int loop) const {
        if (!f) return false;
        if (!all_grains && grains.find(grain) == grains.end()) return false;
        return all_loops || loops.find(loop) != loops.end();
    }

    void write(int kind, int loop, int grain, const int box[6], int dtype, const void* data, int64_t count) {
        if (!f) return;
        std::lock_guard<std::mutex> lock(mu);
        uint32_t magic = 0x52444747u;  // "GGDR"
        int32_t hdr[10] = {kind, loop, grain, box[0], box[1], box[2], box[3], box[4], box[5], dtype};
        std::fwrite(&magic, 4, 1, f);
        std::fwrite(hdr, 4, 10, f);
        std::fwrite(&count, 8, 1, f);
        if (count > 0) std::fwrite(data, dtype == 0 ? 8 : 4, (size_t)count, f);
    }
};

Dumper& dumper() {
    static Dumper d;
    return d;
}

void box_of(DimensionalBufferReal* b, int box[6]) {
    box[0] = b->getMinX(); box[1] = b->getMaxX();
    box[2] = b->getMinY(); box[3] = b->getMaxY();
    box[4] = b->getMinZ(); box[5] = b->getMaxZ();
}

void dump_sdf(int kind, int loop, int grain, DimensionalBufferReal* b) {
    int box[6];
    box_of(b, box);
    dumper().write(kind, loop, grain, box, 0, b->getRawData(), (int64_t)b->m_values.size());
}

void dump_ids(int kind, int loop, int grain, DimensionalBufferIDLocal& ids) {
    int box[6] = {ids.getMinX(), ids.getMaxX(), ids.getMinY(), ids.getMaxY(), ids.getMinZ(), ids.getMaxZ()};
    std::vector<uint32_t> v(ids.m_values.size());
    for (size_t i = 0; i < v.size(); i++) v[i] = ids.m_values[i].grainID;
    dumper().write(kind, loop, grain, box, 1, v.data(), (int64_t)v.size());
}

void dump_list(int kind, int loop, int grain, const std::vector<unsigned int>& l) {
    int box[6] = {0, 0, 0, 0, 0, 0};
    dumper().write(kind, loop, grain, box, 1, l.data(), (int64_t)l.size());
}

int loop_of(LSbox* b) { return b->m_grainHandler->loop; }

// LOOP_TIME record: wall-clock seconds when the first grain of a loop iteration
// enters its convolution, i.e. when the iteration's convolution stage starts.
// Written whenever GG_REF_DUMP is set.
void stamp_loop(int loop) {
    static std::atomic<int> last(-1000);
    int prev = last.load();
    while (prev < loop) {
        if (last.compare_exchange_weak(prev, loop)) {
            timeval tv;
            gettimeofday(&tv, nullptr);
            double t = tv.tv_sec + tv.tv_usec * 1e-6;
            int box[6] = {0, 0, 0, 0, 0, 0};
            dumper().write(K_LOOP_TIME, loop, 0, box, 0, &t, 1);
            return;
        }
    }
}

}  // namespace

extern "C" {
void __real__ZN8grainhdl20initializeSimulationEv(grainhdl*);
void __real__ZN5LSbox23computeDirectNeighboursERK5RTreeIjiLi3EfLi8ELi4EE(LSbox*, const void*);
void __real__ZN5LSbox18executeConvolutionER15ExpandingVectorIcE(LSbox*, void*);
void __real__ZN5LSbox28computeSecondOrderNeighboursEv(LSbox*);
void __real__ZN5LSbox17executeComparisonEv(LSbox*);
void __real__ZN5LSbox20executeSetComparisonEv(LSbox*);
void __real__ZN5LSbox14extractContourEv(LSbox*);
void __real__ZN5LSbox19executeRedistancingEv(LSbox*);

void __wrap__ZN8grainhdl20initializeSimulationEv(grainhdl* self) {
    self->BoundaryGrainTube = 0.0;
    __real__ZN8grainhdl20initializeSimulationEv(self);
}

void __wrap__ZN5LSbox23computeDirectNeighboursERK5RTreeIjiLi3EfLi8ELi4EE(LSbox* self, const void* tree) {
    __real__ZN5LSbox23computeDirectNeighboursERK5RTreeIjiLi3EfLi8ELi4EE(self, tree);
    if (dumper().f && dumper().stats && dumper().init) {
        dump_sdf(K_INIT_SDF, -1, (int)self->m_ID, self->m_outputDistance);
        dump_list(K_INIT_LIST, -1, (int)self->m_ID, self->m_secondOrderNeighbours);
    }
}

void __wrap__ZN5LSbox18executeConvolutionER15ExpandingVectorIcE(LSbox* self, void* pool) {
    stamp_loop(loop_of(self));
    const bool w = self->m_exists && dumper().want_buffers((int)self->m_ID, loop_of(self));
    if (w) dump_sdf(K_CONV_IN, loop_of(self), (int)self->m_ID, self->m_inputDistance);
    __real__ZN5LSbox18executeConvolutionER15ExpandingVectorIcE(self, pool);
    if (w) dump_sdf(K_CONV_OUT, loop_of(self), (int)self->m_ID, self->m_outputDistance);
}

void __wrap__ZN5LSbox28computeSecondOrderNeighboursEv(LSbox* self) {
    __real__ZN5LSbox28computeSecondOrderNeighboursEv(self);
    if (dumper().f && dumper().stats && self->m_exists)
        dump_list(K_LIST, loop_of(self), (int)self->m_ID, self->m_comparisonList);
}

void __wrap__ZN5LSbox17executeComparisonEv(LSbox* self) {
    __real__ZN5LSbox17executeComparisonEv(self);
    if (self->m_exists && dumper().want_buffers((int)self->m_ID, loop_of(self))) {
        dump_sdf(K_CMP_OUT, loop_of(self), (int)self->m_ID, self->m_outputDistance);
        dump_ids(K_CMP_ID, loop_of(self), (int)self->m_ID, self->m_IDLocal);
    }
}

void __wrap__ZN5LSbox20executeSetComparisonEv(LSbox* self) {
    __real__ZN5LSbox20executeSetComparisonEv(self);
    if (self->m_exists && dumper().want_buffers((int)self->m_ID, loop_of(self))) {
        int box[6] = {self->m_newXMin, self->m_newXMax, self->m_newYMin, self->m_newYMax,
                      self->m_newZMin, self->m_newZMax};
        DimensionalBufferReal* b = self->m_outputDistance;
        dumper().write(K_SETCMP_OUT, loop_of(self), (int)self->m_ID, box, 0, b->getRawData(),
                       (int64_t)b->m_values.size());
    }
}

void __wrap__ZN5LSbox14extractContourEv(LSbox* self) {
    const int loop = loop_of(self);
    const bool w = dumper().want_buffers((int)self->m_ID, loop);
    if (w) {
        dump_sdf(K_MC_IN, loop, (int)self->m_ID, self->m_inputDistance);
        dump_ids(K_MC_ID, loop, (int)self->m_ID, self->m_IDLocal);
    }
    __real__ZN5LSbox14extractContourEv(self);
    if (dumper().f && dumper().stats) {
        int box[6];
        box_of(self->m_exists ? self->m_outputDistance : self->m_inputDistance, box);
        double st[3] = {self->m_exists ? 1.0 : 0.0, self->m_volume, self->m_surface};
        dumper().write(K_STATS, loop, (int)self->m_ID, box, 0, st, 3);
        if (self->m_exists) dump_list(K_NEIGHBORS, loop, (int)self->m_ID, self->m_explicitHull.getAllNeighbors());
    }
}

void __wrap__ZN5LSbox19executeRedistancingEv(LSbox* self) {
    const int loop = loop_of(self);
    const bool w = self->m_exists && dumper().want_buffers((int)self->m_ID, loop);
    if (w) dump_sdf(K_REDIST_IN, loop, (int)self->m_ID, self->m_inputDistance);
    __real__ZN5LSbox19executeRedistancingEv(self);
    if (w) dump_sdf(K_REDIST_OUT, loop, (int)self->m_ID, self->m_outputDistance);
}
}  // extern "C"

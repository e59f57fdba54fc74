/*
 * voro_stubs.cpp (oracle shim, TEST INFRASTRUCTURE) -- link stubs for the eight
 * voro++ symbols that the reference's mode-1 Voronoi generator references
 * (grainhdl.cpp:226-396, grahamScan.cpp:23).  The oracle only runs mode 4
 * (voxelised microstructure files), so none of them is ever called; each one
 * aborts with a message if it is.  The prebuilt voro++ library that ships with
 * the reference is neither opened nor linked.  The stubs are bound to the
 * mangled names directly, so no voro++ header is needed.
 */
#include <cstdio>
#include <cstdlib>

namespace {
[[noreturn]] void gg_no_voro() {
    std::fprintf(stderr, "voro++ is not linked into the oracle build (only MicrostructureGenMode=4 is supported)\n");
    std::abort();
}
}  // namespace

#define GG_VORO_STUB(fn, sym) \
    extern "C" void fn() __asm__(sym); \
    extern "C" void fn() { gg_no_voro(); }

GG_VORO_STUB(gg_voro_compute_cell, "_ZN4voro12voro_computeINS_9containerEE12compute_cellINS_20voronoicell_neighborEEEbRT_iiiii")
GG_VORO_STUB(gg_voro_container_base_dtor, "_ZN4voro14container_baseD2Ev")
GG_VORO_STUB(gg_voro_vertices, "_ZN4voro16voronoicell_base8verticesEdddRSt6vectorIdSaIdEE")
GG_VORO_STUB(gg_voro_cell_ctor, "_ZN4voro20voronoicell_neighborC1Ev")
GG_VORO_STUB(gg_voro_cell_dtor, "_ZN4voro20voronoicell_neighborD1Ev")
GG_VORO_STUB(gg_voro_find_cell, "_ZN4voro9container17find_voronoi_cellEdddRdS1_S1_Ri")
GG_VORO_STUB(gg_voro_put, "_ZN4voro9container3putEiddd")
GG_VORO_STUB(gg_voro_container_ctor, "_ZN4voro9containerC1Eddddddiiibbbi")

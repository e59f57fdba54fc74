"""Grid coarsening (grainhdl::gridCoarsement, grainhdl.cpp:1446-1498; LSbox::resizeGrid and
recalculateIDLocal, box.cpp:2595-2702) on the FP64 path against the compiled reference's
own run (tests/golden/coarsen.npz): 40^3, 150 Voronoi grains, border 5, GridCoarsement on
with gradient 0.99, 40 timesteps.  The reference re-grids twice (to 34 and then 33); every
loop's existence, boxes (on the current grid), volumes, surfaces and hull neighbours must
match bit for bit, and the grid size must follow the reference's.
"""
import os

import numpy as np
import pytest

from gragles_3d_b200 import microstructure as msgen

pytestmark = pytest.mark.gpu


def test_coarsening_fp64_matches_reference_golden(gpu):
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "coarsen.npz")))
    N, G, border = int(d["N"]), int(d["G"]), int(d["border"])
    assert len(d["coarse_loop"]) >= 2  # the case re-grids more than once
    ms = msgen.voronoi(N, G, seed=int(d["seed"]))
    ext, counts = ms.grain_extents()
    gh = gpu.GrainHandler(N, border, 0.2, G, precision=gpu.PRECISION_FP64, grid_coarsening=True,
                          coarsening_gradient=float(d["set_coarsening_gradient"]))
    gh.load(ms.labels, ext, counts)
    gh.set_lists(d["init_list_off"], d["init_list_ids"])
    nb_base = np.concatenate([[0], np.cumsum(d["nb_len"])])
    size = N
    events = dict(zip(d["coarse_loop"].tolist(), d["coarse_size"].tolist()))
    for s in range(d["exists"].shape[0]):
        gh.step()
        size = events.get(s, size)
        assert gh.domain_size == size, f"loop {s}: grid size {gh.domain_size}, reference {size}"
        st = gh.stats()
        nb_ids = d["nb_ids"][nb_base[s]:nb_base[s + 1]]
        for g in range(1, G + 1):
            assert bool(st.exists[g]) == bool(d["exists"][s, g]), f"loop {s} grain {g}: exists"
            if not st.exists[g]:
                continue
            assert tuple(st.boxes[g]) == tuple(d["box"][s, g]), f"loop {s} grain {g}: box"
            assert st.volume[g] == d["volume"][s, g], f"loop {s} grain {g}: volume"
            assert st.surface[g] == d["surface"][s, g], f"loop {s} grain {g}: surface"
            want = nb_ids[d["nb_off"][s][g]:d["nb_off"][s][g + 1]]
            assert np.array_equal(gh.neighbors(g), want), f"loop {s} grain {g}: neighbours"
    gh.close()


def test_coarsening_mixed_runs_and_regrids(gpu):
    """The mixed path re-grids at the same loops on the same case, and two loops after the
    first coarsening its per-grain volumes stay within 1e-3 of the FP64 path's (95% of the
    grains: a wall voxel's sign below FP32 resolution can move a wall grain's hull volume)."""
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "coarsen.npz")))
    N, G, border = int(d["N"]), int(d["G"]), int(d["border"])
    ms = msgen.voronoi(N, G, seed=int(d["seed"]))
    ext, counts = ms.grain_extents()
    hs = []
    for prec in (gpu.PRECISION_MIXED, gpu.PRECISION_FP64):
        gh = gpu.GrainHandler(N, border, 0.2, G, precision=prec, grid_coarsening=True,
                              coarsening_gradient=float(d["set_coarsening_gradient"]))
        gh.load(ms.labels, ext, counts)
        gh.set_lists(d["init_list_off"], d["init_list_ids"])
        hs.append(gh)
    first = int(d["coarse_loop"][0])
    for s in range(first + 2):
        for gh in hs:
            gh.step()
        assert hs[0].domain_size == hs[1].domain_size, f"loop {s}"
    assert hs[0].domain_size == int(d["coarse_size"][0])
    a, b = hs[0].stats(), hs[1].stats()
    both = a.exists & b.exists
    both[0] = False
    rel = np.abs(a.volume[both] - b.volume[both]) / b.volume[both]
    assert np.quantile(rel, 0.95) < 1e-3, np.quantile(rel, 0.95)
    for gh in hs:
        gh.close()

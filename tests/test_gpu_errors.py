"""Capacity errors of the device pool and the list rows, raised on the host side of the
C ABI and by the kernels' own checks (nothing faults: an over-capacity kernel skips
the access and sets an error bit that the host turns into a status code).

The reference has no such limits (its boxes, lists and hulls are std::vectors); the
device pool and the fixed-capacity rows here replace them, so running out is an error
the caller must see, with a message naming the capacity, and the context must still
answer read-back calls afterwards.
"""
import numpy as np
import pytest

from gragles_3d_b200 import microstructure as msgen

pytestmark = pytest.mark.gpu


def _case(N=40, G=60, seed=7):
    ms = msgen.voronoi(N, G, seed=seed)
    ext, counts = ms.grain_extents()
    return ms, ext, counts


def test_pool_smaller_than_the_initial_boxes(gpu):
    ms, ext, counts = _case()
    G = ms.n_grains
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64) as big:
        big.load(ms.labels, ext, counts)
        st = big.stats()
        need = sum((int(b[1] - b[0]) ** 3 + 31) // 32 * 32 for g, b in enumerate(st.boxes) if g and st.exists[g])
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64, pool_voxels=need - 32) as gh:
        with pytest.raises(gpu.GGError) as ei:
            gh.load(ms.labels, ext, counts)
        assert ei.value.code == gpu.GG_ERR_POOL_EXHAUSTED
        assert f"pool holds {need - 32}" in str(ei.value) and f"need {need} voxels" in str(ei.value)
    # exactly enough: loads and steps
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64, pool_voxels=need) as gh:
        gh.load(ms.labels, ext, counts)
        gh.default_lists()
        gh.step()
        assert gh.stats().exists[1:].any()


def test_hull_capacity_exhausted_in_the_loop(gpu):
    """The correction's hull capture holds hull_capacity triangles per grain; a hull
    with more stops the step with GG_ERR_POOL_EXHAUSTED, and nothing past the capture
    arrays is written (read-back still works)."""
    ms, ext, counts = _case()
    G = ms.n_grains
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64, correction=True, unique_energies=False,
                          mobility_model=True, hull_capacity=8) as gh:
        gh.load(ms.labels, ext, counts)
        gh.default_lists()
        gh.set_orientations(ms.euler)
        with pytest.raises(gpu.GGError) as ei:
            gh.step()
        assert ei.value.code == gpu.GG_ERR_POOL_EXHAUSTED
        assert "hull_capacity" in str(ei.value)
        st = gh.stats()
        assert st.exists.shape == (G + 1,)
        assert np.isfinite(st.volume).all()


def test_list_capacity_exhausted(gpu):
    """Comparison lists longer than list_capacity: refused by gg_set_lists on the host,
    and flagged by the device-built default lists."""
    ms, ext, counts = _case()
    G = ms.n_grains
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64) as ref:
        ref.load(ms.labels, ext, counts)
        ref.default_lists()
        lens = [len(ref.comparison_list(g)) for g in range(1, G + 1)]
    cap = max(lens) - 1
    assert cap > 0
    with gpu.GrainHandler(ms.n, 6, 0.2, G, precision=gpu.PRECISION_FP64, list_capacity=cap) as gh:
        gh.load(ms.labels, ext, counts)
        with pytest.raises(gpu.GGError) as ei:
            gh.default_lists()
        assert ei.value.code == gpu.GG_ERR_LIST_OVERFLOW
        assert "list capacity" in str(ei.value)
        assert gh.stats().exists[1:].any()
        # the same lists from the host are refused before anything is copied
        off = np.zeros(G + 2, np.int64)
        ids = np.concatenate([np.arange(1, n + 1, dtype=np.uint32) % G + 1 for n in lens])
        off[2:] = np.cumsum(lens)
        with pytest.raises(gpu.GGError) as ei:
            gh.set_lists(off, ids)
        assert ei.value.code == gpu.GG_ERR_LIST_OVERFLOW
        assert f"has {max(lens)} entries" in str(ei.value)

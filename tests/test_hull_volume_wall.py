"""The reference's hull volume (GrainHull::computeGrainVolume over the marching-cubes
triangles, grainHull.cpp:40-55, with VertexInterp's 1e-5 snapping, marchingCubes.cpp:
484-499) is not continuous in the field where a grain meets the domain wall: the
comparison leaves a plane of voxels within 1e-6 of zero there, and one of them changing
sign moves the volume by tens of voxels.  This bounds how far any other rounding of the
same flow (the mixed path's FP32 storage) can follow per-grain volumes of wall grains.
The fixture is one grain's field from the oracle (tests/golden/make_golden.py wall)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def wall():
    return dict(np.load(os.path.join(HERE, "golden", "wall.npz")))


def _volume(oracle, d, sdf):
    N = int(d["N"])
    return oracle.mc_box(tuple(int(v) for v in d["box"]), sdf, d["idlocal"], int(d["gid"]), 1.0 / N)[1] * N ** 3


def test_one_wall_voxel_sign_moves_the_volume(oracle, wall):
    sdf = wall["sdf"]
    z, y, x = (int(v) for v in wall["flip"])
    assert abs(sdf[z, y, x]) < 1e-8  # far below FP32 rounding of the field's O(0.1) values
    flipped = sdf.copy()
    flipped[z, y, x] = -flipped[z, y, x]
    assert abs(_volume(oracle, wall, flipped) - _volume(oracle, wall, sdf)) > 20.0  # voxels


def test_sign_preserving_rounding_keeps_the_volume(oracle, wall):
    sdf = wall["sdf"]
    base = _volume(oracle, wall, sdf)
    rng = np.random.default_rng(1)
    for _ in range(3):
        perturbed = sdf * (1.0 + rng.uniform(-1e-7, 1e-7, sdf.shape))  # no sign changes
        assert abs(_volume(oracle, wall, perturbed) - base) < 1e-4 * base
    # FP32 storage of the same field, where no voxel changes sign
    f32 = sdf.astype(np.float32).astype(np.float64)
    assert np.array_equal(np.sign(f32), np.sign(sdf))
    assert abs(_volume(oracle, wall, f32) - base) < 1e-4 * base

"""GPU parity of the analysis outputs against the compiled reference's own files
(tests/golden/analysis.npz, made by tests/golden/make_golden.py from the correction
case run on one thread with NeighborTracking on): Texture_<loop>.bin and
Faces_<loop>.bin every loop (grainhdl.cpp:750-790) and the voxel container every
second loop (grainhdl.cpp:1074-1123).  IDs, counts, flags and box centres are exact;
volumes, surfaces and face areas within 1e-9 relative (the element energies use CUDA's
acos/log/exp/pow, a few ULP from libm, which moves the FP64 fields by ~1e-13)."""
import os

import numpy as np
import pytest

from gragles_3d_b200 import microstructure as msgen

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "analysis.npz")


def _close(a, b, rel=1e-9):
    return np.all(np.abs(a - b) <= rel * np.maximum(np.abs(b), 1e-300))


def test_texture_faces_and_container_match_reference(gpu, tmp_path):
    d = dict(np.load(GOLD))
    N, G, border = int(d["N"]), int(d["G"]), int(d["border"])
    ms = msgen.voronoi(N, G, seed=int(d["seed"]))
    ext, counts = ms.grain_extents()
    gh = gpu.GrainHandler(N, border, 0.2, G, precision=gpu.PRECISION_FP64, correction=True,
                          unique_energies=bool(d["phys_unique_energies"]),
                          mobility_model=bool(d["phys_mobility_factor"]),
                          stored_energy=bool(d["phys_stored_energy"]),
                          triple_line_drag=float(d["phys_triple_line_drag"]))
    gh.load(ms.labels, ext, counts)
    gh.set_lists(d["init_list_off"], d["init_list_ids"])
    gh.set_orientations(d["euler"])
    gh.set_stored_energy(2.5e-10 * d["uds_stored_energy"] / 1.0 * 2.52e-4)
    t_off = np.concatenate([[0], np.cumsum(d["texture_len"])])
    f_off = np.concatenate([[0], np.cumsum(d["faces_len"])])
    cont_at = {int(l): i for i, l in enumerate(d["container_loops"])}
    gh.step()  # loop 0 writes the text form of the texture file
    for loop in range(1, int(d["steps"]) + 1):
        gh.step()
        want = d["texture"][t_off[loop - 1]:t_off[loop]]
        got = gh.texture()
        assert len(got) == len(want), f"loop {loop}: texture records"
        for f in ("id", "NeighbourCount", "intersectsBoundaryGrain", "x", "y", "z", "GBEnergy", "BulkEnergy"):
            assert np.array_equal(got[f], want[f]), f"loop {loop}: texture {f}"
        for f in ("phi1", "PHI", "phi2"):
            assert _close(got[f], want[f], 1e-12), f"loop {loop}: texture {f}"
        for f in ("volume", "surfaceArea"):
            assert _close(got[f], want[f]), f"loop {loop}: texture {f}"
        want_f = d["faces"][f_off[loop - 1]:f_off[loop]]
        got_f = gh.faces()
        assert np.array_equal(got_f["grainA"], want_f["grainA"]), f"loop {loop}: face owners"
        assert np.array_equal(got_f["grainB"], want_f["grainB"]), f"loop {loop}: face neighbours"
        assert _close(got_f["area"], want_f["area"]), f"loop {loop}: face areas"
        if loop in cont_at:
            got_c = gh.voxel_container()
            assert np.array_equal(got_c, d["container"][cont_at[loop]]), f"loop {loop}: voxel container"
    # the files, in the reference's names and layouts
    tex = gh.texture()
    path = msgen.write_texture(str(tmp_path), tex, 8)
    assert os.path.getsize(path) == len(tex) * 96
    gh.close()


def test_faces_without_the_correction(gpu):
    """keep_elements builds the elements (and the faces) on an isotropic run too; each
    face appears once, from its higher ID, with a positive area."""
    d = dict(np.load(GOLD))
    N, G, border = int(d["N"]), int(d["G"]), int(d["border"])
    ms = msgen.voronoi(N, G, seed=int(d["seed"]))
    ext, counts = ms.grain_extents()
    gh = gpu.GrainHandler(N, border, 0.2, G, precision=gpu.PRECISION_FP64, keep_elements=True)
    gh.load(ms.labels, ext, counts)
    gh.default_lists()
    for _ in range(3):
        gh.step()
    f = gh.faces()
    assert len(f) > 0 and np.all(f["grainA"] > f["grainB"]) and np.all(f["area"] > 0)
    gh.close()


def test_text_texture_and_saved_network_match_reference(gpu, tmp_path):
    """Texture_<loop>.ori and the saved network's Microstructure_<loop>.uds written from the
    device state equal the compiled reference's own files byte for byte (tests/golden/
    text.npz: the isotropic path, bit-exact), and the volume-energy file holds each
    voxel's grain's stored energy."""
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "text.npz")))
    N, G, border = int(d["N"]), int(d["G"]), int(d["border"])
    ms = msgen.voronoi(N, G, seed=int(d["seed"]))
    ext, counts = ms.grain_extents()
    gh = gpu.GrainHandler(N, border, 0.2, G, precision=gpu.PRECISION_FP64, keep_elements=True)
    gh.load(ms.labels, ext, counts)
    gh.set_lists(d["init_list_off"], d["init_list_ids"])
    gh.set_orientations(d["euler"])
    see = 2.5e-10 * d["uds_stored_energy"] / 1.0 * 2.52e-4  # box.cpp:232-233
    gh.set_stored_energy(see)
    gh.step()  # loop 0 writes no texture (grainhdl.cpp:751)
    uds_loops = d["uds_loops"].tolist()
    for loop in range(1, int(d["steps"]) + 1):
        gh.step()
        path = msgen.write_texture_text(str(tmp_path), gh.texture_text(), loop)
        with open(path) as f:
            assert f.read() == str(d["ori"][loop - 1]), f"Texture_{loop}.ori"
        if loop in uds_loops:
            labels = gh.voxel_container()
            uds, _, energy = msgen.write_network(str(tmp_path), loop, gh.network_rows(), labels, see=see)
            with open(uds) as f:
                assert f.read() == str(d["uds"][uds_loops.index(loop)]), f"Microstructure_{loop}.uds"
            e = np.fromfile(energy, "<f8")
            assert e.size == labels.size  # every voxel belongs to a grain or to the boundary grain
            want = np.where(labels.ravel() > 0, np.concatenate([[0.0], see])[labels.ravel()], 0.0)
            assert np.array_equal(e, want)
    gh.close()

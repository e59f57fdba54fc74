"""Generate the golden fixtures in tests/golden/ from the reference solver itself.

The reference (compiled from its own sources by `make -C oracle ref`, with the
specified DFT standing in for MKL) runs on seeded voxelised microstructures; the
observation hooks record the initial state and, every step, each grain's
existence, volume, surface, box, hull neighbours (first-seen order) and
comparison list, plus single-box buffers of one grain around every stage.
The "correction" case turns on the convolution correction (box.cpp:426-535) with
a mix of low-angle and random orientations, the mobility model, a weak
triple-line drag and stored elastic energies.

The "coarsen" case turns grid coarsening on (GridCoarsement=1, gradient 0.99), so the
grid shrinks several times within its 40 steps.

The "c1" case is the plain-method configuration (64^3, 200 grains, 50 timesteps) the
FP64 device path is pinned on at full length.

The "analysis" case reruns the correction case on one thread with the reference's
analysis outputs on: Texture and Faces records every loop and the voxel container.

The "text" case keeps the reference's text outputs: Texture_<loop>.ori and the saved
network's Microstructure_<loop>.uds.

The "wall" case keeps one grain's field where it meets the domain wall (from the
oracle restatement): the evidence that the reference's hull volume jumps when one
voxel within 1e-8 of zero changes sign.

    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gragles_3d_b200 import microstructure as msgen  # noqa: E402
import refdump  # noqa: E402

CASES = {
    # name: (N, grains, border, seed, steps, grain whose buffers are kept, loop of those buffers)
    "tiny": (32, 20, 5, 1032, 6, 14, 2),
    "vanish": (40, 150, 5, 1040, 40, 0, 0),
    "correction": (32, 30, 5, 2032, 8, 0, 0),
    # the plain-method configuration: 64^3, 200 Voronoi grains, 10-voxel border, 50 timesteps
    # (51 loop iterations, grainhdl.cpp:837); comparison lists kept for the last loop only
    "c1": (64, 200, 10, 1001, 50, 0, 0),
    # grid coarsening on (grainhdl.cpp:1446-1498): the grid shrinks whenever the grain count
    # falls below 0.99 of its count at the last coarsening
    "coarsen": (40, 150, 5, 1040, 40, 0, 0),
}
# parameters.xml settings of the cases beyond the defaults
SETTINGS = {"coarsen": dict(grid_coarsening=True, coarsening_gradient=0.99)}
# cases whose per-loop comparison lists are kept only for the final loop (fixture size)
LAST_LIST_ONLY = {"c1", "coarsen"}

# physics of the cases that run the convolution correction
PHYSICS = {
    "correction": dict(unique_energies=False, mobility_factor=True, stored_energy=True, triple_line_drag=20.0),
}


def textured(ms, seed):
    """70 % of the grains within a few degrees of one orientation (Read-Shockley
    energies and mobility factors well below 1), the rest random; log-normal
    stored energies."""
    G = ms.n_grains
    rng = np.random.default_rng(seed)
    low = rng.random(G) < 0.7
    ms.euler[:] = np.where(low[:, None], np.array([0.3, 0.5, 0.2]) + rng.normal(0, 0.08, (G, 3)),
                           np.stack([rng.uniform(0, 2 * np.pi, G), rng.uniform(0, np.pi, G),
                                     rng.uniform(0, 2 * np.pi, G)], 1))
    ms.stored_energy[:] = rng.lognormal(0, 0.5, G) * 1e5


def ragged(d: dict, G: int):
    off = np.zeros(G + 2, np.int64)
    vals = []
    for g in range(G + 1):
        v = d.get(g, np.zeros(0, np.uint32))
        vals.append(np.asarray(v, np.uint32))
        off[g + 1] = off[g] + len(v)
    return off, (np.concatenate(vals) if vals else np.zeros(0, np.uint32))


def make(name, N, G, border, seed, steps, keep_grain, keep_loop):
    ms = msgen.voronoi(N, G, seed=seed)
    phys = PHYSICS.get(name)
    if phys:
        textured(ms, seed)
    with tempfile.TemporaryDirectory() as d:
        msgen.write_mode4(ms, d)
        msgen.write_parameters(os.path.join(d, "parameters.xml"), n_grains=G, border=border, steps=steps,
                               correction=bool(phys), **(phys or {}), **SETTINGS.get(name, {}))
        res, timers = refdump.run_case(d, threads=4, grains=str(keep_grain) if keep_grain else None,
                                       loops=str(keep_loop) if keep_grain else None)
    out = {"N": N, "G": G, "border": border, "seed": seed, "steps": steps}
    for k, v in SETTINGS.get(name, {}).items():
        out["set_" + k] = v
    if SETTINGS.get(name, {}).get("grid_coarsening"):
        ev = np.array(timers["coarsening"], np.int64).reshape(-1, 2)
        out["coarse_loop"], out["coarse_size"] = ev[:, 0], ev[:, 1]
    if phys:
        out["euler"] = ms.euler.copy()
        out["uds_stored_energy"] = ms.stored_energy.copy()
        for k, v in phys.items():
            out["phys_" + k] = v
    out["init_list_off"], out["init_list_ids"] = ragged(res["init_list"], G)
    loops = sorted(res["stats"])
    S = len(loops)
    exists = np.zeros((S, G + 1), np.uint8)
    vol = np.zeros((S, G + 1))
    sur = np.zeros((S, G + 1))
    box = np.zeros((S, G + 1, 6), np.int32)
    nb_off, nb_ids, li_off, li_ids = [], [], [], []
    for s, loop in enumerate(loops):
        for g, (dat, b) in res["stats"][loop].items():
            exists[s, g] = dat[0] == 1.0
            vol[s, g], sur[s, g] = dat[1], dat[2]
            box[s, g] = b
        o, i = ragged(res["neighbors"].get(loop, {}), G)
        nb_off.append(o); nb_ids.append(i)
        keep = name not in LAST_LIST_ONLY or loop == loops[-1]
        o, i = ragged(res["lists"].get(loop, {}) if keep else {}, G)
        li_off.append(o); li_ids.append(i)
    out.update(exists=exists, volume=vol, surface=sur, box=box,
               nb_off=np.stack(nb_off), nb_ids=np.concatenate(nb_ids), nb_len=np.array([len(x) for x in nb_ids]),
               list_off=np.stack(li_off), list_ids=np.concatenate(li_ids),
               list_len=np.array([len(x) for x in li_ids]))
    if keep_grain:
        for (kind, loop, g), r in res["buffers"].items():
            out[f"buf_{kind}"] = r.data
            out[f"box_{kind}"] = np.array(r.box, np.int32)
        out["buf_grain"], out["buf_loop"] = keep_grain, keep_loop
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "ok", {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


# the reference's analysis output records (Structs.h: Face, TextureData)
TEXTURE_DTYPE = np.dtype([("volume", "<f8"), ("surfaceArea", "<f8"), ("GBEnergy", "<f8"), ("BulkEnergy", "<f8"),
                          ("phi1", "<f8"), ("PHI", "<f8"), ("phi2", "<f8"), ("x", "<f8"), ("y", "<f8"),
                          ("z", "<f8"), ("id", "<u4"), ("NeighbourCount", "<u4"),
                          ("intersectsBoundaryGrain", "<u4"), ("pad", "<u4")])
FACE_DTYPE = np.dtype([("area", "<f8"), ("grainA", "<u4"), ("grainB", "<u4")])


def make_analysis(N=32, G=30, border=5, seed=2032, steps=8, plot_every=2):
    """The correction case again, one thread (the voxel container's writer order), with
    NeighborTracking on (Texture_<loop>.bin, Faces_<loop>.bin every loop, grainhdl.cpp:
    750-790) and the voxel container every plot_every loops (grainhdl.cpp:1074-1123)."""
    ms = msgen.voronoi(N, G, seed=seed)
    textured(ms, seed)
    phys = PHYSICS["correction"]
    with tempfile.TemporaryDirectory() as d:
        msgen.write_mode4(ms, d)
        msgen.write_parameters(os.path.join(d, "parameters.xml"), n_grains=G, border=border, steps=steps,
                               correction=True, analysis_every=1, neighbor_tracking=True,
                               plot_interval=plot_every, **phys)
        res, _ = refdump.run_case(d, threads=1)
        out = {"N": N, "G": G, "border": border, "seed": seed, "steps": steps, "plot_every": plot_every,
               "euler": ms.euler.copy(), "uds_stored_energy": ms.stored_energy.copy()}
        for k, v in phys.items():
            out["phys_" + k] = v
        out["init_list_off"], out["init_list_ids"] = ragged(res["init_list"], G)
        tex, tex_len, faces, face_len, cont, cont_loops = [], [], [], [], [], []
        for loop in range(1, steps + 1):
            t = np.fromfile(os.path.join(d, f"Texture_{loop}.bin"), TEXTURE_DTYPE)
            f = np.fromfile(os.path.join(d, f"Faces_{loop}.bin"), FACE_DTYPE)
            tex.append(t); tex_len.append(len(t)); faces.append(f); face_len.append(len(f))
            path = os.path.join(d, f"Container_size_{N}_t_{loop}.raw")
            if os.path.exists(path):
                cont.append(np.fromfile(path, np.uint32).reshape(N, N, N)); cont_loops.append(loop)
    out.update(texture=np.concatenate(tex), texture_len=np.array(tex_len), faces=np.concatenate(faces),
               faces_len=np.array(face_len), container=np.stack(cont), container_loops=np.array(cont_loops))
    np.savez_compressed(os.path.join(HERE, "analysis.npz"), **out)
    print("analysis ok", {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


def make_text(N=32, G=30, border=5, seed=2032, steps=6, plot_every=2):
    """The reference's text outputs on the isotropic path (bit-exact on the device): the
    correction case's microstructure and stored energies, NeighborTracking off so that
    save_Texture writes Texture_<loop>.ori every loop (grainhdl.cpp:776-805), and
    saveNetworkAsVoxelContainer every plot_every loops (Microstructure_<loop>.uds and the
    container, grainhdl.cpp:1074-1123).  Stored energy stays off in the loop, so the
    reference's ContainerVolumeEnergy loop writes nothing."""
    ms = msgen.voronoi(N, G, seed=seed)
    textured(ms, seed)
    with tempfile.TemporaryDirectory() as d:
        msgen.write_mode4(ms, d)
        msgen.write_parameters(os.path.join(d, "parameters.xml"), n_grains=G, border=border, steps=steps,
                               analysis_every=1, neighbor_tracking=False, plot_interval=plot_every)
        res, _ = refdump.run_case(d, threads=1)
        out = {"N": N, "G": G, "border": border, "seed": seed, "steps": steps, "plot_every": plot_every,
               "euler": ms.euler.copy(), "uds_stored_energy": ms.stored_energy.copy()}
        out["init_list_off"], out["init_list_ids"] = ragged(res["init_list"], G)
        ori, uds, uds_loops = [], [], []
        for loop in range(1, steps + 1):
            with open(os.path.join(d, f"Texture_{loop}.ori")) as f:
                ori.append(f.read())
            path = os.path.join(d, f"Microstructure_{loop}.uds")
            if os.path.exists(path):
                with open(path) as f:
                    uds.append(f.read())
                uds_loops.append(loop)
                assert os.path.getsize(os.path.join(d, f"ContainerVolumeEnergy_size_{N}_t_{loop}.raw")) == 0
    out.update(ori=np.array(ori), uds=np.array(uds), uds_loops=np.array(uds_loops))
    np.savez_compressed(os.path.join(HERE, "text.npz"), **out)
    print("text ok", len(ori), uds_loops)


def make_wall(N=64, G=600, border=10, seed=2064, loops=19, gid=159):
    """One grain's field where it meets the domain wall, from the oracle restatement (bit-
    exact with the reference on the device path's parity cases): Voronoi 64^3 / 600 grains,
    random orientations, Read-Shockley energies, the mobility model and the correction,
    after `loops` loops.  Its wall plane holds voxels with |phi| < 1e-6; the fixture keeps
    the one whose sign change moves the reference's hull volume the most."""
    import pyoracle

    ms = msgen.voronoi(N, G, seed=seed)
    ext, cnt = ms.grain_extents()
    sim = pyoracle.OracleSim(N, border, 0.2, ms.labels, ext, cnt)
    sim.set_physics(True, unique_energies=False, mobility_model=True)
    sim.set_orientations(ms.euler)
    for _ in range(loops):
        sim.step()
    box, sdf = sim.sdf(gid)
    ibox, idl = sim.idlocal(gid)
    assert ibox == box
    h = 1.0 / N
    base = pyoracle.mc_box(box, sdf, idl, gid, h)[1]
    best, at = 0.0, None
    for z, y, x in np.argwhere(np.abs(sdf) < 1e-6):
        f = sdf.copy()
        f[z, y, x] = -f[z, y, x]
        d = abs(pyoracle.mc_box(box, f, idl, gid, h)[1] - base)
        if d > best:
            best, at = d, (int(z), int(y), int(x))
    np.savez_compressed(os.path.join(HERE, "wall.npz"), N=N, gid=gid, loops=loops, box=np.array(box, np.int32),
                        sdf=sdf, idlocal=idl, flip=np.array(at, np.int32))
    print("wall ok", box, at, best * N ** 3)


if __name__ == "__main__":
    only = sys.argv[1:]
    for name, args in CASES.items():
        if not only or name in only:
            make(name, *args)
    if not only or "analysis" in only:
        make_analysis()
    if not only or "text" in only:
        make_text()
    if not only or "wall" in only:
        make_wall()

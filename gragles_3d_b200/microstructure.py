"""Seeded synthetic microstructures in the reference's voxelised input format.

The reference reads a voxelised microstructure with ``MicrostructureGenMode=4``
(grainhdl.cpp:404-578): a ``Container.raw`` file of N^3 little-endian uint32
grain IDs, x fastest, then y, then z (grainhdl.cpp:534-557), plus a ``.uds``
text file with a 12-line header (line 2 = ID offset, lines 6-8 = NX, NY, NZ,
line 9 = number of grains, grainhdl.cpp:421-463) and one row per grain
``id x y z phi1 PHI phi2 xmin xmax ymin ymax zmin zmax count storedEnergy``
(grainhdl.cpp:484-490; extents are inclusive domain voxel indices).

Everything here is deterministic: a splitmix64 stream (seeded per config) drives
the seed points, orientations and energies, and each voxel (centre at
``index + 0.5``) belongs to the nearest seed (Voronoi) or the seed of smallest
power distance ``|x - s|^2 - r^2`` (Laguerre).  The same files feed the oracle
and the GPU path, so both start from byte-identical state.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """``count`` consecutive outputs of splitmix64 started at ``seed``."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = (np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)) & _MASK
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of splitmix64."""
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, count: int) -> np.ndarray:
    """Standard normals by Box-Muller from two splitmix64 streams."""
    u1 = uniform01(seed, count)
    u2 = uniform01(seed ^ 0x5DEECE66D, count)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


@dataclasses.dataclass
class Microstructure:
    """A labelled voxel domain plus per-grain attributes (IDs are 1..n_grains)."""

    labels: np.ndarray            # (N, N, N) uint32, [z][y][x]; 0 never occurs
    euler: np.ndarray             # (G, 3) Bunge angles, radians
    stored_energy: np.ndarray     # (G,) value written in the .uds column
    seeds: np.ndarray             # (G, 3) seed points (x, y, z), voxel units

    @property
    def n(self) -> int:
        return int(self.labels.shape[0])

    @property
    def n_grains(self) -> int:
        return int(self.euler.shape[0])

    def grain_extents(self):
        """Per grain (1..G): inclusive xmin,xmax,ymin,ymax,zmin,zmax and voxel count.

        Grains that own no voxel get count 0 (the reference skips them)."""
        G = self.n_grains
        lab = self.labels
        counts = np.bincount(lab.ravel(), minlength=G + 1)[1:].astype(np.int64)
        ext = np.zeros((G, 6), dtype=np.int64)
        z, y, x = np.indices(lab.shape, sparse=True)
        for axis, coord in ((0, x), (2, y), (4, z)):
            full = np.broadcast_to(coord, lab.shape).ravel()
            lo = np.full(G + 1, np.iinfo(np.int64).max, dtype=np.int64)
            hi = np.full(G + 1, -1, dtype=np.int64)
            np.minimum.at(lo, lab.ravel(), full)
            np.maximum.at(hi, lab.ravel(), full)
            ext[:, axis] = lo[1:]
            ext[:, axis + 1] = hi[1:]
        ext[counts == 0] = 0
        return ext, counts


def _uniform_orientations(seed: int, G: int) -> np.ndarray:
    """Uniformly random orientations (Haar measure) as Bunge Euler angles."""
    u = uniform01(seed, 3 * G).reshape(G, 3)
    phi1 = 2.0 * np.pi * u[:, 0]
    PHI = np.arccos(np.clip(2.0 * u[:, 1] - 1.0, -1.0, 1.0))
    phi2 = 2.0 * np.pi * u[:, 2]
    return np.stack([phi1, PHI, phi2], axis=1)


def _label_nearest(N: int, seeds: np.ndarray, weights: Optional[np.ndarray]) -> np.ndarray:
    """Label every voxel centre by its nearest seed (power distance if weighted)."""
    from scipy.spatial import cKDTree

    G = seeds.shape[0]
    labels = np.empty((N, N, N), dtype=np.uint32)
    ax = np.arange(N, dtype=np.float64) + 0.5
    yy, xx = np.meshgrid(ax, ax, indexing="ij")
    plane = np.stack([xx.ravel(), yy.ravel()], axis=1)
    if weights is None:
        tree = cKDTree(seeds)
        for z in range(N):
            pts = np.column_stack([plane, np.full(plane.shape[0], ax[z])])
            _, idx = tree.query(pts, k=1, workers=-1)
            labels[z] = (idx.astype(np.uint32) + 1).reshape(N, N)
        return labels
    # Laguerre: lift to 4D so that the power distance is a Euclidean distance,
    # |x-s|^2 - r^2 = |(x,0) - (s, sqrt(R^2 - r^2))|^2 - R^2.
    R2 = float(np.max(weights ** 2))
    lift = np.sqrt(np.maximum(R2 - weights ** 2, 0.0))
    tree = cKDTree(np.column_stack([seeds, lift]))
    for z in range(N):
        pts = np.column_stack([plane, np.full(plane.shape[0], ax[z]), np.zeros(plane.shape[0])])
        _, idx = tree.query(pts, k=1, workers=-1)
        labels[z] = (idx.astype(np.uint32) + 1).reshape(N, N)
    del G
    return labels


def voronoi(N: int, n_grains: int, seed: int) -> Microstructure:
    """Voronoi tessellation of ``n_grains`` uniform random seeds in an N^3 domain."""
    pts = uniform01(seed, 3 * n_grains).reshape(n_grains, 3) * N
    labels = _label_nearest(N, pts, None)
    return Microstructure(labels, _uniform_orientations(seed + 1, n_grains),
                          np.zeros(n_grains), pts)


def laguerre(N: int, n_grains: int, seed: int, sigma: float = 0.3) -> Microstructure:
    """Laguerre tessellation with lognormal radii (median 1, log-sd ``sigma``),
    scaled so that the mean cell volume is N^3 / n_grains."""
    pts = uniform01(seed, 3 * n_grains).reshape(n_grains, 3) * N
    r = np.exp(sigma * normal(seed + 2, n_grains))
    r *= (N ** 3 / n_grains * 3.0 / (4.0 * np.pi)) ** (1.0 / 3.0) / np.mean(r)
    labels = _label_nearest(N, pts, r)
    return Microstructure(labels, _uniform_orientations(seed + 1, n_grains),
                          np.zeros(n_grains), pts)


# Settings the reference turns the .uds stored-energy column into m_StoredElasticEnergy
# with (box.cpp:232-233): DislocEnPerM * column / HAGB_Energy * Physical_Domain_Size.
DISLOC_EN_PER_M, HAGB_ENERGY, PHYSICAL_DOMAIN_SIZE = 2.5e-10, 1.0, 2.52e-4


def stored_energy_of(column: np.ndarray) -> np.ndarray:
    """m_StoredElasticEnergy of each grain from its .uds column (box.cpp:232-233)."""
    return DISLOC_EN_PER_M * np.asarray(column, np.float64) / HAGB_ENERGY * PHYSICAL_DOMAIN_SIZE


def lognormal_stored_energy(ms: Microstructure, seed: int, sigma: float = 0.5, scale: float = 0.1) -> None:
    """Per-grain stored elastic energy scale * X, X ~ LogNormal(0, sigma), in units of the
    high-angle boundary energy (m_StoredElasticEnergy = scale * X * HAGB_Energy), written
    into the .uds column that the reference scales by DislocEnPerM / HAGB_Energy *
    Physical_Domain_Size (box.cpp:232-233)."""
    x = np.exp(sigma * normal(seed, ms.n_grains))
    ms.stored_energy[:] = scale * x * HAGB_ENERGY * HAGB_ENERGY / (DISLOC_EN_PER_M * PHYSICAL_DOMAIN_SIZE)


def with_nuclei(ms: Microstructure, seed: int, fraction: float = 0.05, rmin: float = 2.0,
                rmax: float = 3.0) -> Microstructure:
    """The microstructure plus round(fraction * G) spherical nuclei (radius uniform in
    [rmin, rmax] voxels, centres uniform in the domain, uniformly random orientations,
    zero stored energy) appended as grains G + 1, G + 2, ...: every voxel whose centre lies
    within a nucleus's radius takes its ID (later nuclei over earlier ones).  A parent grain
    the nuclei cover completely owns no voxel and is skipped by the reader."""
    N, G = ms.n, ms.n_grains
    K = int(round(fraction * G))
    centres = uniform01(seed, 3 * K).reshape(K, 3) * N
    radii = rmin + (rmax - rmin) * uniform01(seed + 1, K)
    labels = ms.labels.copy()
    for k in range(K):
        c, r = centres[k], radii[k]
        lo = np.maximum(np.floor(c - r - 0.5).astype(int), 0)
        hi = np.minimum(np.ceil(c + r + 0.5).astype(int), N)
        z, y, x = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                              indexing="ij")
        inside = (x + 0.5 - c[0]) ** 2 + (y + 0.5 - c[1]) ** 2 + (z + 0.5 - c[2]) ** 2 <= r * r
        labels[z[inside], y[inside], x[inside]] = G + 1 + k
    return Microstructure(labels, np.concatenate([ms.euler, _uniform_orientations(seed + 2, K)]),
                          np.concatenate([ms.stored_energy, np.zeros(K)]), np.concatenate([ms.seeds, centres]))


def c4(N: int = 384, n_grains: int = 100000, seed: int = 1004) -> Microstructure:
    """The stored-energy configuration: Voronoi grains with lognormal stored energy
    (sigma 0.5, 0.1 of the boundary energy) plus 5% nuclei of radius 2-3 voxels with none."""
    ms = voronoi(N, n_grains, seed)
    lognormal_stored_energy(ms, seed + 3)
    return with_nuclei(ms, seed + 4)


def write_mode4(ms: Microstructure, directory: str, raw_name: str = "Container.raw",
                uds_name: str = "Microstructure.uds", id_offset: int = 1) -> tuple[str, str]:
    """Write ``Container.raw`` + ``.uds`` in the layout grainhdl.cpp:404-578 reads."""
    os.makedirs(directory, exist_ok=True)
    raw_path = os.path.join(directory, raw_name)
    uds_path = os.path.join(directory, uds_name)
    (ms.labels.astype("<u4") + np.uint32(id_offset - 1)).tofile(raw_path)
    ext, counts = ms.grain_extents()
    N = ms.n
    lines = [
        "gg-b200 synthetic microstructure",
        f"ID_offset\t{id_offset}",
        "DX\t1", "DY\t1", "DZ\t1",
        f"NX\t{N}", f"NY\t{N}", f"NZ\t{N}",
        f"NumberOfGrains\t{ms.n_grains}",
        "", "",
        "id\tx\ty\tz\tphi1\tPHI\tphi2\txmin\txmax\tymin\tymax\tzmin\tzmax\tcount\tstoredEnergy",
    ]
    rows = []
    for g in range(ms.n_grains):
        sx, sy, sz = (int(v) for v in np.floor(ms.seeds[g]))
        e = ms.euler[g]
        x0, x1, y0, y1, z0, z1 = (int(v) for v in ext[g])
        rows.append(f"{g + id_offset}\t{sx}\t{sy}\t{sz}\t{e[0]:.17g}\t{e[1]:.17g}\t{e[2]:.17g}\t"
                    f"{x0}\t{x1}\t{y0}\t{y1}\t{z0}\t{z1}\t{int(counts[g])}\t{ms.stored_energy[g]:.17g}")
    with open(uds_path, "w") as f:
        f.write("\n".join(lines) + "\n")
        f.write("\n".join(rows) + "\n")
    return raw_path, uds_path


def write_parameters(path: str, *, n_grains: int, border: int = 10, steps: int = 10, time_step: float = 0.2,
                     raw_name: str = "Container.raw", uds_name: str = "Microstructure.uds",
                     breakup: int = 0, threads: int = 8, correction: bool = False,
                     unique_energies: bool = True, mobility_factor: bool = False,
                     stored_energy: bool = False, triple_line_drag: float = 1e6,
                     analysis_every: int = 1000000, neighbor_tracking: bool = False,
                     plot_interval: int = 1000000, grid_coarsening: bool = False,
                     coarsening_gradient: float = 0.95) -> None:
    """A ``parameters.xml`` for the reference (Settings.cpp:81-270) in mode 4.

    ``NumberOfParticles`` must already hold the grain count: the reference sizes
    its thread work lists from it (grainhdl.cpp:1300-1311) before the mode-4
    header overrides it (grainhdl.cpp:159-224)."""
    p = {
        "StartTime": 0, "NumberOfParticles": n_grains, "NumberOfPointsPerGrain": 10,
        "AnalysisTimestep": analysis_every, "NumberOfTimesteps": steps,
        "PlotInterval": plot_interval, "TimeStepSize": repr(float(time_step)),
        "BreakupNumber": breakup, "DiscreteSamplingRate": 25, "DomainBorderSize": border,
        "MicrostructureGenMode": 4, "ReadFromFilename": raw_name, "AdditionalFilename": uds_name,
        "HAGB_Energy": "1.", "HAGB_Mobility": "7.5e-14", "DislocEnPerM": "2.5e-10",
        "Physical_Domain_Size": "2.52e-4", "TripleLineDrag": repr(float(triple_line_drag)),
        "UseMobilityFactor": int(mobility_factor), "UseStoredElasticEnergy": int(stored_energy),
        "UseMagneticField": 0, "DisableConvolutionCorrection": int(not correction),
        "UseTexture": 0, "ExecuteInParallel": 1, "MaximumNumberOfThreads": threads,
        "GridCoarsement": int(grid_coarsening), "GridCoarsementGradient": repr(float(coarsening_gradient)),
        "ConvolutionMode": 2,
        "UniqueGBEnergies": int(unique_energies), "GrainScheduler": 0, "DecoupleGrains": 0,
        "NeighborTracking": int(neighbor_tracking), "StoreTaskDistribution": 0,
    }
    body = "\n".join(f"   <{k}>{v}</{k}>" for k, v in p.items())
    with open(path, "w") as f:
        f.write('<?xml version="1.0" encoding="utf-8"?>\n<Parameters>\n' + body + "\n</Parameters>\n")


def write_container(directory: str, labels: np.ndarray, loop: int) -> str:
    """The voxel container of a network (GrainHandler.voxel_container) as the reference's
    saveNetworkAsVoxelContainer names and writes it (grainhdl.cpp:1116-1123): raw uint32
    grain IDs, x fastest, in Container_size_<N>_t_<loop>.raw."""
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    path = os.path.join(directory, f"Container_size_{lab.shape[0]}_t_{int(loop)}.raw")
    lab.tofile(path)
    return path


def write_texture(directory: str, records: np.ndarray, loop: int) -> str:
    """Texture_<loop>.bin as save_Texture writes it with NeighborTracking on
    (grainhdl.cpp:753-771): the records of GrainHandler.texture(), back to back."""
    path = os.path.join(directory, f"Texture_{int(loop)}.bin")
    np.ascontiguousarray(records).tofile(path)
    return path


def write_faces(directory: str, records: np.ndarray, loop: int) -> str:
    """Faces_<loop>.bin (grainhdl.cpp:758-775): the records of GrainHandler.faces()."""
    path = os.path.join(directory, f"Faces_{int(loop)}.bin")
    np.ascontiguousarray(records).tofile(path)
    return path


def _cxx(v) -> str:
    """A value as the reference's ostream prints it (default precision: %g, 6 digits)."""
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return "%g" % float(v)


def write_texture_text(directory: str, rows: list, loop: int) -> str:
    """Texture_<loop>.ori as save_Texture writes it without NeighborTracking (grainhdl.cpp:
    776-805): tab-separated rows of GrainHandler.texture_text()."""
    path = os.path.join(directory, f"Texture_{int(loop)}.ori")
    with open(path, "w") as f:
        for r in rows:
            f.write("\t".join(_cxx(v) for v in r) + "\n")
    return path


def write_network(directory: str, loop: int, rows: list, labels: np.ndarray, see=None) -> list:
    """The saved network of saveNetworkAsVoxelContainer (grainhdl.cpp:1074-1154):
    Microstructure_<loop>.uds (rows of GrainHandler.network_rows(), no header, as the
    reference writes it), the voxel container, and ContainerVolumeEnergy_size_<N>_t_<loop>.raw.
    The energy file holds, for every voxel in [z][y][x] order whose grain is in the network
    (ID 0 = the boundary grain, stored energy 0), that grain's stored elastic energy as a
    double; with `see` None (UseStoredElasticEnergy off) it is empty.  The reference opens
    this file but writes the values to the container's file handle after closing it
    (grainhdl.cpp:1124-1147); here they go to the file it opened."""
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    n = lab.shape[0]
    uds = os.path.join(directory, f"Microstructure_{int(loop)}.uds")
    with open(uds, "w") as f:
        for r in rows:
            f.write("\t".join(_cxx(v) for v in r) + "\n")
    cont = write_container(directory, lab, loop)
    energy = os.path.join(directory, f"ContainerVolumeEnergy_size_{n}_t_{int(loop)}.raw")
    if see is None:
        open(energy, "wb").close()
    else:
        in_network = np.zeros(len(see) + 1, bool)
        in_network[0] = True  # getGrainByID(0) is the boundary grain
        for r in rows:
            in_network[int(r[0])] = True
        energy_of = np.zeros(len(see) + 1)
        energy_of[1:] = np.asarray(see, np.float64)
        ids = lab.ravel()
        np.ascontiguousarray(energy_of[ids[in_network[ids]]], "<f8").tofile(energy)
    return [uds, cont, energy]

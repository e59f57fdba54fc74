"""B200-native GraGLeS_3D level-set timestep.

Python mirror of the reference's ``grainhdl`` driver (grainhdl.cpp:821-943) on
top of the C ABI in ``include/gg_b200.h`` (``libgg_b200.so``, built in-tree by
``gragles_3d_b200.build``).  The library is required: there is no CPU path, and
loading fails loudly when the extension is missing.
"""
from __future__ import annotations

import ctypes as C
import math
import dataclasses
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgg_b200.so")

GG_OK = 0
GG_ERR_INVALID = -1
GG_ERR_CUDA = -2
GG_ERR_POOL_EXHAUSTED = -3
GG_ERR_LIST_OVERFLOW = -4
GG_ERR_UNSUPPORTED = -5
PRECISION_FP64 = 0
PRECISION_MIXED = 1

EXPORTED = [
    "gg_create", "gg_destroy", "gg_last_error", "gg_load_state", "gg_set_lists", "gg_default_lists", "gg_step",
    "gg_stage_convolution", "gg_stage_update_lists", "gg_stage_comparison", "gg_stage_level_set",
    "gg_stage_redistancing", "gg_get_grain_stats", "gg_get_neighbors", "gg_get_list", "gg_get_sdf",
    "gg_get_idlocal", "gg_grain_count", "gg_loop", "gg_convolve_boxes_f64", "gg_convolve_boxes_mixed",
    "gg_convolve_boxes_f64_noalloc", "gg_set_orientations", "gg_set_stored_energy", "gg_get_elements",
    "gg_voxel_container", "gg_get_faces", "gg_domain_size", "gg_rtree_lists", "gg_rtree_lists_from_boxes",
    "gg_launch_config",
]


class GGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gg error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("domain_size", C.c_int32), ("border", C.c_int32), ("time_step", C.c_double),
        ("n_grains", C.c_int32), ("precision", C.c_int32), ("disable_correction", C.c_int32),
        ("list_capacity", C.c_int32), ("pool_voxels", C.c_int64), ("device", C.c_int32),
        ("unique_gb_energies", C.c_int32), ("mobility_model", C.c_int32), ("use_stored_energy", C.c_int32),
        ("triple_line_drag", C.c_double), ("hull_capacity", C.c_int32), ("keep_elements", C.c_int32),
        ("grid_coarsening", C.c_int32), ("points_per_grain", C.c_int32), ("coarsening_gradient", C.c_double),
        ("autotune", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("loop", C.c_int32), ("grain_count", C.c_int32), ("live_grains", C.c_int32), ("kernel_launches", C.c_int32),
        ("voxel_updates", C.c_int64), ("ms_convolution", C.c_float), ("ms_lists", C.c_float),
        ("ms_comparison", C.c_float), ("ms_levelset", C.c_float), ("ms_redistancing", C.c_float),
        ("ms_total", C.c_float), ("ms_compare_kernel", C.c_float), ("compare_voxels", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libgg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m gragles_3d_b200.build`")
    L = C.CDLL(path)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.gg_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    L.gg_destroy.argtypes = [vp]
    L.gg_last_error.argtypes = [vp]
    L.gg_last_error.restype = C.c_char_p
    L.gg_load_state.argtypes = [vp, vp, vp, vp]
    L.gg_set_lists.argtypes = [vp, vp, vp]
    L.gg_default_lists.argtypes = [vp]
    L.gg_rtree_lists.argtypes = [vp]
    L.gg_launch_config.argtypes = [vp, vp]
    L.gg_rtree_lists_from_boxes.argtypes = [i32, vp, vp, vp, vp, i64]
    L.gg_rtree_lists_from_boxes.restype = i64
    L.gg_step.argtypes = [vp, C.POINTER(StepStats)]
    for s in ("gg_stage_convolution", "gg_stage_update_lists", "gg_stage_comparison", "gg_stage_level_set",
              "gg_stage_redistancing", "gg_grain_count", "gg_loop", "gg_domain_size"):
        getattr(L, s).argtypes = [vp]
    L.gg_get_grain_stats.argtypes = [vp, vp, vp, vp, vp, vp]
    L.gg_get_neighbors.argtypes = [vp, i32, vp, i32]
    L.gg_get_list.argtypes = [vp, i32, vp, i32]
    L.gg_get_sdf.argtypes = [vp, i32, i32, vp, vp, i64]
    L.gg_get_sdf.restype = i64
    L.gg_get_idlocal.argtypes = [vp, i32, vp, vp, i64]
    L.gg_get_idlocal.restype = i64
    L.gg_convolve_boxes_f64.argtypes = [vp, vp, vp, vp, i32, i32, C.c_double]
    L.gg_convolve_boxes_mixed.argtypes = [vp, vp, vp, vp, i32, i32, C.c_double]
    L.gg_set_orientations.argtypes = [vp, vp]
    L.gg_set_stored_energy.argtypes = [vp, vp]
    L.gg_get_elements.argtypes = [vp, i32, vp]
    L.gg_voxel_container.argtypes = [vp, vp]
    L.gg_get_faces.argtypes = [vp, vp, vp, vp, i64]
    L.gg_get_faces.restype = i64
    _lib = L
    return L


# the reference's analysis records (Structs.h: TextureData, Face), 8-byte aligned
TEXTURE_DTYPE = np.dtype([("volume", "<f8"), ("surfaceArea", "<f8"), ("GBEnergy", "<f8"), ("BulkEnergy", "<f8"),
                          ("phi1", "<f8"), ("PHI", "<f8"), ("phi2", "<f8"), ("x", "<f8"), ("y", "<f8"),
                          ("z", "<f8"), ("id", "<u4"), ("NeighbourCount", "<u4"),
                          ("intersectsBoundaryGrain", "<u4"), ("pad", "<u4")])
FACE_DTYPE = np.dtype([("area", "<f8"), ("grainA", "<u4"), ("grainB", "<u4")])


def euler_to_quaternion(e) -> tuple:
    """myQuaternion::euler2Quaternion (myQuaternion.cpp:168-191), Bunge ZXZ."""
    p1, t, p2 = float(e[0]), float(e[1]), float(e[2])
    co1, s1 = math.cos(t / 2), math.sin(t / 2)
    return (co1 * math.cos((p1 + p2) / 2), s1 * math.cos((p1 - p2) / 2), s1 * math.sin((p1 - p2) / 2),
            co1 * math.sin((p1 + p2) / 2))


def quaternion_to_euler(q) -> tuple:
    """myQuaternion::Quaternion2Euler (myQuaternion.cpp:193-240): (phi1, PHI, phi2)."""
    q0, q1, q2, q3 = q
    cos_phi = q3 * q3 - q2 * q2 - q1 * q1 + q0 * q0
    y0 = 2 * q1 * q3 - 2 * q0 * q2
    x0 = 2 * q2 * q3 + 2 * q0 * q1
    y1 = 2 * q1 * q3 + 2 * q0 * q2
    x1 = -2 * q2 * q3 + 2 * q0 * q1
    if cos_phi > 1.0:
        cos_phi = 1.0
    PHI = 0.0 if (1.0 - cos_phi) * (1.0 - cos_phi) <= 1e-20 else math.acos(cos_phi)  # QUAT2EUL_ETA
    sP = math.sin(PHI)
    if sP != 0:
        phi2 = math.atan2(y0 / sP, x0 / sP)
        phi1 = math.atan2(y1 / sP, x1 / sP)
    else:
        phi1 = math.atan2(2 * q1 * q2 + 2 * q0 * q3, q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3)
        phi2 = 0.0
    if phi1 < 0.0:
        phi1 += 2 * math.pi
    if phi2 < 0.0:
        phi2 += 2 * math.pi
    return phi1, PHI, phi2


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def box_shape(box) -> tuple:
    x0, x1, y0, y1, z0, z1 = (int(v) for v in box)
    return (z1 - z0, y1 - y0, x1 - x0)


@dataclasses.dataclass
class GrainStats:
    exists: np.ndarray      # (G+1,) bool, entry 0 unused
    volume: np.ndarray
    surface: np.ndarray
    boxes: np.ndarray       # (G+1, 6)
    n_neighbors: np.ndarray


class GrainHandler:
    """One simulation on one GPU: the reference's grainhdl, stage for stage.

    ``labels`` (N^3 uint32, [z][y][x], grain IDs 1..G), ``extents`` (G x 6 inclusive
    domain extents) and ``counts`` (voxels per grain) are the mode-4 input; see
    ``gragles_3d_b200.microstructure``.
    """

    def __init__(self, domain_size: int, border: int, time_step: float, n_grains: int,
                 precision: int = PRECISION_FP64, list_capacity: int = 0, pool_voxels: int = 0,
                 device: int = 0, correction: bool = False, unique_energies: bool = True,
                 mobility_model: bool = False, stored_energy: bool = False, triple_line_drag: float = 0.0,
                 hull_capacity: int = 0, keep_elements: bool = False, grid_coarsening: bool = False,
                 points_per_grain: int = 0, coarsening_gradient: float = 0.0, autotune: bool = False):
        L = load_library()
        self.G = int(n_grains)
        self.N = int(domain_size)
        self.border = int(border)
        self.M = self.N + 2 * self.border
        self.precision = precision
        p = Params(domain_size, border, float(time_step), n_grains, precision, int(not correction), list_capacity,
                   pool_voxels, device, int(unique_energies), int(mobility_model), int(stored_energy),
                   float(triple_line_drag), hull_capacity, int(keep_elements), int(grid_coarsening),
                   int(points_per_grain), float(coarsening_gradient), int(autotune))
        self._euler = np.zeros((self.G, 3))
        self._see = np.zeros(self.G)
        h = C.c_void_p()
        self._lib = L  # held for close() at interpreter exit, when module globals are gone
        rc = L.gg_create(C.byref(p), C.byref(h))
        self._h = h
        self._check(rc)

    def _check(self, rc: int) -> int:
        if rc < 0:
            msg = load_library().gg_last_error(self._h).decode() if self._h else ""
            raise GGError(rc, msg)
        return rc

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gg_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- set-up -----------------------------------------------------------
    def load(self, labels: np.ndarray, extents: np.ndarray, counts: np.ndarray) -> None:
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        ext = np.ascontiguousarray(extents, dtype=np.int32)
        cnt = np.ascontiguousarray(counts, dtype=np.int64)
        self._check(load_library().gg_load_state(self._h, _p(lab), _p(ext), _p(cnt)))

    def set_lists(self, offsets: np.ndarray, ids: np.ndarray) -> None:
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        self._check(load_library().gg_set_lists(self._h, _p(off), _p(ids)))

    def default_lists(self) -> None:
        self._check(load_library().gg_default_lists(self._h))

    def rtree_lists(self) -> None:
        """The initial comparison lists in the reference's R-tree search order
        (find_neighbors, grainhdl.cpp:1029-1054)."""
        self._check(load_library().gg_rtree_lists(self._h))

    def set_orientations(self, euler: np.ndarray) -> None:
        """Bunge angles (G, 3) in radians for grain IDs 1..G."""
        e = np.ascontiguousarray(euler, dtype=np.float64)
        self._check(load_library().gg_set_orientations(self._h, _p(e)))
        self._euler = e.reshape(self.G, 3).copy()

    def set_stored_energy(self, see: np.ndarray) -> None:
        """m_StoredElasticEnergy (G,) for grain IDs 1..G."""
        v = np.ascontiguousarray(see, dtype=np.float64)
        self._check(load_library().gg_set_stored_energy(self._h, _p(v)))
        self._see = v.reshape(self.G).copy()

    def elements(self, gid: int) -> tuple:
        """(GB, TL, QJ, HJ) element counts of the grain's last hull (correction on)."""
        c = np.zeros(4, np.int32)
        self._check(load_library().gg_get_elements(self._h, gid, _p(c)))
        return tuple(int(v) for v in c)

    # --- the loop ---------------------------------------------------------
    def step(self) -> dict:
        st = StepStats()
        self._check(load_library().gg_step(self._h, C.byref(st)))
        return st.as_dict()

    def stage(self, name: str) -> None:
        self._check(getattr(load_library(), f"gg_stage_{name}")(self._h))

    @property
    def grain_count(self) -> int:
        return self._check(load_library().gg_grain_count(self._h))

    @property
    def loop(self) -> int:
        return self._check(load_library().gg_loop(self._h))

    def launch_config(self) -> tuple:
        """(CTAs per SM of each stage's kernels, chosen): the stages are the convolution with
        the correction, lists, comparison, level set and redistancing."""
        m = np.zeros(5, np.int32)
        done = self._check(load_library().gg_launch_config(self._h, _p(m)))
        return tuple(int(v) for v in m), bool(done)

    @property
    def domain_size(self) -> int:
        """The current grid size N (grainhdl::realDomainSize; shrinks with grid coarsening)."""
        return self._check(load_library().gg_domain_size(self._h))

    # --- read-back ---------------------------------------------------------
    def stats(self) -> GrainStats:
        G1 = self.G + 1
        ex = np.zeros(G1, np.uint8); vol = np.zeros(G1); sur = np.zeros(G1)
        box = np.zeros((G1, 6), np.int32); nn = np.zeros(G1, np.int32)
        self._check(load_library().gg_get_grain_stats(self._h, _p(ex), _p(vol), _p(sur), _p(box), _p(nn)))
        return GrainStats(ex.astype(bool), vol, sur, box, nn)

    def neighbors(self, gid: int) -> np.ndarray:
        buf = np.zeros(256, np.uint32)
        n = self._check(load_library().gg_get_neighbors(self._h, gid, _p(buf), buf.size))
        return buf[:min(n, buf.size)].copy()

    def comparison_list(self, gid: int) -> np.ndarray:
        buf = np.zeros(1 << 16, np.uint32)
        n = self._check(load_library().gg_get_list(self._h, gid, _p(buf), buf.size))
        return buf[:n].copy()

    def sdf(self, gid: int, which: int = 1):
        box = np.zeros(6, np.int32)
        n = self._check(load_library().gg_get_sdf(self._h, gid, which, _p(box), None, 0))
        out = np.zeros(n, np.float64)
        load_library().gg_get_sdf(self._h, gid, which, _p(box), _p(out), n)
        return tuple(int(v) for v in box), out.reshape(box_shape(box))

    def faces(self) -> np.ndarray:
        """Faces_<loop>.bin's records (grainhdl.cpp:753-775): FACE_DTYPE, every existing
        grain's boundaries toward lower IDs (needs correction or keep_elements)."""
        L = load_library()
        n = self._check(L.gg_get_faces(self._h, None, None, None, 0))
        area = np.zeros(n); ga = np.zeros(n, np.uint32); gb = np.zeros(n, np.uint32)
        self._check(L.gg_get_faces(self._h, _p(area), _p(ga), _p(gb), n))
        out = np.zeros(n, FACE_DTYPE)
        out["area"], out["grainA"], out["grainB"] = area, ga, gb
        return out

    def texture(self) -> np.ndarray:
        """Texture_<loop>.bin's records (LSbox::collectTextureData, box.cpp:3034-3045):
        TEXTURE_DTYPE, one per existing grain in ascending ID order.  GBEnergy is the
        reference's m_energy, which no code path of it assigns (0)."""
        st = self.stats()
        h_grid = 1.0 / self.domain_size
        ids = [g for g in range(1, self.G + 1) if st.exists[g]]
        out = np.zeros(len(ids), TEXTURE_DTYPE)
        for r, g in enumerate(ids):
            x0, x1, y0, y1, z0, z1 = (int(v) for v in st.boxes[g])
            phi1, PHI, phi2 = quaternion_to_euler(euler_to_quaternion(self._euler[g - 1]))
            out[r] = (st.volume[g], st.surface[g], 0.0, self._see[g - 1], phi1, PHI, phi2,
                      ((x1 - x0) // 2 + x0) * h_grid, ((y1 - y0) // 2 + y0) * h_grid,
                      ((z1 - z0) // 2 + z0) * h_grid, g, st.n_neighbors[g],
                      int(0 in set(self.neighbors(g).tolist())), 0)
        return out

    def texture_text(self) -> list:
        """The rows of Texture_<loop>.ori, the text form of save_Texture (grainhdl.cpp:776-805),
        one per existing grain in ascending ID order: ID, hull neighbour count, boundary
        flag, volume, surface, m_energy, mean width, triple-line length, triple lines,
        quadruple points, high-order junctions, stored elastic energy, Bunge angles.
        m_energy is never assigned by the reference (0); GrainHull::meanWidth and
        computeTriplelineLength (grainHull.cpp:1211-1329) have no caller in it, so the
        members it prints for them keep their initial value, 0 here.  The junction counts
        need the interfacial elements (correction or keep_elements)."""
        st = self.stats()
        rows = []
        for g in range(1, self.G + 1):
            if not st.exists[g]:
                continue
            _, tl, qj, hj = self.elements(g)
            phi1, PHI, phi2 = quaternion_to_euler(euler_to_quaternion(self._euler[g - 1]))
            rows.append((g, int(st.n_neighbors[g]), int(0 in set(self.neighbors(g).tolist())), st.volume[g],
                         st.surface[g], 0.0, 0.0, 0.0, float(tl), float(qj), float(hj), self._see[g - 1], phi1, PHI,
                         phi2))
        return rows

    def network_rows(self) -> list:
        """The rows of Microstructure_<loop>.uds that saveNetworkAsVoxelContainer writes
        (grainhdl.cpp:1093-1111), one per existing grain in ascending ID order: ID, box
        centre (integer midpoint times h), Bunge angles, box, volume, stored elastic energy."""
        st = self.stats()
        h = 1.0 / self.domain_size
        rows = []
        for g in range(1, self.G + 1):
            if not st.exists[g]:
                continue
            x0, x1, y0, y1, z0, z1 = (int(v) for v in st.boxes[g])
            phi1, PHI, phi2 = quaternion_to_euler(euler_to_quaternion(self._euler[g - 1]))
            rows.append((g, ((x1 - x0) // 2 + x0) * h, ((y1 - y0) // 2 + y0) * h, ((z1 - z0) // 2 + z0) * h, phi1,
                         PHI, phi2, x0, x1, y0, y1, z0, z1, st.volume[g], self._see[g - 1]))
        return rows

    def voxel_container(self) -> np.ndarray:
        """The network as an (N, N, N) [z][y][x] array of grain IDs (the reference's
        Container_size_N_t_loop.raw)."""
        n = self.domain_size
        out = np.zeros((n, n, n), np.uint32)
        self._check(load_library().gg_voxel_container(self._h, _p(out)))
        return out

    def idlocal(self, gid: int):
        box = np.zeros(6, np.int32)
        n = self._check(load_library().gg_get_idlocal(self._h, gid, _p(box), None, 0))
        out = np.zeros(n, np.uint32)
        load_library().gg_get_idlocal(self._h, gid, _p(box), _p(out), n)
        return tuple(int(v) for v in box), out


def from_microstructure(ms, border: int = 10, time_step: float = 0.2, precision: int = PRECISION_FP64,
                        lists=None, **kw) -> GrainHandler:
    """Create a handler, load a ``microstructure.Microstructure`` and its lists."""
    ext, counts = ms.grain_extents()
    gh = GrainHandler(ms.n, border, time_step, ms.n_grains, precision=precision, **kw)
    gh.load(ms.labels, ext, counts)
    if lists is None:
        gh.default_lists()
    else:
        gh.set_lists(*lists)
    return gh


def rtree_lists(boxes: np.ndarray, valid: np.ndarray):
    """find_neighbors' R-tree search on host boxes ((G + 1) x 6, valid (G + 1) flags):
    the initial comparison lists as CSR (offsets[G + 2], ids) in the reference's order.
    Host only: no GPU needed."""
    L = load_library()
    b = np.ascontiguousarray(boxes, dtype=np.int32)
    v = np.ascontiguousarray(valid, dtype=np.uint8)
    G = b.shape[0] - 1
    off = np.zeros(G + 2, np.int64)
    n = L.gg_rtree_lists_from_boxes(G, _p(b), _p(v), _p(off), None, 0)
    if n < 0:
        raise GGError(int(n), "gg_rtree_lists_from_boxes failed")
    ids = np.zeros(max(n, 1), np.uint32)
    L.gg_rtree_lists_from_boxes(G, _p(b), _p(v), _p(off), _p(ids), n)
    return off, ids[:n]


def convolve_boxes_f64(boxes: list, domain_size: int, time_step: float) -> list:
    """FP64 Gaussian convolution of cubic boxes on the GPU (torch manages the device memory)."""
    return _convolve_boxes(boxes, domain_size, time_step, np.float64, "gg_convolve_boxes_f64")


def convolve_boxes_mixed(boxes: list, domain_size: int, time_step: float) -> list:
    """The mixed path's FP32 convolution (tensor cores when all sides are <= 64) of cubic boxes."""
    return _convolve_boxes(boxes, domain_size, time_step, np.float32, "gg_convolve_boxes_mixed")


def _convolve_boxes(boxes: list, domain_size: int, time_step: float, dtype, fn: str) -> list:
    import torch

    L = load_library()
    sides = np.array([b.shape[0] for b in boxes], np.int32)
    offs = np.zeros(len(boxes), np.int64)
    total = 0
    for i, b in enumerate(boxes):
        offs[i] = total
        total += (b.size + 31) // 32 * 32
    host = np.zeros(max(total, 1), dtype)
    for i, b in enumerate(boxes):
        host[offs[i]:offs[i] + b.size] = b.ravel()
    d_in = torch.from_numpy(host).cuda()
    d_out = torch.zeros_like(d_in)
    rc = getattr(L, fn)(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), _p(sides), _p(offs),
                        len(boxes), domain_size, float(time_step))
    if rc < 0:
        raise GGError(rc, f"{fn} failed")
    out = d_out.cpu().numpy()
    return [out[offs[i]:offs[i] + b.size].reshape(b.shape).copy() for i, b in enumerate(boxes)]

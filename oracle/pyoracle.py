"""ctypes binding of the C restatement (oracle/liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_double
        L.ggo_create.restype = vp
        L.ggo_create.argtypes = [i32, i32, dbl, i32]
        L.ggo_destroy.argtypes = [vp]
        L.ggo_load.argtypes = [vp, vp, vp, vp]
        L.ggo_set_lists.argtypes = [vp, vp, vp]
        L.ggo_default_lists.argtypes = [vp]
        L.ggo_step.argtypes = [vp]
        L.ggo_loop.argtypes = [vp]
        L.ggo_grain_info.argtypes = [vp, i32, vp, vp, vp, vp, vp]
        L.ggo_grain_neighbors.argtypes = [vp, i32, vp, i32]
        L.ggo_grain_list.argtypes = [vp, i32, vp, i32]
        L.ggo_grain_sdf.restype = i64
        L.ggo_grain_sdf.argtypes = [vp, i32, vp, vp, i64]
        L.ggo_grain_idlocal.restype = i64
        L.ggo_grain_idlocal.argtypes = [vp, i32, vp, vp, i64]
        L.ggo_last_voxels.restype = i64
        L.ggo_last_voxels.argtypes = [vp]
        L.ggo_convolve_box.argtypes = [i32, i32, dbl, vp, vp]
        L.ggo_redistance_box.argtypes = [vp, vp, vp, vp, dbl, dbl]
        L.ggo_mc_box.restype = i64
        L.ggo_mc_box.argtypes = [vp, vp, vp, C.c_uint32, dbl, vp, vp, vp, vp, i32]
        L.ggo_compare_box.argtypes = [vp, i32, vp, vp, vp, vp, vp, i32, i32, dbl]
        L.ggo_set_compare_box.argtypes = [vp, vp, vp, dbl, i32, i32, vp]
        L.ggo_resize_to_cube.argtypes = [vp, i32]
        L.ggo_set_physics.argtypes = [vp, i32, i32, i32, dbl, i32]
        L.ggo_set_orientations.argtypes = [vp, vp]
        L.ggo_set_stored_energy.argtypes = [vp, vp]
        L.ggo_grain_elements.argtypes = [vp, i32, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def box_shape(box):
    x0, x1, y0, y1, z0, z1 = (int(v) for v in box)
    return (z1 - z0, y1 - y0, x1 - x0)


class OracleSim:
    """The restated loop over one microstructure (isotropic path)."""

    def __init__(self, N: int, border: int, time_step: float, labels: np.ndarray,
                 extents: np.ndarray, counts: np.ndarray, lists=None):
        L = lib()
        self.G = int(extents.shape[0])
        self.N, self.border = N, border
        self.h = 1.0 / N
        self.delta = border / float(N)
        self._s = L.ggo_create(N, border, float(time_step), self.G)
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        ext = np.ascontiguousarray(extents, dtype=np.int32)
        cnt = np.ascontiguousarray(counts, dtype=np.int64)
        L.ggo_load(self._s, _p(lab), _p(ext), _p(cnt))
        if lists is None:
            L.ggo_default_lists(self._s)
        else:
            off, ids = lists
            off = np.ascontiguousarray(off, dtype=np.int64)
            ids = np.ascontiguousarray(ids, dtype=np.uint32)
            L.ggo_set_lists(self._s, _p(off), _p(ids))

    def __del__(self):
        if getattr(self, "_s", None):
            lib().ggo_destroy(self._s)
            self._s = None

    def set_physics(self, correction: bool, unique_energies: bool = True, mobility_model: bool = False,
                    triple_line_drag: float = 0.0, stored_energy: bool = False) -> None:
        """The convolution correction and its settings (box.cpp:426-535)."""
        lib().ggo_set_physics(self._s, int(correction), int(unique_energies), int(mobility_model),
                              float(triple_line_drag), int(stored_energy))

    def set_orientations(self, euler: np.ndarray) -> None:
        """Bunge angles per grain, (G, 3) for IDs 1..G."""
        e = np.zeros((self.G + 1, 3), np.float64)
        e[1:] = euler
        lib().ggo_set_orientations(self._s, _p(e))

    def set_stored_energy(self, see: np.ndarray) -> None:
        """m_StoredElasticEnergy per grain, (G,) for IDs 1..G."""
        v = np.zeros(self.G + 1, np.float64)
        v[1:] = see
        lib().ggo_set_stored_energy(self._s, _p(v))

    def elements(self, gid: int):
        """(GB, TL, QJ, HJ) counts of the grain's last hull."""
        c = np.zeros(4, np.int32)
        lib().ggo_grain_elements(self._s, gid, _p(c))
        return tuple(int(v) for v in c)

    def step(self) -> int:
        return int(lib().ggo_step(self._s))

    @property
    def loop(self) -> int:
        return int(lib().ggo_loop(self._s))

    def last_voxels(self) -> int:
        return int(lib().ggo_last_voxels(self._s))

    def info(self, gid: int):
        ex = C.c_int(); box = np.zeros(6, np.int32); vol = C.c_double(); sur = C.c_double(); nn = C.c_int()
        present = lib().ggo_grain_info(self._s, gid, C.byref(ex), _p(box), C.byref(vol), C.byref(sur), C.byref(nn))
        return {"present": bool(present), "exists": bool(ex.value), "box": tuple(int(v) for v in box),
                "volume": vol.value, "surface": sur.value, "n_neighbors": nn.value}

    def neighbors(self, gid: int) -> np.ndarray:
        buf = np.zeros(4096, np.uint32)
        n = lib().ggo_grain_neighbors(self._s, gid, _p(buf), buf.size)
        return buf[:max(n, 0)].copy()

    def comparison_list(self, gid: int) -> np.ndarray:
        buf = np.zeros(1 << 16, np.uint32)
        n = lib().ggo_grain_list(self._s, gid, _p(buf), buf.size)
        return buf[:max(n, 0)].copy()

    def sdf(self, gid: int):
        box = np.zeros(6, np.int32)
        n = lib().ggo_grain_sdf(self._s, gid, _p(box), None, 0)
        out = np.zeros(max(n, 0), np.float64)
        lib().ggo_grain_sdf(self._s, gid, _p(box), _p(out), out.size)
        return tuple(int(v) for v in box), out.reshape(box_shape(box))

    def idlocal(self, gid: int):
        box = np.zeros(6, np.int32)
        n = lib().ggo_grain_idlocal(self._s, gid, _p(box), None, 0)
        out = np.zeros(max(n, 0), np.uint32)
        lib().ggo_grain_idlocal(self._s, gid, _p(box), _p(out), out.size)
        return tuple(int(v) for v in box), out


def convolve_box(sdf: np.ndarray, N: int, time_step: float) -> np.ndarray:
    n = sdf.shape[0]
    a = np.ascontiguousarray(sdf, dtype=np.float64)
    out = np.empty_like(a)
    lib().ggo_convolve_box(n, N, float(time_step), _p(a), _p(out))
    return out


def redistance_box(in_box, sdf_in: np.ndarray, out_box, h: float, delta: float) -> np.ndarray:
    ib = np.asarray(in_box, np.int32)
    ob = np.asarray(out_box, np.int32)
    a = np.ascontiguousarray(sdf_in, dtype=np.float64)
    out = np.empty(box_shape(ob), np.float64)
    lib().ggo_redistance_box(_p(ib), _p(a), _p(ob), _p(out), float(h), float(delta))
    return out


def mc_box(box, sdf: np.ndarray, idlocal: np.ndarray, own_id: int, h: float):
    b = np.asarray(box, np.int32)
    a = np.ascontiguousarray(sdf, dtype=np.float64)
    ids = np.ascontiguousarray(idlocal, dtype=np.uint32)
    vol = C.c_double(); sur = C.c_double(); nn = C.c_int()
    nb = np.zeros(4096, np.uint32)
    ntri = lib().ggo_mc_box(_p(b), _p(a), _p(ids), own_id, float(h), C.byref(vol), C.byref(sur),
                            _p(nb), C.byref(nn), nb.size)
    return int(ntri), vol.value, sur.value, nb[:nn.value].copy()


def compare_box(box, nb_boxes, nb_ids, nb_sdfs, idlocal: np.ndarray, M: int, border: int, h: float):
    b = np.asarray(box, np.int32)
    K = len(nb_ids)
    boxes = np.ascontiguousarray(np.asarray(nb_boxes, np.int32).reshape(K, 6))
    ids = np.ascontiguousarray(np.asarray(nb_ids, np.uint32))
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in nb_sdfs]
    ptrs = (C.c_void_p * max(K, 1))(*[a.ctypes.data for a in arrs])
    out = np.empty(box_shape(b), np.float64)
    idl = np.ascontiguousarray(idlocal, dtype=np.uint32).copy()
    lib().ggo_compare_box(_p(b), K, _p(boxes), _p(ids), C.cast(ptrs, C.c_void_p), _p(out), _p(idl), M, border, float(h))
    return out, idl


def set_compare_box(box, sdf_in: np.ndarray, cmp_out: np.ndarray, delta: float, M: int, border: int):
    b = np.asarray(box, np.int32)
    a = np.ascontiguousarray(sdf_in, dtype=np.float64)
    out = np.ascontiguousarray(cmp_out, dtype=np.float64).copy()
    nb = np.zeros(6, np.int32)
    lib().ggo_set_compare_box(_p(b), _p(a), _p(out), float(delta), M, border, _p(nb))
    return out, tuple(int(v) for v in nb)


def resize_to_cube(box, M: int):
    b = np.asarray(box, np.int32).copy()
    lib().ggo_resize_to_cube(_p(b), M)
    return tuple(int(v) for v in b)

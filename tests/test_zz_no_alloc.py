"""The allocation-free FP64 box convolution (gg_convolve_boxes_f64_noalloc).

It serves callers of this library that cannot call cudaMalloc -- a program that
gives all device memory to its own pool at start-up, or one whose device footprint
must stay fixed after start-up -- by keeping its scratch in fixed device arrays.  Its output must be bit-identical to gg_convolve_boxes_f64 (the
FP64 path's tolerance is exactness), call after call, although every call reuses
and leaves behind the same scratch.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pack(boxes):
    sides = np.array([b.shape[0] for b in boxes], np.int32)
    offs = np.zeros(len(boxes), np.int64)
    total = 0
    for i, b in enumerate(boxes):
        offs[i] = total
        total += (b.size + 31) // 32 * 32
    host = np.zeros(max(total, 1), np.float64)
    for i, b in enumerate(boxes):
        host[offs[i]:offs[i] + b.size] = b.ravel()
    return sides, offs, host


def _run(lib, fn, boxes, N, ts):
    import torch

    sides, offs, host = _pack(boxes)
    d_in = torch.from_numpy(host).cuda()
    d_out = torch.full_like(d_in, float("nan"))
    f = getattr(lib, fn)
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double]
    rc = f(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), sides.ctypes.data_as(C.c_void_p),
           offs.ctypes.data_as(C.c_void_p), len(boxes), N, ts)
    assert rc == 0, f"{fn} returned {rc}"
    out = d_out.cpu().numpy()
    return [out[offs[i]:offs[i] + b.size].reshape(b.shape) for i, b in enumerate(boxes)]


def test_noalloc_convolution_matches_the_allocating_one_twice(gpu):
    lib = gpu.load_library()
    rng = np.random.default_rng(11)
    # two calls in a row with different sizes and parameters: the second must not see
    # anything the first left in the shared scratch
    for sides, N, ts in (([7, 16, 33, 40, 48], 128, 0.2), ([12, 25, 9], 64, 0.15)):
        boxes = [rng.uniform(-0.1, 0.1, (n, n, n)) for n in sides]
        want = _run(lib, "gg_convolve_boxes_f64", boxes, N, ts)
        got = _run(lib, "gg_convolve_boxes_f64_noalloc", boxes, N, ts)
        for w, g in zip(want, got):
            assert np.array_equal(w, g), f"side {w.shape[0]}: max diff {np.abs(w - g).max()}"


def test_noalloc_convolution_at_its_limits(gpu):
    """The largest side the arrays take (96) and a call that fills the 2^21-complex
    scratch to 99%, each compared bit for bit with the allocating entry point."""
    lib = gpu.load_library()
    rng = np.random.default_rng(12)
    near_full = [96, 96, 96, 96, 64, 48, 40, 36, 32]
    used = sum(n * n * (n // 2 + 1) for n in near_full)
    assert 0.98 * (1 << 21) < used <= (1 << 21)
    for sides in ([96], near_full):
        boxes = [rng.uniform(-0.05, 0.05, (n, n, n)) for n in sides]
        want = _run(lib, "gg_convolve_boxes_f64", boxes, 256, 0.2)
        got = _run(lib, "gg_convolve_boxes_f64_noalloc", boxes, 256, 0.2)
        for w, g in zip(want, got):
            assert np.array_equal(w, g), f"side {w.shape[0]}: max diff {np.abs(w - g).max()}"


def test_noalloc_convolution_refuses_sizes_beyond_its_arrays(gpu):
    lib = gpu.load_library()
    f = lib.gg_convolve_boxes_f64_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double]
    dummy = C.c_void_p(16)  # never dereferenced: the limits are checked first
    too_wide = np.array([97], np.int32)
    offs = np.zeros(1, np.int64)
    assert f(dummy, dummy, too_wide.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), 1, 128,
             0.2) == gpu.GG_ERR_UNSUPPORTED
    many = np.full(257, 8, np.int32)
    offs = np.zeros(257, np.int64)
    assert f(dummy, dummy, many.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), 257, 128,
             0.2) == gpu.GG_ERR_UNSUPPORTED
    big = np.full(40, 96, np.int32)  # 40 * 96*96*49 complex values > 2^21
    offs = np.zeros(40, np.int64)
    assert f(dummy, dummy, big.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), 40, 128,
             0.2) == gpu.GG_ERR_UNSUPPORTED

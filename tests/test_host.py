"""CPU tests of the host side: the C ABI library loads and exports every symbol
include/gg_b200.h declares (no compute calls without a GPU), the microstructure
generator and its mode-4 files, and the replica aggregation of the multi-GPU
bench path over a two-rank gloo group."""
import os
import re
import socket
import tempfile

import numpy as np
import pytest

from gragles_3d_b200 import microstructure as msgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gg_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import ctypes

    import gragles_3d_b200 as gg

    lib_path = gg.LIB_PATH
    if not os.path.exists(lib_path):
        from gragles_3d_b200 import build

        build.build()
    lib = ctypes.CDLL(lib_path)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(gg.EXPORTED) == names


def test_create_rejects_bad_parameters_without_touching_the_device():
    import gragles_3d_b200 as gg

    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(1, 10, 0.2, 5)
    assert e.value.code == gg.GG_ERR_INVALID
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(64, 10, 0.2, 5, precision=7)
    assert e.value.code == gg.GG_ERR_INVALID


def test_generator_is_deterministic_and_consistent():
    from gragles_3d_b200 import microstructure as msgen

    a = msgen.voronoi(24, 30, seed=5)
    b = msgen.voronoi(24, 30, seed=5)
    assert np.array_equal(a.labels, b.labels) and np.array_equal(a.euler, b.euler)
    assert a.labels.min() >= 1 and a.labels.max() <= 30
    ext, counts = a.grain_extents()
    assert counts.sum() == 24 ** 3
    for g in range(30):
        if counts[g] == 0:
            continue
        z, y, x = np.nonzero(a.labels == g + 1)
        assert tuple(ext[g]) == (x.min(), x.max(), y.min(), y.max(), z.min(), z.max())
    c = msgen.laguerre(24, 30, seed=5, sigma=0.3)
    assert c.labels.min() >= 1


def test_mode4_files_follow_the_reference_reader():
    """The header/rows parse the way grainhdl.cpp:404-578 reads them (fscanf)."""
    from gragles_3d_b200 import microstructure as msgen

    ms = msgen.voronoi(16, 9, seed=3)
    with tempfile.TemporaryDirectory() as d:
        raw, uds = msgen.write_mode4(ms, d)
        data = np.fromfile(raw, dtype="<u4").reshape(16, 16, 16)
        assert np.array_equal(data, ms.labels)
        lines = open(uds).read().split("\n")
        assert lines[1].split() == ["ID_offset", "1"]
        assert [l.split()[1] for l in lines[5:8]] == ["16", "16", "16"]
        assert lines[8].split() == ["NumberOfGrains", "9"]
        assert lines[9] == "" and lines[10] == ""
        rows = [l.split() for l in lines[12:] if l.strip()]
        assert len(rows) == 9 and all(len(r) == 15 for r in rows)
        ext, counts = ms.grain_extents()
        for g, r in enumerate(rows):
            assert int(r[0]) == g + 1
            assert [int(v) for v in r[7:13]] == list(ext[g]) and int(r[13]) == counts[g]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _replica_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    elapsed = [10.0, 14.0][rank]
    vox = [1000.0, 1200.0][rank]
    q.put((rank, bench.aggregate_replicas(elapsed, vox, dist, device="cpu")))
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks_gloo():
    """N>1 bench path: throughput = all ranks' voxel-updates / slowest rank's time."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        elapsed, vox = res[r]
        assert elapsed == 14.0 and vox == 2200.0


def test_container_file_layout(tmp_path):
    """write_container writes the reference's raw uint32 layout (x fastest) under its name."""
    from gragles_3d_b200 import microstructure as msgen

    lab = np.arange(4 * 4 * 4, dtype=np.uint32).reshape(4, 4, 4)
    path = msgen.write_container(str(tmp_path), lab, 7)
    assert os.path.basename(path) == "Container_size_4_t_7.raw"
    back = np.fromfile(path, np.uint32)
    assert np.array_equal(back, lab.ravel())


def test_texture_euler_angles_follow_the_reference():
    """The Texture records' angles: Quaternion2Euler(euler2Quaternion(.uds angles)) as the
    reference computes them, checked against its own Texture_1.bin (tests/golden/analysis.npz)."""
    import gragles_3d_b200 as gg

    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "analysis.npz")))
    t = d["texture"][:int(d["texture_len"][0])]
    for rec in t:
        e = gg.quaternion_to_euler(gg.euler_to_quaternion(d["euler"][rec["id"] - 1]))
        assert np.allclose(e, (rec["phi1"], rec["PHI"], rec["phi2"]), rtol=0, atol=1e-12)


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The Python mirrors of gg_params and gg_step_stats have the C layout: size and
    every field's offset, from a program gcc compiles against include/gg_b200.h."""
    import ctypes as C
    import shutil
    import subprocess

    if not shutil.which("gcc"):
        pytest.skip("gcc missing")
    from gragles_3d_b200 import Params, StepStats

    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gg_b200.h"', "int main(void) {"]
    for cname, py in (("gg_params", Params), ("gg_step_stats", StepStats)):
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = row.split()
        got[(cname, field)] = int(value)
    for cname, py in (("gg_params", Params), ("gg_step_stats", StepStats)):
        assert got[(cname, "size")] == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_stored_energy_and_nuclei_generator():
    """The stored-energy configuration's generator: lognormal stored energy of 0.1 boundary
    energy (the .uds column scaled back through box.cpp:232-233), then 5% nuclei of radius
    2-3 voxels appended as new IDs with none; deterministic for a seed."""
    a, b = msgen.c4(48, 200, seed=5), msgen.c4(48, 200, seed=5)
    assert np.array_equal(a.labels, b.labels) and np.array_equal(a.stored_energy, b.stored_energy)
    G, K = 200, 10
    assert a.n_grains == G + K and a.labels.max() == G + K
    see = msgen.stored_energy_of(a.stored_energy)
    assert np.all(see[G:] == 0) and np.all(see[:G] > 0)
    assert 0.05 < np.median(see[:G]) < 0.2  # 0.1 * LogNormal(0, 0.5): median 0.1
    _, counts = a.grain_extents()
    vol = 4.0 / 3.0 * np.pi
    assert np.all(counts[G:] >= 0.5 * vol * 2 ** 3) and np.all(counts[G:] <= 1.5 * vol * 3 ** 3)


def test_text_writers_print_like_the_reference_ostream(tmp_path):
    """Texture_<loop>.ori and Microstructure_<loop>.uds rows: tab-separated, integers as
    they are, doubles as the reference's ostream prints them by default (6 significant
    digits, %g)."""
    rows = [(3, 7, 1, 0.0195446123, 0.5, 0.0, 0.0, 0.0, 12.0, 6.0, 1.0, 8.399876e-09, 0.158441, 1e6, 2.0)]
    path = msgen.write_texture_text(str(tmp_path), rows, 4)
    assert os.path.basename(path) == "Texture_4.ori"
    with open(path) as f:
        assert f.read() == "3\t7\t1\t0.0195446\t0.5\t0\t0\t0\t12\t6\t1\t8.39988e-09\t0.158441\t1e+06\t2\n"
    labels = np.array([[[1, 2], [0, 2]], [[1, 1], [2, 2]]], np.uint32)
    out = msgen.write_network(str(tmp_path), 4, [(1, 0.5, 0.5, 0.5, 0.1, 0.2, 0.3, 0, 2, 0, 2, 0, 2, 0.125, 3.0),
                                                   (2, 0.5, 0.5, 0.5, 0.1, 0.2, 0.3, 0, 2, 0, 2, 0, 2, 0.25, 5.0)],
                              labels, see=np.array([3.0, 5.0]))
    assert [os.path.basename(p) for p in out] == ["Microstructure_4.uds", "Container_size_2_t_4.raw",
                                                  "ContainerVolumeEnergy_size_2_t_4.raw"]
    e = np.fromfile(out[2], "<f8")
    assert np.array_equal(e, np.array([3.0, 5.0, 0.0, 5.0, 3.0, 3.0, 5.0, 5.0]))


def _resize_to_cube(b, M):
    """DimensionalBuffer::resizeToCube (dimensionalBuffer.h:139-219)."""
    x0, x1, y0, y1, z0, z1 = b
    w, h, d = x1 - x0, y1 - y0, z1 - z0
    if w == h == d:
        return [x0, x1, y0, y1, z0, z1]
    ref = max(w, h, d)
    if ref > w:
        x0, x1 = x0 - (ref - w) // 2, x1 + (ref - w) // 2 + (ref - w) % 2
    if ref > h:
        y0, y1 = y0 - (ref - h) // 2, y1 + (ref - h) // 2 + (ref - h) % 2
    if ref > d:
        z0, z1 = z0 - (ref - d) // 2, z1 + (ref - d) // 2 + (ref - d) % 2
    out = []
    for lo, hi in ((x0, x1), (y0, y1), (z0, z1)):
        if lo < 0:
            lo, hi = 0, hi - lo
        elif hi > M - 1:
            lo, hi = lo + (M - 1 - hi), M - 1
        out += [lo, hi]
    return out


@pytest.mark.parametrize("name", ["tiny", "vanish", "correction", "c1", "coarsen"])
def test_rtree_lists_follow_the_reference_order(name):
    """find_neighbors' R-tree (grainhdl.cpp:1029-1054) restated on the host gives the
    reference's own initial comparison lists, member for member and in order, from the
    mode-4 constructor's boxes (box.cpp:239-304, then resizeToCube)."""
    import gragles_3d_b200 as gg

    d = dict(np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz")))
    N, G, gb = int(d["N"]), int(d["G"]), int(d["border"])
    M = N + 2 * gb
    ext, counts = msgen.voronoi(N, G, seed=int(d["seed"])).grain_extents()
    boxes = np.zeros((G + 1, 6), np.int32)
    valid = np.zeros(G + 1, np.uint8)
    for g in range(1, G + 1):
        if counts[g - 1] <= 0:
            continue
        x0, x1, y0, y1, z0, z1 = (int(v) for v in ext[g - 1])
        x1, y1, z1 = min(x1 + 2 * gb, M), min(y1 + 2 * gb, M), min(z1 + 2 * gb, M)
        boxes[g] = _resize_to_cube([max(x0, 0), x1, max(y0, 0), y1, max(z0, 0), z1], M)
        valid[g] = 1
    off, ids = gg.rtree_lists(boxes, valid)
    assert np.array_equal(off, d["init_list_off"])
    assert np.array_equal(ids, d["init_list_ids"])


def test_small_division_by_fp32_reciprocal_is_exact():
    """The redistancing kernels take a flat element index q apart into (row, column) with
    trunc((q + 1/2) * fl(1/d)) in FP32 (gg_redist.cu, div_small) for the fixed-side
    classes: q < 2^12 and d <= 64.  Every such pair, in IEEE FP32 arithmetic as the
    kernel does it (no fused multiply-add), gives q // d."""
    q = np.arange(4096, dtype=np.int64)
    for d in range(1, 65):
        rd = np.float32(1.0) / np.float32(d)
        prod = (q.astype(np.float32) + np.float32(0.5)) * rd
        assert prod.dtype == np.float32
        assert np.array_equal(np.trunc(prod).astype(np.int64), q // d), f"divisor {d}"


def test_marching_cubes_edge_table_is_empty_only_for_uniform_cubes():
    """The marching-cubes kernel treats a cube as active when its eight corner signs are not
    all alike (cube index neither 0 nor 255; gg_mc.cu, the row words any & ~all) instead of
    looking the edge table up: the table has no other empty entry."""
    src = open(os.path.join(ROOT, "gragles_3d_b200", "csrc", "gg_mc_tables.inc")).read()
    body = src[src.index("gg_mc_edge_table"):src.index("gg_mc_tri_table")]
    body = body[body.index("{") + 1:]
    vals = [int(v, 16) if v.lower().startswith("0x") else int(v)
            for v in re.findall(r"0[xX][0-9a-fA-F]+|\b\d+\b", body)][:256]
    assert len(vals) == 256
    assert [i for i, v in enumerate(vals) if v == 0] == [0, 255]


def test_junction_distance_test_without_square_root():
    """The element build tests the reference's sqrt(d2) < 2 as d2 < 4 (gg_hull.cu, the
    junction merges).  With a correctly rounded square root the two agree for every double:
    checked around 4 (the 2^20 doubles below it, and above) and on random squared
    distances."""
    import math

    xs = [4.0 - k * 2.0 ** -51 for k in range(1 << 20)] + [4.0 + k * 2.0 ** -50 for k in range(1024)]
    rng = np.random.default_rng(3)
    xs += list(rng.uniform(0.0, 100.0, 200000)) + list(rng.uniform(3.99, 4.01, 200000))
    for x in xs:
        assert (math.sqrt(x) < 2) == (x < 4.0), repr(x)

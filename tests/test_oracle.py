"""CPU tests of the oracle: the specified DFT against numpy and analytic answers,
the marching-cubes tables, and the C restatement against golden vectors the
reference solver itself produced (tests/golden/make_golden.py)."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _dft(oracle):
    L = oracle.lib()
    L.ggdft_forward_r2c_3d.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    L.ggdft_backward_c2r_3d.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    return L


@pytest.mark.parametrize("n", [1, 2, 5, 8, 13, 20, 33])
def test_specified_dft_matches_numpy(oracle, n):
    L = _dft(oracle)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    h = n // 2 + 1
    spec = np.zeros((n, n, h, 2))
    L.ggdft_forward_r2c_3d(n, x.ctypes.data, spec.ctypes.data)
    want = np.fft.rfftn(x)
    got = spec[..., 0] + 1j * spec[..., 1]
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())
    back = np.zeros((n, n, n))
    L.ggdft_backward_c2r_3d(n, spec.ctypes.data, back.ctypes.data)
    assert np.abs(back / n ** 3 - x).max() <= 1e-12 * max(1.0, np.abs(x).max())


def test_convolution_of_a_delta_is_the_separable_kernel(oracle):
    """IDFT(DFT(delta) G) = c (x) c (x) c with c the first column of the per-axis circulant."""
    n, N, ts = 21, 64, 0.2
    x = np.zeros((n, n, n))
    x[0, 0, 0] = 1.0
    out = oracle.convolve_box(x, N, ts)
    a = np.sqrt(2 / np.pi) * 4.0 * (ts / N ** 2) * N ** 2 / n ** 2 * np.pi ** 2
    f = np.minimum(np.arange(n), n - np.arange(n))
    g = np.exp(-a * f ** 2)
    c = np.array([np.sum(g * np.cos(2 * np.pi * np.arange(n) * d / n)) / n for d in range(n)])
    want = c[:, None, None] * c[None, :, None] * c[None, None, :]
    assert np.abs(out - want).max() <= 1e-14
    assert abs(out.sum() - 1.0) <= 1e-13  # G(0) = 1/n^3: the kernel preserves the mean


def test_mc_tables_are_consistent():
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import gen_mc_tables as g

    src = open(os.path.join(os.path.dirname(HERE), "gragles_3d_b200", "csrc", "gg_mc_tables.inc")).read()
    edge = [int(t, 16) for t in src.split("gg_mc_edge_table[256] = {")[1].split("};")[0].replace(",", " ").split()]
    body = src.split("gg_mc_tri_table[256][16] = {")[1].split("};")[0]
    tri = [[int(v) for v in row.split(",") if v.strip()] for row in body.replace("{", "").split("}") if row.strip(", \n")]
    g.check(edge, tri)


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def _ragged(off, ids, g):
    return ids[off[g]:off[g + 1]]


def golden_stored_energy(d):
    """m_StoredElasticEnergy = DislocEnPerM * storedEnergy / HAGB_Energy *
    Physical_Domain_Size (box.cpp:232-233) for the fixture's .uds column."""
    return 2.5e-10 * d["uds_stored_energy"] / 1.0 * 2.52e-4


def golden_sim(oracle, d):
    from gragles_3d_b200 import microstructure as msgen

    N, G, border, seed = int(d["N"]), int(d["G"]), int(d["border"]), int(d["seed"])
    ms = msgen.voronoi(N, G, seed=seed)
    ext, counts = ms.grain_extents()
    sim = oracle.OracleSim(N, border, 0.2, ms.labels, ext, counts, lists=(d["init_list_off"], d["init_list_ids"]))
    if "euler" in d:
        sim.set_physics(True, unique_energies=bool(d["phys_unique_energies"]),
                        mobility_model=bool(d["phys_mobility_factor"]),
                        triple_line_drag=float(d["phys_triple_line_drag"]),
                        stored_energy=bool(d["phys_stored_energy"]))
        sim.set_orientations(d["euler"])
        sim.set_stored_energy(golden_stored_energy(d))
    return sim


@pytest.mark.parametrize("name", ["tiny", "vanish", "correction"])
def test_restatement_matches_reference_golden(oracle, name):
    d = _load(name)
    G = int(d["G"])
    sim = golden_sim(oracle, d)
    nb_base = np.concatenate([[0], np.cumsum(d["nb_len"])])
    li_base = np.concatenate([[0], np.cumsum(d["list_len"])])
    for s in range(d["exists"].shape[0]):
        sim.step()
        nb_ids = d["nb_ids"][nb_base[s]:nb_base[s + 1]]
        li_ids = d["list_ids"][li_base[s]:li_base[s + 1]]
        for g in range(1, G + 1):
            inf = sim.info(g)
            if not d["exists"][s, g] and not inf["exists"]:
                continue
            assert inf["exists"] == bool(d["exists"][s, g]), (s, g)
            assert inf["box"] == tuple(d["box"][s, g]), (s, g)
            assert inf["volume"] == d["volume"][s, g], (s, g)
            assert inf["surface"] == d["surface"][s, g], (s, g)
            assert np.array_equal(sim.neighbors(g), _ragged(d["nb_off"][s], nb_ids, g)), (s, g)
        for g in range(1, G + 1):
            want = _ragged(d["list_off"][s], li_ids, g)
            if want.size:
                assert np.array_equal(sim.comparison_list(g), want), (s, g)


def test_single_box_stages_match_reference_golden(oracle):
    """Each single-box stage of the restatement reproduces the reference's own buffers."""
    d = _load("tiny")
    N, border = int(d["N"]), int(d["border"])
    h, delta = 1.0 / N, border / float(N)
    M = N + 2 * border

    def cube(kind):
        b = tuple(int(v) for v in d[f"box_{kind}"])
        return b, d[f"buf_{kind}"].reshape(b[5] - b[4], b[3] - b[2], b[1] - b[0])

    bi, cin = cube("CONV_IN")
    bo, cout = cube("CONV_OUT")
    assert np.array_equal(oracle.convolve_box(cin, N, 0.2), cout)
    bm, cmp_out = cube("CMP_OUT")
    # SETCMP_OUT's box field holds the new bounding box of executeSetComparison;
    # the buffer itself lies on the comparison box
    bs = tuple(int(v) for v in d["box_SETCMP_OUT"])
    set_out = d["buf_SETCMP_OUT"].reshape(cmp_out.shape)
    res, newbox = oracle.set_compare_box(bm, cout, cmp_out, delta, M, border)
    assert np.array_equal(res, set_out) and newbox == bs
    bmc, mc_in = cube("MC_IN")
    _, mc_id = cube("MC_ID")
    assert np.array_equal(mc_in, set_out)
    ntri, vol, sur, nbrs = oracle.mc_box(bmc, mc_in, mc_id.ravel(), int(d["buf_grain"]), h)
    s = int(d["buf_loop"])
    g = int(d["buf_grain"])
    assert ntri > 0 and vol == d["volume"][s, g] and sur == d["surface"][s, g]
    bri, rin = cube("REDIST_IN")
    bro, rout = cube("REDIST_OUT")
    assert np.array_equal(oracle.redistance_box(bri, rin, bro, h, delta), rout)


def test_resize_to_cube_cases(oracle):
    M = 52
    assert oracle.resize_to_cube((3, 13, 3, 13, 3, 13), M) == (3, 13, 3, 13, 3, 13)   # already cubic
    # y grows by 3: -1 below, +2 above (diff/2, diff/2 + diff%2)
    assert oracle.resize_to_cube((5, 15, 5, 12, 4, 14), M) == (5, 15, 4, 14, 4, 14)
    # y -1 and z -3 below 0: shifted up into the grid
    assert oracle.resize_to_cube((0, 10, 0, 7, 0, 4), M) == (0, 10, 0, 10, 0, 10)
    # y grows 18..28; x max 55 beyond grid_size 51: shifted down by 4
    assert oracle.resize_to_cube((45, 55, 20, 25, 0, 10), M) == (41, 51, 18, 28, 0, 10)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ggls_ref")),
                    reason="compiled reference not built")
def test_restatement_matches_reference_live(oracle):
    """A fresh seeded case through the compiled reference and the restatement."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import refdump
    from gragles_3d_b200 import microstructure as msgen

    N, G, border, steps = 36, 40, 6, 8
    ms = msgen.voronoi(N, G, seed=4242)
    with tempfile.TemporaryDirectory() as tmp:
        msgen.write_mode4(ms, tmp)
        msgen.write_parameters(os.path.join(tmp, "parameters.xml"), n_grains=G, border=border, steps=steps)
        res, _ = refdump.run_case(tmp, threads=4)
    ext, counts = ms.grain_extents()
    off = np.zeros(G + 2, np.int64)
    ids = []
    for g in range(1, G + 1):
        l = res["init_list"].get(g, np.zeros(0, np.uint32))
        ids.extend(l.tolist())
        off[g + 1] = off[g] + len(l)
    sim = oracle.OracleSim(N, border, 0.2, ms.labels, ext, counts, lists=(off, np.array(ids, np.uint32)))
    for g, r in res["init_sdf"].items():
        box, sdf = sim.sdf(g)
        assert box == r.box and np.array_equal(sdf.ravel(), r.data)
    for loop in range(steps + 1):
        sim.step()
        for g, (dat, box) in res["stats"][loop].items():
            inf = sim.info(g)
            assert inf["exists"] == (dat[0] == 1.0)
            if inf["exists"]:
                assert inf["box"] == box and inf["volume"] == dat[1] and inf["surface"] == dat[2]
                assert np.array_equal(sim.neighbors(g), res["neighbors"][loop][g])

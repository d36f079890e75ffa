"""3D hybrid path, CPU side: the oracle (oracle/hybrid_oracle.cpp) against the
reference's own 3d_hybrid_reconstruction outputs committed in
tests/golden/hybrid_small.npz (made by tests/golden/make_hybrid_golden.py),
the host-side file formats and generator of stripmlem.hybrid, and the C ABI
of include/hybridmlem.h (exports; no compute without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

GOLDEN = os.path.join(ROOT, "tests", "golden", "hybrid_small.npz")
HEADER = os.path.join(ROOT, "include", "hybridmlem.h")


def golden_inputs():
    from stripmlem import hybrid as hy
    z = np.load(GOLDEN)
    n, n_planes = (int(v) for v in z["setup"])
    p, z_left, length, s_z, s_dl = (float(v) for v in z["setup_f"])
    meta = z["m_meta"]
    m = hy.SystemMatrix(meta[0], meta[1], meta[2], z["m_lor_a"], z["m_lor_b"], z["m_px"],
                        z["m_py"], z["m_hits"])
    resp = tuple(z[k] for k in ("r_first", "r_second", "r_z_up", "r_z_dn", "r_dl"))
    centers = hy.detector_centers(z["polygons"])
    return z, (n, n_planes, p, z_left, length, s_z, s_dl), m, resp, centers


def oracle_setup(cfg):
    from oracle import hybrid as oh
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    return oh.setup(n, n, n_planes, p, z_left, length, s_z, s_dl)


@pytest.mark.parametrize("case,n_iter,kw", [
    ("calc", 3, {}),
    ("one", 2, {"sens_mode": "one"}),
    ("inactive", 2, {"inactive": [3, 40]}),
])
def test_oracle_reproduces_reference_bit_for_bit(case, n_iter, kw):
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    res = oh.reconstruct(oracle_setup(cfg), centers, m, resp, n_iter, **kw)
    ref = z[f"{case}_rho"]
    assert np.array_equal(res["rho"], ref), np.abs(res["rho"] - ref).max()
    st = res["stats"]
    assert [st["used_events"], st["used_pixels"], st["used_voxels"]] == list(z[f"{case}_counts"])


def test_fp64_oracle_close_to_reference():
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    res = oh.reconstruct(oracle_setup(cfg), centers, m, resp, 3, f64=True)
    ref = z["calc_rho"].astype(np.float64)
    rel = np.linalg.norm(res["rho"] - ref) / np.linalg.norm(ref)
    assert rel < 1e-5


def test_geometry_layout_and_frame_ranges():
    """Pixel infos sorted by position within each LOR; frame ranges inside
    the arrays, ending at most one info past their LOR (the reference's
    upper_bound + 1); planes inside the grid."""
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    s = oracle_setup(cfg)
    geo = oh.soa_from_matrix(s, centers, m)
    assert len(geo["pos"]) == len(m)
    for li in np.flatnonzero(geo["lend"] > geo["lbeg"])[::37]:
        seg = geo["pos"][geo["lbeg"][li]:geo["lend"][li]]
        assert np.all(np.diff(seg) >= 0)
    sens = oh.sensitivity(s, geo)
    w = oh.normalize(s, geo, sens)
    frames, keep = oh.frame_events(s, geo, w, *resp)
    assert len(frames) == keep.sum()
    ib, ie = frames["info_begin"], frames["info_end"]
    lor = frames["lor_index"]
    assert np.all(ib >= geo["lbeg"][lor]) and np.all(ie <= geo["lend"][lor] + 1)
    assert np.all(ie <= len(geo["pos"]))
    assert np.all(frames["plane_begin"] >= 0) and np.all(frames["plane_end"] <= s.n_planes)
    assert np.any(ie == geo["lend"][lor] + 1)  # the quirk occurs in practice


def test_responses_with_bad_lor_are_dropped():
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    s = oracle_setup(cfg)
    geo = oh.soa_from_matrix(s, centers, m)
    w = oh.normalize(s, geo, oh.sensitivity(s, geo))
    first = np.array([resp[0][0], 64, -1, 200], np.int16)
    second = np.array([resp[1][0], 0, 0, 3], np.int16)
    zz = np.zeros(4, np.float32)
    frames, keep = oh.frame_events(s, geo, w, first, second, zz + resp[2][0], zz + resp[3][0],
                                   zz + resp[4][0])
    assert keep.tolist() == [True, False, False, False]


def test_matrix_file_round_trip(tmp_path):
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    path = tmp_path / "m.bin"
    m.write(str(path))
    m2 = hy.SystemMatrix.read(str(path))
    assert (m2.n_pixels_in_row, m2.n_emissions, m2.n_detectors) == \
        (m.n_pixels_in_row, m.n_emissions, m.n_detectors)
    key = lambda a: np.lexsort((a.px, a.py, np.minimum(a.lor_a, a.lor_b),  # noqa: E731
                                np.maximum(a.lor_a, a.lor_b)))
    k1, k2 = key(m), key(m2)
    for f in ("px", "py", "hits"):
        assert np.array_equal(getattr(m, f)[k1], getattr(m2, f)[k2])
    raw = open(path, "rb").read()
    assert raw[:4] == b"PETP"


def test_response_and_detector_files_round_trip(tmp_path):
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    hy.write_responses(str(tmp_path / "r.bin"), *resp)
    assert os.path.getsize(tmp_path / "r.bin") == 16 * len(resp[0])
    back = hy.read_responses(str(tmp_path / "r.bin"))
    for a, b in zip(resp, back):
        assert np.array_equal(a, b)
    hy.write_detector_file(str(tmp_path / "d.txt"), z["polygons"])
    assert np.array_equal(hy.read_detector_file(str(tmp_path / "d.txt")), z["polygons"])
    hy.write_symmetry_file(str(tmp_path / "s.txt"), 4)
    lines = open(tmp_path / "s.txt").read().split("\n")
    assert lines[0] == "4 8" and lines[1].split() == ["0"] * 9


def test_host_generator_is_seeded_and_prefix_stable():
    from stripmlem import hybrid as hy
    b = hy.Barrel(radius=(0.15, 0.17), n_detectors=(32, 32), rotation=(0, 0.5),
                  w_detector=0.009, h_detector=0.015)
    ph = [(0.0, 0.0, 0.0, 0.1, 0.12, 1.0)]
    a = hy.generate_responses(b, ph, 4000, 0.3, 0.01, 0.04, seed=7)
    c = hy.generate_responses(b, ph, 1000, 0.3, 0.01, 0.04, seed=7)
    d = hy.generate_responses(b, ph, 1000, 0.3, 0.01, 0.04, seed=8)
    for x, y in zip(a, c):
        assert np.array_equal(x[:1000], y)
    assert not np.array_equal(a[2][:1000], d[2])
    first, second = a[0], a[1]
    assert np.all(first > second) and np.all(second >= 0) and np.all(first < 64)
    assert np.all(np.abs(a[2]) < 0.15 + 8 * 0.01)


def test_host_generator_rejects_bad_input():
    from stripmlem import hybrid as hy
    b = hy.Barrel(radius=(0.15,), n_detectors=(32,), rotation=(0,))
    with pytest.raises(hy.HybridError):
        hy.generate_responses(b, [(0, 0, 0, -0.1, 0.1, 1.0)], 10, 0.3, 0.01, 0.04)
    shuffled = hy.Barrel(radius=(0.15,), n_detectors=(32,), rotation=(0,))
    shuffled.polygons = shuffled.polygons[::-1].copy()[np.r_[5:32, 0:5]]
    shuffled.polygons[[3, 9]] = shuffled.polygons[[9, 3]]
    with pytest.raises(hy.HybridError):
        hy.generate_responses(shuffled, [(0, 0, 0, 0.1, 0.1, 1.0)], 10, 0.3, 0.01, 0.04)


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(hybrid_\w+)\s*\(", text,
                                 flags=re.M)))


def test_library_exports_every_hybrid_symbol(lib):
    from stripmlem import _lib
    names = declared_functions()
    assert "hybrid_iterate" in names and "hybrid_set_geometry_from_matrix" in names
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_hybrid_create_without_device_or_with_bad_setup(lib):
    from stripmlem import _lib
    ctx = ctypes.c_void_p()
    bad = _lib.HybridSetup(24, 24, 0, 0, 0.01, -0.12, 0.3, 0.01, 0.04)
    assert lib.hybrid_ctx_create(ctypes.byref(bad), 0, ctypes.byref(ctx)) == _lib.STRIP_E_INVALID
    assert lib.hybrid_ctx_destroy(None) == _lib.STRIP_E_INVALID
    if not gpu_available():
        good = _lib.HybridSetup(24, 24, 24, 0, 0.01, -0.12, 0.3, 0.01, 0.04)
        assert lib.hybrid_ctx_create(ctypes.byref(good), 0, ctypes.byref(ctx)) == \
            _lib.STRIP_E_NODEVICE
        assert not ctx.value


@pytest.mark.parametrize("case,kw", [("calc", {}), ("inactive", {"inactive": [3, 40]})])
def test_cli_naive_image_matches_reference(case, kw):
    """The drop-in CLI's naive image (Reconstruction::naive) from the kept
    responses equals the reference's rho.bin bit for bit."""
    from oracle import hybrid as oh
    from stripmlem import hybrid_cli
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left = cfg[0], cfg[1], cfg[2], cfg[3]
    res = oh.reconstruct(oracle_setup(cfg), centers, m, resp, 0, **kw)
    ll = -p * n / 2
    img = hybrid_cli.naive_image(np.flatnonzero(res["keep"]), resp, n, n, n_planes, p, ll, ll,
                                 z_left, hybrid_cli.lor_segments(centers))
    assert np.array_equal(img, z[f"{case}_naive"])


def test_cli_naive_image_non_square_grid():
    """A grid of nc != nr (the --geometry path): x bins by columns, y by
    rows, each from its own lower-left coordinate; the image is
    (n_planes, nr, nc).  Cropping the golden square grid to fewer rows keeps
    every count of the rows inside and drops the rest."""
    from oracle import hybrid as oh
    from stripmlem import hybrid_cli
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left = cfg[0], cfg[1], cfg[2], cfg[3]
    res = oh.reconstruct(oracle_setup(cfg), centers, m, resp, 0)
    kept = np.flatnonzero(res["keep"])
    segs = hybrid_cli.lor_segments(centers)
    ll = -p * n / 2
    full = hybrid_cli.naive_image(kept, resp, n, n, n_planes, p, ll, ll, z_left, segs)
    r0, nr = 5, n - 9  # rows [5, n - 4): lower-left y moves up by 5 pixels
    crop = hybrid_cli.naive_image(kept, resp, n, nr, n_planes, p, ll, ll + r0 * p, z_left, segs)
    assert crop.shape == (n_planes, nr, n)
    assert np.array_equal(crop, full[:, r0:r0 + nr, :])


def test_cli_writes_reference_file_layout(tmp_path):
    from stripmlem import hybrid_cli
    data = np.arange(2 * 3 * 4, dtype=np.float32).reshape(4, 3, 2)
    hybrid_cli._write_map(str(tmp_path / "rho_07"), ".bin", data, (2, 3, 4), "float")
    assert np.array_equal(np.fromfile(tmp_path / "rho_07.bin", np.float32), data.reshape(-1))
    hdr = open(tmp_path / "rho_07.nrrd").read()
    assert "type: float" in hdr and "sizes: 2 3 4" in hdr and "data file: ./rho_07.bin" in hdr
    hybrid_cli._write_map(str(tmp_path / "naive"), ".txt", data.astype(np.int32), (2, 3, 4), "int")
    lines = open(tmp_path / "naive.txt").read().split("\n")
    assert lines[0] == "0 1" and len([x for x in lines if x]) == 12
    a = hybrid_cli.parse(["--system", "m", "--detector-file", "d", "-p", "0.004", "-i", "2",
                          "-I", "5", "--inactive", "3,40", "r.bin"])
    assert (a.blocks, a.iterations, a.responses) == (2, 5, ["r.bin"])
    assert hybrid_cli._ints(a.inactive) == [3, 40]


def test_text_responses_parse_as_the_reference(tmp_path):
    """Text responses (mixed number formats) read by the library's statement
    of the reference's fast text parser (hybrid_parse_responses_text)
    reproduce the reference's image from the same file bit for bit through
    the oracle."""
    from oracle import hybrid as oh
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    path = tmp_path / "r.txt"
    path.write_text(str(z["text_in"]))
    parsed = hy.read_responses(str(path))
    assert np.array_equal(parsed[0], resp[0]) and np.array_equal(parsed[1], resp[1])
    res = oh.reconstruct(oracle_setup(cfg), centers, m, parsed, 3)
    assert np.array_equal(res["rho"], z["text_rho"])
    st = res["stats"]
    assert [st["used_events"], st["used_pixels"], st["used_voxels"]] == list(z["text_counts"])


def test_text_responses_malformed_line_reported(tmp_path):
    from stripmlem import hybrid as hy
    path = tmp_path / "bad.txt"
    path.write_text("1 0 1.5 -2 30\n3 2 1e2 . 4\n")
    with pytest.raises(ValueError, match="line 2"):
        hy.read_responses(str(path))
    path.write_text("70000 -1 1.5 -2 30\n4 3 2 1 0")  # last line unterminated
    f, s_, zu, zd, dl = hy.read_responses(str(path))
    assert len(f) == 1 and f[0] == np.int16(70000 - 65536) and s_[0] == -1
    assert zu[0] == np.float32(1.5) and dl[0] == np.float32(30)


def test_geometry_file_path_reproduces_reference(tmp_path):
    """--geometry: a LOR geometry file read and flattened by stripmlem.hybrid
    (GeometrySOA(Geometry) and load_weights_from_matrix_file) reproduces the
    reference's image from the same file bit for bit through the oracle."""
    import sys
    from oracle import hybrid as oh
    from stripmlem import hybrid as hy
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_hybrid_golden as mk
    z, cfg, m, resp, centers = golden_inputs()

    class B:
        pass
    b = B()
    b.centers, b.n_detectors = centers, len(centers)
    path = str(tmp_path / "g.bin")
    mk.write_golden_geometry(path, b, m)
    soa = hy.geometry_soa_from_file(hy.read_geometry(path), m)
    s = oracle_setup(cfg)
    geo = oh.geo_from_soa(soa)
    sens = oh.sensitivity(s, geo)
    w = oh.normalize(s, geo, sens)
    frames, keep = oh.frame_events(s, geo, w, *resp)
    img, st = oh.mlem(s, geo, w, sens, frames, 3)
    assert np.array_equal(img, z["geom_rho"])
    assert [st["used_events"], st["used_pixels"], st["used_voxels"]] == list(z["geom_counts"])

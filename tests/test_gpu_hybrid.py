"""3D hybrid path on the GPU, through the C ABI (include/hybridmlem.h):

* the flattened LOR geometry equals the oracle's bit for bit (pixel infos,
  positions, LOR ranges, segments);
* the device sensitivity equals the oracle's binary32 sum to its rounding;
* frame events (LOR, pixel-info range, plane range, kept responses) equal
  the oracle's bit for bit;
* images are within 1e-4 relative L2 of the FP64 oracle and of the
  reference's own images (tests/golden/hybrid_small.npz);
* the device response generator equals the host generator."""
import os

import numpy as np
import pytest

from test_hybrid_oracle import golden_inputs, oracle_setup

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative L2 of images against the FP64 oracle


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def f32_live(s, geo, w, sens, frames):
    """Frames whose binary32 denominator is positive at rho = 1.  Where the
    kernel underflows binary32 on every voxel of an event (a lone pixel
    info far from the TOF position, e.g. the one info the reference's
    upper_bound + 1 takes from the next LOR), the reference and the device
    drop the event while a binary64 evaluation keeps it; the FP64
    comparison leaves such events out."""
    from oracle import hybrid as oh
    keep = np.ones(len(frames), bool)
    for e in range(len(frames)):
        img, _ = oh.mlem(s, geo, w, sens, frames[e:e + 1], 1)
        keep[e] = img.any()
    return frames[keep]


def device_rec(cfg, centers, m, sens="calculate", inactive=None):
    from stripmlem import hybrid as hy
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    rec = hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl)
    rec.set_geometry_from_matrix(centers, m, inactive)
    rec.set_sensitivity(sens)
    return rec


@pytest.mark.parametrize("case,n_iter,kw", [
    ("calc", 3, {}),
    ("one", 2, {"sens": "one"}),
    ("inactive", 2, {"inactive": [3, 40]}),
])
def test_golden_cases(case, n_iter, kw):
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    s = oracle_setup(cfg)
    with device_rec(cfg, centers, m, **kw) as rec:
        geo_d = rec.geometry()
        ora = oh.reconstruct(s, centers, m, resp, n_iter,
                             sens_mode=kw.get("sens", "calculate"),
                             inactive=kw.get("inactive"))
        geo = ora["geo"]
        for k in ("pix", "pos", "lbeg", "lend", "seg"):
            assert np.array_equal(geo_d[k], geo[k], equal_nan=True), k
        sens_d = rec.sensitivity
        assert np.allclose(sens_d, ora["sens"], rtol=2e-6, atol=0)
        rec.set_responses(*resp)
        fr = rec.frames()
        of = ora["frames"]
        assert len(fr["lor"]) == len(of)
        assert np.array_equal(fr["lor"], of["lor_index"])
        assert np.array_equal(fr["info_begin"], of["info_begin"])
        assert np.array_equal(fr["info_end"], of["info_end"])
        assert np.array_equal(fr["plane_begin"], of["plane_begin"])
        assert np.array_equal(fr["plane_end"], of["plane_end"])
        assert np.array_equal(fr["index"], np.flatnonzero(ora["keep"]))
        st = rec.stats()
        assert [st["n_events"], st["used_pixels"], st["used_voxels"]] == \
            list(z[f"{case}_counts"])
        rec(n_iter)
        img = rec.rho
        # FP64 oracle from the device's own normalised weights and sensitivity
        live = f32_live(s, geo, geo_d["w"], sens_d, of)
        f64, _ = oh.mlem(s, geo, geo_d["w"], sens_d, live, n_iter, f64=True)
    assert rel_l2(img, f64) < TOL
    assert rel_l2(img, z[f"{case}_rho"]) < TOL


def test_big_barrel_against_fp64_oracle():
    """The default big-barrel geometry (three rings, 192 detectors) on a
    coarse 60 x 60 grid of 1.2 cm pixels, 40 planes; 20000 responses."""
    from oracle import hybrid as oh
    from stripmlem import hybrid as hy
    b = hy.Barrel()
    n, p, n_planes = 60, 0.012, 40
    z_left, length, s_z, s_dl = -0.24, 0.5, 0.015, 0.06
    m = hy.synthetic_matrix(b, n, p, 0.36)
    ph = [(0.1, 0.05, 0.02, 0.05, 0.05, 3.0), (0, 0, 0, 0.3, 0.2, 1.0)]
    resp = hy.generate_responses(b, ph, 20000, length, s_z, s_dl, seed=9)
    cfg = (n, n_planes, p, z_left, length, s_z, s_dl)
    s = oracle_setup(cfg)
    with device_rec(cfg, b.centers, m) as rec:
        rec.set_responses(*resp)
        rec(3)
        img = rec.rho
        g = rec.geometry()
        sens = rec.sensitivity
        fr = rec.frames()
    geo = oh.soa_from_matrix(s, b.centers, m)
    frames, keep = oh.frame_events(s, geo, g["w"], *resp)
    assert np.array_equal(fr["info_end"], frames["info_end"])
    assert np.array_equal(fr["index"], np.flatnonzero(keep))
    f64, _ = oh.mlem(s, geo, g["w"], sens, f32_live(s, geo, g["w"], sens, frames), 3,
                     f64=True)
    assert rel_l2(img, f64) < TOL


def test_image_round_trip_and_restart():
    """set_image / get_image keep the boundary layout; running 2 + 1
    iterations equals 3 (the image carries the state)."""
    z, cfg, m, resp, centers = golden_inputs()
    with device_rec(cfg, centers, m) as a, device_rec(cfg, centers, m) as b:
        x = np.random.default_rng(1).random(a.shape).astype(np.float32)
        a.rho = x
        assert np.array_equal(a.rho, x)
        a.rho = np.ones(a.shape, np.float32)
        a.set_responses(*resp)
        b.set_responses(*resp)
        a(2)
        mid = a.rho
        a(1)
        b.rho = mid
        b(1)
        assert rel_l2(b.rho, a.rho) < 1e-6


def test_empty_and_dropped_responses():
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    with device_rec(cfg, centers, m) as rec:
        rec.set_responses(*(r[:0] for r in resp))
        assert rec.stats()["n_events"] == 0
        rec(1)
        assert not rec.rho.any()  # nothing back-projected
        zz = np.zeros(3, np.float32)
        rec.set_responses(np.array([64, -1, 300], np.int16), np.array([0, 0, 2], np.int16),
                          zz, zz, zz)
        assert rec.stats()["n_events"] == 0
        from stripmlem import _lib
        assert rec.lib.hybrid_set_responses(rec._ctx, None, None, None, None, None, 1) == \
            _lib.STRIP_E_INVALID


def test_calls_out_of_order_rejected():
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    with hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as rec:
        with pytest.raises(hy.HybridError):
            rec.set_responses(*resp)
        with pytest.raises(hy.HybridError):
            rec.set_sensitivity()


def test_device_generator_equals_host_generator():
    from stripmlem import hybrid as hy
    b = hy.Barrel()
    ph = [(0.1, 0.05, 0.02, 0.05, 0.05, 3.0), (0, 0, 0, 0.3, 0.2, 1.0)]
    h = hy.generate_responses(b, ph, 50000, 0.5, 0.015, 0.06, seed=3, device=-1)
    d = hy.generate_responses(b, ph, 50000, 0.5, 0.015, 0.06, seed=3, device=0)
    same = (h[0] == d[0]) & (h[1] == d[1])
    assert same.mean() > 0.999  # libm and CUDA sin / cos / log may round apart
    for a, c in zip(h[2:], d[2:]):
        assert np.allclose(a[same], c[same], rtol=0, atol=1e-5)



def test_geometry_soa_and_frames_entry_points():
    """The GPU run()'s inputs: the oracle's flattened geometry with its
    normalised weights and sensitivity (HYBRID_SENS_GIVEN) and its frame
    events reproduce the reference's image."""
    from oracle import hybrid as oh
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    s = oracle_setup(cfg)
    ora = oh.reconstruct(s, centers, m, resp, 0)
    geo, fr = ora["geo"], ora["frames"]
    with hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as rec:
        rec.set_geometry_soa(len(centers), geo["seg"][:, :4], geo["pix"], geo["pos"], ora["w"],
                             geo["lbeg"], geo["lend"])
        rec.set_sensitivity(ora["sens"], given=True)
        g = rec.geometry()
        assert np.array_equal(g["seg"], geo["seg"], equal_nan=True)
        assert np.array_equal(g["w"], ora["w"])
        rec.set_frames(fr["lor_index"], fr["info_begin"], fr["info_end"], fr["plane_begin"],
                       fr["plane_end"], fr["up"], fr["right"], fr["tan"], fr["sec"])
        assert rec.stats()["used_voxels"] == int(z["calc_counts"][2])
        rec(3)
        img = rec.rho
    assert rel_l2(img, z["calc_rho"]) < TOL


@pytest.mark.parametrize("case,n_iter,extra", [("calc", 3, []), ("inactive", 2, ["--inactive", "3,40"]),
                                               ("one", 2, ["--sens-to-one"])])
def test_cli_drop_in(tmp_path, case, n_iter, extra):
    """python -m stripmlem.hybrid_cli with the reference's flags on the
    reference's file formats: the naive image bit for bit, the iterated image
    within 1e-4 of the reference's own, the reference's output names."""
    from stripmlem import hybrid as hy
    from stripmlem import hybrid_cli
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    m.write(str(tmp_path / "m.bin"))
    hy.write_detector_file(str(tmp_path / "det.txt"), z["polygons"])
    hy.write_symmetry_file(str(tmp_path / "sym.txt"), len(z["polygons"]))
    hy.write_responses(str(tmp_path / "r.bin"), *resp)
    out = str(tmp_path / "rho.bin")
    rc = hybrid_cli.main(["--system", str(tmp_path / "m.bin"),
                          "--detector-file", str(tmp_path / "det.txt"),
                          "--detector-file-sym", str(tmp_path / "sym.txt"),
                          "-n", str(n), "-p", repr(p), "--n-planes", str(n_planes),
                          "--z-left", repr(z_left), "--length", repr(length), "--s-z", repr(s_z),
                          "--s-dl", repr(s_dl), "-i", "1", "-I", str(n_iter), "-o", out, *extra,
                          str(tmp_path / "r.bin")])
    assert rc == 0
    naive = np.fromfile(out, np.int32).reshape(n_planes, n, n)
    assert np.array_equal(naive, z[f"{case}_naive"])
    img = np.fromfile(str(tmp_path / f"rho_{n_iter}.bin"), np.float32).reshape(n_planes, n, n)
    assert rel_l2(img, z[f"{case}_rho"]) < TOL
    assert (tmp_path / f"rho_{n_iter}.nrrd").exists() and (tmp_path / "rho.nrrd").exists()


def test_twenty_iterations_against_fp64_oracle():
    """20 iterations on the golden case stay within 1e-4 of the FP64 oracle."""
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    s = oracle_setup(cfg)
    with device_rec(cfg, centers, m) as rec:
        rec.set_responses(*resp)
        rec(20)
        img = rec.rho
        g = rec.geometry()
        sens = rec.sensitivity
    ora = oh.reconstruct(s, centers, m, resp, 0)
    live = f32_live(s, ora["geo"], g["w"], sens, ora["frames"])
    f64, _ = oh.mlem(s, ora["geo"], g["w"], sens, live, 20, f64=True)
    assert rel_l2(img, f64) < TOL


def test_cli_text_responses(tmp_path):
    """The CLI on a text responses file (mixed number formats): within 1e-4
    of the reference's image from the same text file."""
    from stripmlem import hybrid as hy
    from stripmlem import hybrid_cli
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    m.write(str(tmp_path / "m.bin"))
    hy.write_detector_file(str(tmp_path / "det.txt"), z["polygons"])
    (tmp_path / "r.txt").write_text(str(z["text_in"]))
    out = str(tmp_path / "rho.bin")
    assert hybrid_cli.main(["--system", str(tmp_path / "m.bin"),
                            "--detector-file", str(tmp_path / "det.txt"), "-n", str(n),
                            "-p", repr(p), "--n-planes", str(n_planes), "--z-left", repr(z_left),
                            "--length", repr(length), "--s-z", repr(s_z), "--s-dl", repr(s_dl),
                            "-i", "1", "-I", "3", "-o", out, str(tmp_path / "r.txt")]) == 0
    img = np.fromfile(str(tmp_path / "rho_3.bin"), np.float32).reshape(n_planes, n, n)
    assert rel_l2(img, z["text_rho"]) < TOL


def test_cli_geometry_file(tmp_path):
    """The CLI's --geometry path (a LOR geometry file, weights from the
    matrix): within 1e-4 of the reference's image from the same files."""
    import sys
    from stripmlem import hybrid as hy
    from stripmlem import hybrid_cli
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_hybrid_golden as mk
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg

    class B:
        pass
    b = B()
    b.centers, b.n_detectors = centers, len(centers)
    mk.write_golden_geometry(str(tmp_path / "g.bin"), b, m)
    m.write(str(tmp_path / "m.bin"))
    hy.write_responses(str(tmp_path / "r.bin"), *resp)
    out = str(tmp_path / "rho.bin")
    assert hybrid_cli.main(["--system", str(tmp_path / "m.bin"), "--geometry",
                            str(tmp_path / "g.bin"), "--n-planes", str(n_planes),
                            "--z-left", repr(z_left), "--length", repr(length), "--s-z", repr(s_z),
                            "--s-dl", repr(s_dl), "-i", "1", "-I", "3", "-o", out,
                            str(tmp_path / "r.bin")]) == 0
    img = np.fromfile(str(tmp_path / "rho_3.bin"), np.float32).reshape(n_planes, n, n)
    assert rel_l2(img, z["geom_rho"]) < TOL

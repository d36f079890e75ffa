"""The drop-in 2d_strip_reconstruction command (j-pet-mlem-old_b200/bin/):
option surface, .cfg loading, the reference's text-event parsing, output
names and formats.  The GPU tests run whole reconstructions through it."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT
from oracle import oracle as orc

CLI = os.path.join(PKG, "bin", "2d_strip_reconstruction")
PHANTOM_CLI = os.path.join(PKG, "bin", "2d_strip_phantom")
GOLD = os.path.join(ROOT, "tests", "golden")
C1_ARGS = ["-r", "200", "-l", "500", "-p", "2", "--s-z", "10", "--s-dl", "42"]
C1_PHANTOM_T = [(40, 30, 30, 20, 0, 3.0), (-50, -20, 25, 40, 0, 0.3), (0, 0, 150, 100, 0, 1.0)]


def run_cli(*args, cwd=None, check=True):
    p = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, cwd=cwd,
                       timeout=600)
    if check and p.returncode != 0:
        raise AssertionError(f"CLI failed ({p.returncode}): {p.stderr}")
    return p


def dump(tmp_path, *args):
    out = tmp_path / "dump.bin"
    run_cli(*args, "--dump-responses", out)
    return np.fromfile(out, dtype="<f4").reshape(-1, 3)


def test_help_lists_reference_options():
    p = run_cli("--help")
    for opt in ("--radius", "--length", "--s-pixel", "--n-pixels", "--n-z-pixels",
                "--n-y-pixels", "--s-z", "--s-dl", "--blocks", "--iterations", "--output",
                "--rho", "--rho-is-int", "--3d-response", "--dl-is-time",
                "--speed-of-light", "--scale-length", "--scale-time", "--png-max", "--gpu",
                "--cuda-device", "--config", "--verbose", "--n-threads"):
        assert opt in p.stderr, opt


def test_errors_are_reported():
    p = run_cli("-i", "1", check=False)
    assert p.returncode == 1 and "at least one responses input file" in p.stderr
    p = run_cli("--no-such-option", "x.bin", check=False)
    assert p.returncode == 1 and "undefined option" in p.stderr


def test_text_events_parse_like_the_reference(tmp_path):
    """--dump-responses of the text fixture, reconstructed by the oracle's
    binary32 restatement, is bit-identical to the reference's own output on
    the text file: the parsed values are the reference's."""
    t = dump(tmp_path, os.path.join(GOLD, "text.events.txt"), *C1_ARGS)
    assert t.shape[0] == 1499  # the unterminated last line is not read
    assert t[7, 0] == np.float32(1.5) and t[7, 1] == np.float32(-20.0)  # 1.5e2 -> 1.5
    g = orc.geometry(200, 500, 200, 250, 2, 2, 10, 42)
    img = orc.mlem_f32(g, t[:, 0], t[:, 1], t[:, 2], 1)
    ref = np.load(os.path.join(GOLD, "text.ref1.npz"))["nocontract"]
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))


def test_binary_events_and_unit_scaling(tmp_path):
    src = os.path.join(GOLD, "c1_small.events.bin")
    raw = np.fromfile(src, dtype="<f4").reshape(-1, 3)
    assert np.array_equal(dump(tmp_path, src, *C1_ARGS), raw)
    s = dump(tmp_path, src, *C1_ARGS, "--scale-length", "10")
    assert np.array_equal(s, (raw.astype(np.float64) * 10).astype(np.float32))
    d = dump(tmp_path, src, *C1_ARGS, "--dl-is-time", "--scale-time", "1e-12",
             "--speed-of-light", "299792458000")
    assert np.array_equal(d[:, :2], raw[:, :2])
    assert np.array_equal(d[:, 2], (raw[:, 2].astype(np.float64) * 299792458000 * 1e-12)
                          .astype(np.float32))


def test_accompanying_and_included_config(tmp_path):
    src = os.path.join(GOLD, "c1_small.events.bin")
    ev = tmp_path / "ev.bin"
    ev.write_bytes(open(src, "rb").read())
    inc = tmp_path / "sub"
    inc.mkdir()
    (inc / "scale.cfg").write_text("# included\n--scale-length=2\n")
    (tmp_path / "ev.cfg").write_text("--s-z=10\n-c\nsub/scale.cfg\n--output=ignored\n")
    raw = np.fromfile(src, dtype="<f4").reshape(-1, 3)
    out = tmp_path / "d.bin"
    run_cli(ev, "--dump-responses", out, cwd=tmp_path)
    d = np.fromfile(out, dtype="<f4").reshape(-1, 3)
    assert np.array_equal(d, (raw.astype(np.float64) * 2).astype(np.float32))


@pytest.mark.gpu
def test_cpu_semantics_outputs_match_reference(tmp_path):
    src = os.path.join(GOLD, "c1_small.events.bin")
    p = run_cli(src, *C1_ARGS, "-i", "1", "-I", "3", "-o", tmp_path / "r.bin", "-vv")
    for name in ("r_sensitivity.png", "r_3.bin", "r_3.nrrd", "r_3.png"):
        assert (tmp_path / name).exists(), name
    img = np.fromfile(tmp_path / "r_3.bin", dtype="<f4").reshape(200, 250)
    ref = np.load(os.path.join(GOLD, "c1_small.ref3.npz"))["nocontract"]
    assert np.linalg.norm(img - ref) / np.linalg.norm(ref) < 1e-5
    assert "# it     time (ms)" in p.stdout
    assert re.search(r"^# av\s+[0-9.]+\s+total", p.stdout, flags=re.M)
    assert len(re.findall(r"^\s+\d+\s+[0-9.]+$", p.stdout, flags=re.M)) == 3
    nrrd = (tmp_path / "r_3.nrrd").read_text()
    assert "sizes: 250 200" in nrrd and "data file: ./r_3.bin" in nrrd
    assert (tmp_path / "r_3.png").read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"
    # text tuples
    run_cli(src, *C1_ARGS, "-i", "1", "-I", "1", "-o", tmp_path / "t.txt")
    first = (tmp_path / "t_1.txt").read_text().splitlines()[0].split()
    assert len(first) == 3 and re.match(r"^\d+\.\d{12}$", first[2])


@pytest.mark.gpu
def test_gpu_semantics_output_schedule(tmp_path):
    src = os.path.join(GOLD, "c1_small.events.bin")
    run_cli(src, *C1_ARGS, "-i", "2", "-I", "3", "-o", tmp_path / "g.bin", "-G")
    names = sorted(os.listdir(tmp_path))
    for name in ("g_sensitivity.bin", "g_sensitivity.nrrd", "g_sensitivity.png",
                 "g_1.bin", "g_2.bin", "g_3.bin", "g_6.bin"):
        assert name in names, (name, names)
    sens = np.fromfile(tmp_path / "g_sensitivity.bin", dtype="<f4").reshape(200, 250)
    g = orc.geometry(200, 500, 200, 250, 2, 2, 10, 42)
    ref = orc.sensitivity_image_f32(g, five_point=True)
    assert np.max(np.abs(sens - ref)) < 1e-5
    ev = np.fromfile(src, dtype="<f4").reshape(-1, 3)
    img = np.fromfile(tmp_path / "g_6.bin", dtype="<f4").reshape(200, 250)
    r64 = orc.mlem_f64(g, ev[:, 0], ev[:, 1], ev[:, 2], 6, mode=orc.MODE_GPU)
    assert np.linalg.norm(img - r64) / np.linalg.norm(r64) < 1e-4


def run_phantom(*args, cwd=None, check=True):
    p = subprocess.run([PHANTOM_CLI, *map(str, args)], capture_output=True, text=True,
                       cwd=cwd, timeout=600)
    if check and p.returncode != 0:
        raise AssertionError(f"phantom CLI failed ({p.returncode}): {p.stderr}")
    return p


def test_phantom_cli_options_and_errors(tmp_path):
    p = run_phantom("--help")
    for opt in ("--scale", "--additive", "--detected", "--point", "--image-origin",
                "--n-emissions", "--output", "--s-z", "--s-dl", "--seed"):
        assert opt in p.stderr, opt
    bad = tmp_path / "bad"
    bad.write_text("ellipse 0 0 10 10 0 1\ntriangle 0 0 1\n")
    p = run_phantom(bad, "-e", "10", "-o", tmp_path / "x.bin", check=False)
    assert p.returncode == 1 and "unknown phantom type: triangle" in p.stderr


@pytest.mark.gpu
def test_phantom_cli_detected_stream_matches_generator(tmp_path):
    """--detected --uniform-tan with ellipses is the library's generator:
    the same events as stripmlem.generate_events for the same seed."""
    import stripmlem as sm
    ph = tmp_path / "c1_phantom"
    ph.write_text("".join(f"ellipse {z} {y} {a} {b} {ang} {act}\n"
                          for z, y, a, b, ang, act in C1_PHANTOM_T))
    out = tmp_path / "p.bin"
    p = run_phantom(ph, *C1_ARGS, "-e", "20k", "--detected", "--uniform-tan", "--seed", "7",
                    "-o", out, "-v")
    assert "detected: 20000 events" in p.stderr
    ev = np.fromfile(out, dtype="<f4").reshape(-1, 3)
    sc = sm.Scanner(200.0, 500.0, 200, 250, 2.0, 2.0, 10.0, 42.0)
    ref = np.stack(sm.generate_events(sc, C1_PHANTOM_T, 20000, seed=7), 1)
    same = np.all(ev.view(np.uint32) == ref.view(np.uint32), axis=1)
    assert same.mean() >= 1 - 1e-4
    cfg = (tmp_path / "p.cfg").read_text()
    for line in ("--radius=200", "--length=500", "--s-pixel=2", "--s-z=10", "--s-dl=42",
                 "--n-z-pixels=250", "--n-y-pixels=200"):
        assert line in cfg, (line, cfg)
    det = np.fromfile(tmp_path / "p_detected", dtype="<i4").reshape(200, 250)
    assert det.sum() == 20000  # every emission point lies on the image grid
    emi = np.fromfile(tmp_path / "p_emitted", dtype="<i4").reshape(200, 250)
    assert emi.sum() > det.sum()
    naive = np.fromfile(tmp_path / "p_naive", dtype="<i4").reshape(200, 250)
    assert 0.9 * 20000 < naive.sum() <= 20000
    assert "type: int" in (tmp_path / "p_detected.nrrd").read_text()
    # the reconstruction reads the accompanying .cfg
    r = run_cli(out, "-i", "1", "-I", "2", "-o", tmp_path / "r.bin", "-v")
    img = np.fromfile(tmp_path / "r_2.bin", dtype="<f4").reshape(200, 250)
    assert np.isfinite(img).all() and img.sum() > 0


@pytest.mark.gpu
def test_phantom_cli_emissions_and_shapes(tmp_path):
    ph = tmp_path / "shapes"
    ph.write_text("rectangle 0 0 60 40 1\nellipse 30 10 20 10 30 2\npoint 10 20 5000\n"
                  "ellipse 1 2 3\nellipse 0 0 100 100 0 1\n")  # the malformed line ends the file
    out = tmp_path / "e.txt"
    p = run_phantom(ph, *C1_ARGS, "-e", "30000", "--additive", "-o", out, "-v",
                    "--scale", "2")
    assert " emitted: 30000 events" in p.stderr
    lines = out.read_text().splitlines()
    n_det = int(p.stderr.split("detected:")[1].split()[0])
    assert len(lines) == n_det and 0 < n_det < 30000
    assert len(lines[0].split()) == 3
    emi = np.fromfile(tmp_path / "e_emitted", dtype="<i4").reshape(200, 250)
    # scale 2: the rectangle spans |z| <= 120, |y| <= 80 mm; nothing outside
    rows = np.nonzero(emi.sum(1))[0]
    cols = np.nonzero(emi.sum(0))[0]
    assert cols.min() >= 125 - 60 - 1 and cols.max() <= 125 + 60
    assert rows.min() >= 100 - 40 - 1 and rows.max() <= 100 + 40
    # the point source (not scaled) holds its share: weight 5000 vs 4*120*80 + pi*40*20*2
    total_w = 4 * 120 * 80 + np.pi * 40 * 20 * 2 + 5000
    z, y = 10.0, 20.0
    col, row = int(np.floor((z + 250) / 2)), int(np.floor((y + 200) / 2))
    assert emi[row, col] > 0.8 * 30000 * 5000 / total_w


REF_PHANTOM = os.path.join(ROOT, "oracle", "_ref", "2d_strip_phantom")


def _two_sample_chi2(a, b, min_count=20):
    """Chi-squared two-sample test of two histograms with the same bins
    (bins holding fewer than min_count events together are pooled)."""
    from scipy import stats
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    keep = (a + b) >= min_count
    a = np.append(a[keep], a[~keep].sum())
    b = np.append(b[keep], b[~keep].sum())
    if a[-1] + b[-1] == 0:
        a, b = a[:-1], b[:-1]
    ka, kb = np.sqrt(b.sum() / a.sum()), np.sqrt(a.sum() / b.sum())
    chi2 = float(np.sum((ka * a - kb * b) ** 2 / (a + b)))
    return chi2, float(stats.chi2.sf(chi2, len(a) - 1))


@pytest.mark.gpu
@pytest.mark.skipif(not os.access(REF_PHANTOM, os.X_OK),
                    reason="the reference's 2d_strip_phantom was not built")
def test_phantom_cli_matches_reference_generator_in_distribution(tmp_path):
    """The drop-in 2d_strip_phantom (Philox streams, on the GPU) against the
    reference's own (tausworthe, src/2d/strip/phantom_cmd.cpp; the Monte
    Carlo of src/common/phantom_monte_carlo.h:29-109 and
    src/2d/geometry/phantom.h:183-215, uniform emission angle) on the same
    phantom and options: 1e6 detected events each, two-sample
    Kolmogorov-Smirnov tests on z_u, z_d and dl and chi-squared tests on the
    detected- and emitted-point images.  Both runs are seeded (the
    reference's generators are default-seeded with one thread), so the test
    is deterministic; the bar is p > 1e-3."""
    from scipy import stats
    ph = tmp_path / "phantom"
    ph.write_text("".join(f"ellipse {z} {y} {a} {b} {ang} {act}\n"
                          for z, y, a, b, ang, act in C1_PHANTOM_T)
                  + "rectangle -120 -60 20 15 0.5\n")
    n = 1_000_000
    ref = subprocess.run([REF_PHANTOM, str(ph), *C1_ARGS, "-e", str(n), "--detected",
                          "-T", "1", "-o", str(tmp_path / "ref.bin")],
                         capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert ref.returncode == 0, ref.stderr[-500:]
    run_phantom(ph, *C1_ARGS, "-e", n, "--detected", "--seed", "3",
                "-o", tmp_path / "ours.bin")
    a = np.fromfile(tmp_path / "ref.bin", dtype="<f4").reshape(-1, 3)
    b = np.fromfile(tmp_path / "ours.bin", dtype="<f4").reshape(-1, 3)
    assert abs(a.shape[0] - n) <= 64 and b.shape[0] == n
    for k, name in enumerate(("z_u", "z_d", "dl")):
        p = stats.ks_2samp(a[:, k], b[:, k]).pvalue
        assert p > 1e-3, (name, p)
    for img in ("detected", "emitted"):
        ia = np.fromfile(tmp_path / f"ref_{img}", dtype="<i4")
        ib = np.fromfile(tmp_path / f"ours_{img}", dtype="<i4")
        assert ia.shape == ib.shape
        _, p = _two_sample_chi2(ia, ib)
        assert p > 1e-3, (img, p)

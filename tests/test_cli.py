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
GOLD = os.path.join(ROOT, "tests", "golden")
C1_ARGS = ["-r", "200", "-l", "500", "-p", "2", "--s-z", "10", "--s-dl", "42"]


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

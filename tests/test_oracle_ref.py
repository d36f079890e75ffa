"""Pins the oracle's binary32 restatement to the reference itself: the
committed fixtures in tests/golden/ were produced by the reference's own
2d_strip_reconstruction (tests/golden/make_golden.py); when oracle/_ref holds
the reference binaries (built here from the reference sources) the
comparison also runs live on fresh inputs.  CPU only."""
import os

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
C1 = (200.0, 500.0, 200, 250, 2.0, 2.0, 10.0, 42.0)
METRE = (0.5, 1.0, 100, 100, 0.01, 0.01, 0.015, 0.06)


def load_events(name):
    t = np.fromfile(os.path.join(GOLD, name), dtype="<f4").reshape(-1, 3)
    return t[:, 0].copy(), t[:, 1].copy(), t[:, 2].copy()


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def test_oracle_f32_bit_identical_to_reference_c1():
    g = orc.geometry(*C1)
    zu, zd, dl = load_events("c1_small.events.bin")
    ref = np.load(os.path.join(GOLD, "c1_small.ref3.npz"))["nocontract"]
    mine = orc.mlem_f32(g, zu, zd, dl, 3)
    assert bits_equal(mine, ref)


def test_oracle_f32_bit_identical_to_reference_edge_events():
    g = orc.geometry(*C1)
    zu, zd, dl = load_events("edge.events.bin")
    ref = np.load(os.path.join(GOLD, "edge.ref1.npz"))["nocontract"]
    mine = orc.mlem_f32(g, zu, zd, dl, 1)
    assert bits_equal(mine, ref)


def test_oracle_f32_bit_identical_to_reference_metre_units():
    g = orc.geometry(*METRE)
    zu, zd, dl = load_events("metre.events.bin")
    ref = np.load(os.path.join(GOLD, "metre.ref2.npz"))["nocontract"]
    mine = orc.mlem_f32(g, zu, zd, dl, 2)
    assert bits_equal(mine, ref)


def test_fma_contraction_changes_few_pixels():
    """GCC's default contraction (the reference's shipped flags) moves a few
    boundary pixels; the images still agree far inside the 1e-4 tolerance."""
    d = np.load(os.path.join(GOLD, "c1_small.ref3.npz"))
    nc, df = d["nocontract"].astype(np.float64), d["default"].astype(np.float64)
    rel = np.linalg.norm(nc - df) / np.linalg.norm(nc)
    assert rel < 1e-4


def test_oracle_f64_close_to_reference():
    g = orc.geometry(*C1)
    zu, zd, dl = load_events("c1_small.events.bin")
    ref = np.load(os.path.join(GOLD, "c1_small.ref3.npz"))["nocontract"].astype(np.float64)
    # binary64 arithmetic on the reference's (binary32) pixel sets
    r64 = orc.mlem_f64(g, zu, zd, dl, 3, sets_f32=True)
    assert np.linalg.norm(r64 - ref) / np.linalg.norm(r64) < 2e-6
    # binary64 everywhere: boundary pixels of some events differ as well
    r64 = orc.mlem_f64(g, zu, zd, dl, 3, sets_f32=False)
    assert np.linalg.norm(r64 - ref) / np.linalg.norm(r64) < 1e-4


def test_mlem_preserves_event_count():
    """With rho0 = 1, the image total after an iteration equals the number of
    events with a non-zero denominator (reconstruction.h:290-297)."""
    g = orc.geometry(*C1)
    zu, zd, dl = load_events("c1_small.events.bin")
    _, nin, _ = orc.pixel_set_stats(g, zu, zd, dl)
    r = orc.mlem_f64(g, zu, zd, dl, 1)
    assert abs(r.sum() - (nin > 0).sum()) < 1e-6 * r.sum()


def test_pixel_set_stats_match_enumeration():
    g = orc.geometry(*C1)
    zu, zd, dl = load_events("c1_small.events.bin")
    nbb, nin, dig = orc.pixel_set_stats(g, zu[:50], zd[:50], dl[:50])
    mix = orc.lib().orc_mix64
    for i in range(50):
        s = orc.pixel_set(g, float(zu[i]), float(zd[i]), float(dl[i]))
        assert len(s) == nin[i]
        h = 0
        for p in s:
            h = (h + mix(int(p) + 1)) & 0xFFFFFFFFFFFFFFFF
        assert h == int(dig[i])


@pytest.mark.skipif(not orc.ref_available(True), reason="oracle/_ref not built")
def test_oracle_vs_live_reference_fresh_events():
    import stripmlem as sm
    g = orc.geometry(*C1)
    sc = sm.Scanner(*C1)
    zu, zd, dl = sm.generate_events(
        sc, [(0, 0, 200, 150, 10, 1.0), (-100, 40, 40, 30, 0, 4.0)], 3000, seed=77)
    ref, _ = orc.run_ref(g, zu, zd, dl, 2, threads=1, nocontract=True)
    assert bits_equal(orc.mlem_f32(g, zu, zd, dl, 2), ref)
    # --gpu semantics (P = K * s): sum_j s_j rho'_j equals the number of
    # events with a non-zero denominator after one iteration from rho = 1
    r = orc.mlem_f64(g, zu, zd, dl, 1, mode=orc.MODE_GPU)
    s = orc.sensitivity_image_f32(g, five_point=True).astype(np.float64)
    _, nin, _ = orc.pixel_set_stats(g, zu, zd, dl)
    assert abs((s * r).sum() / (nin > 0).sum() - 1) < 1e-6

"""The tile kernel's fixed-point windows.  From an item's second MLEM pass on,
its window accumulates K / D (the image factor applied when the window is
flushed), sized from the item's previous-pass statistic; an event whose
largest addend no longer fits the window's budget is rerun in a weighted
window of its own.  These tests force that rerun (by scaling the statistics
down through strip_debug_scale_item_stats) and check that the images do not
change beyond the run-to-run tolerance and stay within 1e-4 of the FP64
oracle."""
import numpy as np
import pytest

from conftest import C1, C1_PHANTOM
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c1_events():
    import stripmlem as sm
    sc = sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                    C1["s_z"], C1["s_dl"])
    g = orc.geometry(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                     C1["s_z"], C1["s_dl"])
    return sc, g, sm.generate_events(sc, C1_PHANTOM, 80_000, seed=33)


@pytest.mark.parametrize("n_subsets", [1, 4])
def test_forced_reruns_keep_the_images(c1_events, n_subsets):
    import stripmlem as sm
    sc, g, ev = c1_events
    with sm.Reconstruction(sc) as a, sm.Reconstruction(sc) as b:
        a.set_events(*ev, n_subsets=n_subsets)
        b.set_events(*ev, n_subsets=n_subsets)
        a(None, 1)
        b(None, 1)
        assert b.stats()["n_fallback"] == 0  # a first pass is weighted
        a(None, 3)
        # windows 2^10 too fine: most events find no room and are rerun
        b._check(b.lib.strip_debug_scale_item_stats(b._ctx, 1.0 / 1024))
        b(None, 1)
        assert b.stats()["n_fallback"] > len(ev[0]) // 10
        b(None, 2)  # the statistics recover after one pass
        assert b.stats()["n_fallback"] < len(ev[0]) // 1000
        img = b.rho
        assert rel_l2(img, a.rho) < 2e-5
    ref = orc.mlem_f64(g, *ev, 4, n_subsets=n_subsets, sets_f32=True)
    assert rel_l2(img, ref) < 1e-4


def test_scale_item_stats_rejects_bad_factors(c1_events):
    import stripmlem as sm
    sc, g, ev = c1_events
    with sm.Reconstruction(sc) as r:
        r.set_events(*ev)
        for bad in (0.0, -1.0, float("inf"), float("nan")):
            assert r.lib.strip_debug_scale_item_stats(r._ctx, bad) == sm._lib.STRIP_E_INVALID
        assert r.lib.strip_debug_scale_item_stats(r._ctx, 2.0) == sm._lib.STRIP_OK

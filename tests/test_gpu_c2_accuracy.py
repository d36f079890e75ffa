"""Accuracy at the benchmark's own configuration, through the C ABI.

The benchmark reconstructs 2e8 events at the 800 x 400, 1 mm geometry
(R 400 mm, L 800 mm, sigma_z 5 mm, sigma_dl 25 mm, the 10-ellipse phantom)
with 8000-event tile work items, 94 x 112-pixel windows and, from the second
pass on, the unweighted fixed-point windows whose scale comes from each
item's previous pass.  These tests run that same kernel configuration on the
first 1e6 events of the benchmark's event stream (the generator is
counter-based, so they are the benchmark's first events) and hold the
20-iteration image to the FP64 oracle.  Bars: 1e-4 relative L2 against the
FP64 oracle with the reference's binary32 pixel sets, 2e-4 against the full
binary64 oracle (a few boundary pixels change sets in binary64).

Also: 8-subset OSEM at this geometry against the oracle's OSEM."""
import numpy as np
import pytest

from conftest import C2, C2_PHANTOM
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-4
BENCH_SEED = 20260101
N_EVENTS = 1_000_000


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c2():
    import stripmlem as sm
    sc = sm.Scanner(C2["radius"], C2["length"], C2["n_y"], C2["n_z"], C2["p"], C2["p"],
                    C2["s_z"], C2["s_dl"])
    g = orc.geometry(C2["radius"], C2["length"], C2["n_y"], C2["n_z"], C2["p"], C2["p"],
                     C2["s_z"], C2["s_dl"])
    ev = sm.generate_events(sc, C2_PHANTOM, N_EVENTS, seed=BENCH_SEED)
    return sc, g, ev


def test_c2_mlem_20_iterations_vs_fp64(c2):
    import stripmlem as sm
    sc, g, (zu, zd, dl) = c2
    with sm.Reconstruction(sc, mode=sm.MODE_CPU, accumulation=sm.ACCUM_KAHAN) as rec:
        rec.set_item_events(8000)
        rec.set_events(zu, zd, dl)
        st = rec.stats()
        # the benchmark's windows and item size
        assert st["max_item_events"] == 8000
        assert (st["tile_z"], st["tile_y"]) == (32, 32)
        assert st["n_overflow"] == 0
        fallbacks = 0
        for _ in range(20):
            rec(None, 1)
            fallbacks += rec.stats()["n_fallback"]
        img = rec.rho
    assert np.all(np.isfinite(img)) and img.min() >= 0
    ref = orc.mlem_f64(g, zu, zd, dl, 20, sets_f32=True)
    assert rel_l2(img, ref) < REL_L2_TOL
    ref64 = orc.mlem_f64(g, zu, zd, dl, 20, sets_f32=False)
    assert rel_l2(img, ref64) < 2 * REL_L2_TOL
    # the unweighted windows carried the passes: the weighted rerun of events
    # they had no room for stays rare
    assert fallbacks < 1e-5 * N_EVENTS * 20


def test_c2_osem_8_subsets_vs_fp64(c2):
    import stripmlem as sm
    sc, g, (zu, zd, dl) = c2
    n = 500_000
    with sm.Reconstruction(sc, mode=sm.MODE_CPU) as rec:
        rec.set_events(zu[:n], zd[:n], dl[:n], n_subsets=8)
        assert rec.stats()["n_subsets"] == 8
        rec(None, 2, n_subsets=8)
        img = rec.rho
    ref = orc.mlem_f64(g, zu[:n], zd[:n], dl[:n], 2, n_subsets=8, sets_f32=True)
    assert rel_l2(img, ref) < REL_L2_TOL

"""Batches of reconstructions (per step: own tile launches of the members with
at least two work items per SM, one persistent tile launch over the others'
items, CUDA graph replay) and the schedule autotuner, against single-context
runs and the FP64 oracle."""
import numpy as np
import pytest

from conftest import C1, C1_PHANTOM
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

# (radius, length, n_y, n_z, pixel, sigma_z, sigma_dl, events, phantom)
MEMBERS = [
    (200.0, 500.0, 200, 250, 2.0, 10.0, 42.0, 60_000, C1_PHANTOM),
    (100.0, 160.0, 100, 160, 1.0, 6.0, 25.0, 40_000,
     [(10, 5, 20, 12, 30, 2.0), (0, 0, 60, 40, 0, 1.0)]),
    (150.0, 300.0, 100, 100, 3.0, 12.0, 50.0, 25_000,
     [(-40, 20, 30, 25, 0, 0.5), (0, 0, 110, 80, 10, 1.0)]),
    (80.0, 240.0, 40, 60, 4.0, 8.0, 30.0, 15_000, [(0, 0, 90, 50, 0, 1.0)]),
]


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def members():
    import stripmlem as sm
    out = []
    for i, (R, L, ny, nz, p, sz, sdl, n, ph) in enumerate(MEMBERS):
        sc = sm.Scanner(R, L, ny, nz, p, p, sz, sdl)
        g = orc.geometry(R, L, ny, nz, p, p, sz, sdl)
        out.append((sc, g, sm.generate_events(sc, ph, n, seed=100 + i)))
    return out


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_equals_single_contexts(members, mode):
    import stripmlem as sm
    singles, recs = [], []
    try:
        for sc, g, ev in members:
            with sm.Reconstruction(sc, mode=mode) as r:
                r.set_events(*ev)
                r(None, 3)
                singles.append(r.rho)
            rec = sm.Reconstruction(sc, mode=mode)
            rec.set_events(*ev)
            recs.append(rec)
        with sm.Batch(recs, mode=mode) as batch:
            batch(3)
            st = batch.stats()
        assert st["n_events"] == sum(len(ev[0]) for _, _, ev in members)
        assert st["launches_per_iteration"] >= 2
        assert st["last_iterate_ms"] > 0
        for rec, single, (sc, g, ev) in zip(recs, singles, members):
            img = rec.rho
            assert rel(img, single) < 2e-5
            ref = orc.mlem_f64(g, *ev, 3, mode=mode, sets_f32=True)
            assert rel(img, ref) < 1e-4
    finally:
        for r in recs:
            r.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_own_launches_equal_single_contexts(members, mode):
    """Members 0 and 1 binned in 64-event work items (940 and 625 items, past
    two per SM) take tile launches of their own on the side
    streams; members 2 and 3 stay in the persistent launch (all re-binned
    without the cut last wave)."""
    import stripmlem as sm
    item_events = [64, 64, 0, 0]
    singles, recs = [], []
    try:
        for (sc, g, ev), k in zip(members, item_events):
            with sm.Reconstruction(sc, mode=mode) as r:
                r.set_item_events(k)
                r.set_events(*ev)
                r(None, 3)
                singles.append(r.rho)
            rec = sm.Reconstruction(sc, mode=mode)
            rec.set_item_events(k)
            rec.set_events(*ev)
            recs.append(rec)
        with sm.Batch(recs, mode=mode) as batch:
            batch(3)
            st = batch.stats()
            items = [r.stats()["n_work_items"] for r in recs]
        assert min(items[:2]) >= 2 * 148 and max(items[2:]) < 2 * 148
        assert st["n_work_items"] == sum(items)
        assert st["launches_per_iteration"] >= 4  # 2 own + persistent + update
        for rec, single, (sc, g, ev) in zip(recs, singles, members):
            img = rec.rho
            assert rel(img, single) < 2e-5
            ref = orc.mlem_f64(g, *ev, 3, mode=mode, sets_f32=True)
            assert rel(img, ref) < 1e-4
    finally:
        for r in recs:
            r.close()


def test_batch_rejects_bad_members(members):
    import stripmlem as sm
    sc, g, ev = members[0]
    with sm.Reconstruction(sc) as r:
        r.set_events(*ev)
        with pytest.raises(sm.StripError):
            sm.Batch([r, r])
    with sm.Reconstruction(sc) as r:  # no events yet
        with pytest.raises(sm.StripError):
            sm.Batch([r])


def test_autotune_keeps_results(members):
    import stripmlem as sm
    sc, g, ev = members[0]
    with sm.Reconstruction(sc) as r:
        r.set_events(*ev)
        rho0 = r.rho
        best = r.autotune()
        assert best["tile"] in (16, 32, 48, 64) and best["grab"] in (4, 8, 16, 32)
        assert best["ms"] > 0
        assert np.array_equal(r.rho, rho0)  # the image is untouched
        r(None, 5)
        img = r.rho
    ref = orc.mlem_f64(g, *ev, 5, sets_f32=True)
    assert rel(img, ref) < 1e-4


@pytest.mark.parametrize("tile,grab", [(16, 4), (48, 16), (64, 1)])
def test_hand_schedules(members, tile, grab):
    import stripmlem as sm
    sc, g, ev = members[1]
    with sm.Reconstruction(sc) as r:
        r.set_schedule(tile, grab)
        r.set_events(*ev)
        assert r.stats()["tile_z"] in (tile, 16)
        r(None, 4)
        img = r.rho
    ref = orc.mlem_f64(g, *ev, 4, sets_f32=True)
    assert rel(img, ref) < 1e-4

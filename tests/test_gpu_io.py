"""Event input paths through the C ABI: the binary event-file reader
(strip_load_responses_file: pinned staging buffers filled by several host
threads, the triples split on the device), the AoS setter
(strip_set_responses) and the SoA setter from pageable and from pinned host
memory all hand the binning the same events: the exact pixel-work totals of
the binned events (strip_count_work) are equal, and the reconstructions
agree to the run-to-run rounding of the atomic accumulations."""
import numpy as np
import pytest

from conftest import C1, C1_PHANTOM

pytestmark = pytest.mark.gpu


def _scanner():
    import stripmlem as sm
    return sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                      C1["s_z"], C1["s_dl"])


@pytest.fixture(scope="module")
def events():
    import stripmlem as sm
    return sm.generate_events(_scanner(), C1_PHANTOM, 3_000_000, seed=11)


def _reconstruct(load, iters=2):
    """(image after `iters` iterations, stats, exact work totals)."""
    import ctypes
    import stripmlem as sm
    with sm.Reconstruction(_scanner()) as rec:
        load(rec)
        st = rec.stats()
        w = [ctypes.c_int64() for _ in range(3)]
        rec._check(rec.lib.strip_count_work(rec._ctx, *(ctypes.byref(x) for x in w)))
        st["work"] = tuple(x.value for x in w)
        rec(None, iters)
        return rec.rho, st


def _same(got, want):
    (a, sa), (b, sb) = got, want
    assert sa["work"] == sb["work"] and sa["n_events"] == sb["n_events"]
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-6


def test_file_reader_equals_set_events(tmp_path, events):
    zu, zd, dl = events
    path = tmp_path / "events.bin"
    t = np.stack([zu, zd, dl], 1).astype("<f4")
    # 3e6 events = 36 MB: more than one 32 MB staging chunk; a trailing
    # partial triple (8 bytes) that the reader must ignore
    with open(path, "wb") as f:
        f.write(t.tobytes())
        f.write(b"\x00" * 8)
    want = _reconstruct(lambda r: r.set_events(zu, zd, dl))
    got = _reconstruct(lambda r: r.load_responses_file(path))
    assert got[1]["n_events"] == zu.shape[0]
    _same(got, want)
    # a window of the file: events [first, first + n)
    first, n = 123_457, 1_000_000
    want = _reconstruct(lambda r: r.set_events(zu[first:first + n], zd[first:first + n],
                                               dl[first:first + n]))

    def load(r):
        assert r.load_responses_file(path, first=first, n=n) == n
    _same(_reconstruct(load), want)
    # past the end: no events, and a missing file is an error
    import stripmlem as sm
    with sm.Reconstruction(_scanner()) as rec:
        assert rec.load_responses_file(path, first=10_000_000) == 0
        with pytest.raises(sm.StripError):
            rec.load_responses_file(tmp_path / "missing.bin")


def test_aos_and_pinned_setters_equal_set_events(events):
    import torch
    zu, zd, dl = events
    want = _reconstruct(lambda r: r.set_events(zu, zd, dl))
    t = np.ascontiguousarray(np.stack([zu, zd, dl], 1))

    def set_responses(r):
        r.responses = t
    _same(_reconstruct(set_responses), want)
    pinned = [torch.from_numpy(a).pin_memory() for a in (zu, zd, dl)]
    _same(_reconstruct(lambda r: r.set_events(*(p.numpy() for p in pinned))), want)


def test_rebinning_one_context_equals_fresh_contexts(events):
    """One context given event sets that shrink and grow again (its memory
    pool hands each binning the buffers the last one freed) reconstructs as
    a fresh context does for each set."""
    import stripmlem as sm
    zu, zd, dl = events
    with sm.Reconstruction(_scanner()) as rec:
        for n in (3_000_000, 400_000, 3_000_000, 1_300_000):
            rec.set_events(zu[:n], zd[:n], dl[:n])
            assert rec.stats()["n_events"] == n
            rec.rho = np.ones((C1["n_y"], C1["n_z"]), np.float32)
            rec(None, 2)
            got = rec.rho.astype(np.float64)
            want, _ = _reconstruct(lambda r: r.set_events(zu[:n], zd[:n], dl[:n]))
            want = want.astype(np.float64)
            assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-6, n

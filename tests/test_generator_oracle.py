"""The library's host event generator (strip_generate_events) equals the
oracle's separate statement of the same counter-based definition
(oracle/strip_events.c) bit for bit.  The benchmark's CPU arm generates its
events from the oracle alone, so this is what makes its input the GPU arm's
input.  CPU only: the host generator needs no device."""
import numpy as np
import pytest

from conftest import C1, C1_PHANTOM, C2, C2_PHANTOM


def _scanner(c):
    import stripmlem as sm
    return sm.Scanner(c["radius"], c["length"], c["n_y"], c["n_z"], c["p"], c["p"],
                      c["s_z"], c["s_dl"])


@pytest.mark.parametrize("cfg,phantom,seed,n", [
    (C2, C2_PHANTOM, 20260101, 300_000),
    (C1, C1_PHANTOM, 1, 200_000),
    (C1, C1_PHANTOM, (7 << 32) | 99, 50_000),
])
def test_oracle_generator_is_the_library_generator(cfg, phantom, seed, n):
    import stripmlem as sm
    from oracle import oracle as orc
    g = orc.geometry(cfg["radius"], cfg["length"], cfg["n_y"], cfg["n_z"], cfg["p"],
                     cfg["p"], cfg["s_z"], cfg["s_dl"])
    got = orc.generate_events(g, phantom, n, seed)
    want = sm.generate_events(_scanner(cfg), phantom, n, seed=seed)
    for a, b in zip(got, want):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle_generator_prefix_property():
    """Event i depends on (seed, i) only: a prefix of a longer run is the
    shorter run (the benchmark's bounded CPU samples rely on it)."""
    from oracle import oracle as orc
    g = orc.geometry(C2["radius"], C2["length"], C2["n_y"], C2["n_z"], C2["p"], C2["p"],
                     C2["s_z"], C2["s_dl"])
    long = orc.generate_events(g, C2_PHANTOM, 40_000, 5)
    short = orc.generate_events(g, C2_PHANTOM, 12_345, 5)
    for a, b in zip(long, short):
        assert np.array_equal(a[:12_345], b)

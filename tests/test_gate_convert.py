"""GATE text converters (3d_tool_convert, src/3d/tool/convert_cmd.cpp) of
stripmlem.hybrid against the reference binary's own output, committed in
tests/golden/gate_small.npz (made by tests/golden/make_gate_golden.py).
Detector pairs exactly; values, the smeared ones included, to the 6
significant digits the reference prints.  CPU only."""
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "gate_small.npz")


def as_table(r):
    return np.stack([np.asarray(a, np.float64) for a in r], 1)


@pytest.mark.parametrize("key,only", [("warsaw_all", 0), ("warsaw_only1", 1)])
def test_warsaw_matches_reference(key, only):
    from stripmlem import hybrid as hy
    z = np.load(GOLDEN)
    got = as_table(hy.convert_warsaw(list(z["warsaw_in"]), hy.Barrel().polygons, 0.5, only=only))
    ref = z[key]
    assert got.shape == ref.shape
    assert np.array_equal(got[:, :2], ref[:, :2])
    assert np.allclose(got[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-9)
    assert np.all(got[:, 0] >= got[:, 1])


@pytest.mark.parametrize("key,rel", [("tbednarski", False), ("tbednarski_rel", True)])
def test_tbednarski_matches_reference(key, rel):
    from stripmlem import hybrid as hy
    z = np.load(GOLDEN)
    got = as_table(hy.convert_tbednarski(list(z["tbednarski_in"]), relative_time=rel))
    ref = z[key]
    assert got.shape == ref.shape
    assert np.array_equal(got[:, :2], ref[:, :2])
    assert np.allclose(got[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-6)


def test_warsaw_smearing_matches_reference():
    """With --s-z 0.01 --s-dl 0.05 --seed 5 the smeared values are the
    reference's (std::normal_distribution over std::mt19937_64, drawn in
    output order), to the 6 digits it prints."""
    from stripmlem import hybrid as hy
    z = np.load(GOLDEN)
    got = as_table(hy.convert_warsaw(list(z["warsaw_in"]), hy.Barrel().polygons, 0.5,
                                     sigma_z=0.01, sigma_dl=0.05, seed=5))
    ref = z["warsaw_smeared"]
    assert got.shape == ref.shape
    assert np.array_equal(got[:, :2], ref[:, :2])
    assert np.allclose(got[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-9)
    # a different seed gives other errors
    other = as_table(hy.convert_warsaw(list(z["warsaw_in"]), hy.Barrel().polygons, 0.5,
                                       sigma_z=0.01, sigma_dl=0.05, seed=6))
    assert not np.allclose(other[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-9)


def test_warsaw_smearing_and_empty_input():
    from stripmlem import hybrid as hy
    z = np.load(GOLDEN)
    b = hy.Barrel()
    exact = hy.convert_warsaw(list(z["warsaw_in"]), b.polygons, 0.5)
    noisy = hy.convert_warsaw(list(z["warsaw_in"]), b.polygons, 0.5, sigma_z=0.01,
                              sigma_dl=0.05, seed=3)
    assert np.array_equal(exact[0], noisy[0])
    dz = noisy[2] - exact[2]
    assert 0.005 < dz.std() < 0.015
    assert len(hy.convert_warsaw([], b.polygons, 0.5)[0]) == 0
    assert len(hy.convert_tbednarski([])[0]) == 0

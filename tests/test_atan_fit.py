"""The 3D hybrid kernel's arctangent (atan2_pos, csrc/hybrid_kernels.cu):
its polynomial coefficients are the output of tests/golden/fit_atan.py (CPU),
and on the GPU its error against binary64 atan2 over its whole domain stays
within a few binary32 ulps of pi, comparable to CUDA's atan2f (GPU)."""
import ctypes
import importlib.util
import os

import numpy as np
import pytest

from conftest import ROOT

FIT = os.path.join(ROOT, "tests", "golden", "fit_atan.py")


def _fit_module():
    spec = importlib.util.spec_from_file_location("fit_atan", FIT)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_kernel_coefficients_come_from_the_fit_script():
    m = _fit_module()
    err, coef = m.fit()
    assert err < 4e-8
    assert [float(c) for c in m.kernel_coefficients()] == [float(c) for c in coef]


def _grid():
    """atan2_pos(a, b) arguments: a > 0 from 1e-6 to 1e6, b of both signs and
    zero, over ratios that cover every branch (|b| < a, |b| > a, b < 0)."""
    a = np.geomspace(1e-6, 1e6, 1201, dtype=np.float64)
    r = np.concatenate([-np.geomspace(1e4, 1e-4, 601), [0.0], np.geomspace(1e-4, 1e4, 601)])
    A, Rr = np.meshgrid(a, r, indexing="ij")
    B = A * Rr
    return A.ravel().astype(np.float32), B.ravel().astype(np.float32)


@pytest.mark.gpu
def test_atan2_pos_error_bound_on_the_device():
    from stripmlem import _lib
    lib = _lib.load()
    a, b = _grid()
    n = a.size
    ours = np.empty(n, np.float32)
    cuda = np.empty(n, np.float32)
    for which, out in ((0, ours), (1, cuda)):
        rc = lib.hybrid_debug_atan2(0, a.ctypes.data, b.ctypes.data, n, which, out.ctypes.data)
        assert rc == 0
    exact = np.arctan2(a.astype(np.float64), b.astype(np.float64))
    e_ours = np.abs(ours.astype(np.float64) - exact)
    e_cuda = np.abs(cuda.astype(np.float64) - exact)
    # results lie in (0, pi]: 2.4e-7 is one binary32 ulp at pi
    assert e_ours.max() < 3 * 2.4e-7, e_ours.max()
    assert e_ours.max() < e_cuda.max() + 2 * 2.4e-7
    # relative to the result where it is small (a << |b|, b > 0)
    small = exact < 1e-3
    rel = e_ours[small] / exact[small]
    assert rel.max() < 1e-6, rel.max()

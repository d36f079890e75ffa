"""strip_iterate_noalloc: the allocation-free MLEM iteration, for callers that
cannot call cudaMalloc (code inside a framework that owns all device memory
through its own pool, or pipelines that must not hit cudaMalloc/cudaFree,
which can synchronise the device).  It keeps its scratch in a fixed
file-scope device array instead.

Checked through the C ABI against the regular entry point (strip_iterate on
a context) on two calls in a row, at the tolerance of the other parity tests.
This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from conftest import C1, C1_PHANTOM

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-4


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_matches_context_iterations(mode):
    import torch
    import stripmlem as sm
    from stripmlem import _lib

    lib = _lib.load()
    sc = sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                    C1["s_z"], C1["s_dl"])
    zu, zd, dl = sm.generate_events(sc, C1_PHANTOM, 60_000, seed=21)
    # the regular entry point: two iterations on a context
    expected = []
    with sm.Reconstruction(sc, mode=mode) as rec:
        rec.set_events(zu, zd, dl)
        for _ in range(2):
            rec(None, 1)
            expected.append(rec.rho)

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    d_zu = torch.from_numpy(zu).to(dev)
    d_zd = torch.from_numpy(zd).to(dev)
    d_dl = torch.from_numpy(dl).to(dev)
    rho_a = torch.ones((C1["n_y"], C1["n_z"]), dtype=torch.float32, device=dev)
    rho_b = torch.empty_like(rho_a)
    g = sc.geometry()
    stream = torch.cuda.current_stream().cuda_stream
    got = []
    src, dst = rho_a, rho_b
    for _ in range(2):  # two calls in a row share the scratch
        rc = lib.strip_iterate_noalloc(ctypes.byref(g), d_zu.data_ptr(), d_zd.data_ptr(),
                                       d_dl.data_ptr(), zu.shape[0], src.data_ptr(),
                                       dst.data_ptr(), mode, ctypes.c_void_p(stream))
        assert rc == _lib.STRIP_OK
        torch.cuda.synchronize()
        got.append(dst.cpu().numpy().copy())
        src, dst = dst, src
    for e, o in zip(expected, got):
        assert np.all(np.isfinite(o))
        assert rel_l2(o, e) < REL_L2_TOL


def test_noalloc_rejects_oversized_images():
    import torch
    from stripmlem import _lib

    lib = _lib.load()
    torch.cuda.init()
    n_side = 1100  # 1100^2 > STRIP_NOALLOC_MAX_PIXELS = 2^20
    g = _lib.Geometry(550.0, 1100.0, n_side, n_side, 1.0, 1.0, 5.0, 25.0, 0.0, 0.0)
    buf = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    p = buf.data_ptr()
    rc = lib.strip_iterate_noalloc(ctypes.byref(g), p, p, p, 1, p, p, 0, None)
    assert rc == _lib.STRIP_E_INVALID
    rc = lib.strip_iterate_noalloc(None, p, p, p, 1, p, p, 0, None)
    assert rc == _lib.STRIP_E_INVALID

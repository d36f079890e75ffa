"""The C-ABI library loads on a machine without a GPU and exports every
function include/stripmlem.h declares; calls that need a device fail with a
status code instead of crashing.  CPU only."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "stripmlem.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(strip_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("strip_ctx_create", "strip_set_events", "strip_iterate",
                     "strip_get_image", "strip_forward", "strip_adjoint",
                     "strip_grad_sigma", "strip_debug_pixel_sets"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    from stripmlem import _lib
    names = declared_functions()
    assert names
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_abi_version_macro():
    assert "#define STRIPMLEM_ABI_VERSION 1" in open(HEADER).read()


def test_create_without_device_reports_status(lib):
    if gpu_available():
        return
    from stripmlem import _lib
    g = _lib.Geometry(200, 500, 200, 250, 2, 2, 10, 42, 0, 0)
    ctx = ctypes.c_void_p()
    rc = lib.strip_ctx_create(ctypes.byref(g), 0, ctypes.byref(ctx))
    assert rc == _lib.STRIP_E_NODEVICE
    assert not ctx.value


def test_invalid_geometry_rejected(lib):
    from stripmlem import _lib
    ctx = ctypes.c_void_p()
    for bad in (_lib.Geometry(200, 500, 0, 250, 2, 2, 10, 42, 0, 0),
                _lib.Geometry(200, 500, 200, 40000, 2, 2, 10, 42, 0, 0),
                _lib.Geometry(200, 500, 200, 250, 2, 2, 0, 42, 0, 0),
                _lib.Geometry(200, 500, 200, 250, -2, 2, 10, 42, 0, 0)):
        assert lib.strip_ctx_create(ctypes.byref(bad), 0, ctypes.byref(ctx)) == _lib.STRIP_E_INVALID
    assert lib.strip_ctx_create(None, 0, ctypes.byref(ctx)) == _lib.STRIP_E_INVALID


def test_null_context_calls_rejected(lib):
    from stripmlem import _lib
    assert lib.strip_ctx_destroy(None) == _lib.STRIP_E_INVALID
    assert lib.strip_iterate(None, 1, 0, 1, 0, _lib.PROGRESS_CB(), None) == _lib.STRIP_E_INVALID
    assert lib.strip_set_events(None, None, None, None, 0, 1) == _lib.STRIP_E_INVALID
    assert lib.strip_load_responses_file(None, b"x.bin", 0, -1, 1, None) == _lib.STRIP_E_INVALID
    assert lib.strip_set_item_events(None, 8000) == _lib.STRIP_E_INVALID


def test_host_only_entry_points_validate_arguments(lib):
    """The text parser and the converter's smearing run on the host: bad
    arguments are rejected with a status, no device needed."""
    import ctypes
    from stripmlem import _lib
    n = ctypes.c_int64()
    assert lib.hybrid_parse_responses_text(None, 0, 0, None, None, None, None, None,
                                           ctypes.byref(n)) == _lib.STRIP_E_INVALID
    text = b"1 0 1 2 3\n2 1 4 5 6\n"
    assert lib.hybrid_parse_responses_text(text, len(text), 0, None, None, None, None, None,
                                           ctypes.byref(n)) == _lib.STRIP_OK
    assert n.value == 2  # capacity 0: counting only
    z = np.zeros(3)
    assert lib.hybrid_smear_responses(1, -1.0, 1.0, 3, z.ctypes.data, z.ctypes.data,
                                      z.ctypes.data) == _lib.STRIP_E_INVALID
    a, b, c = np.zeros(3), np.zeros(3), np.zeros(3)
    assert lib.hybrid_smear_responses(1, 0.0, 0.0, 3, a.ctypes.data, b.ctypes.data,
                                      c.ctypes.data) == _lib.STRIP_OK
    assert not (a.any() or b.any() or c.any())  # zero sigmas leave the values


def test_generator_runs_on_host_and_is_deterministic():
    import stripmlem as sm
    sc = sm.Scanner(200, 500, 200, 250, 2, 2, 10, 42)
    ph = [(40, 30, 30, 20, 0, 3.0), (0, 0, 150, 100, 0, 1.0)]
    a = sm.generate_events(sc, ph, 5000, seed=3)
    b = sm.generate_events(sc, ph, 5000, seed=3)
    c = sm.generate_events(sc, ph, 5000, seed=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    # prefix property: event i depends only on (seed, i)
    d = sm.generate_events(sc, ph, 1000, seed=3)
    assert np.array_equal(a[0][:1000], d[0])
    # every event was detected: |z_u|, |z_d| stay within L/2 up to smearing
    zu, zd, dl = a
    assert np.all(np.abs(zu) < 250 + 8 * 10) and np.all(np.abs(zd) < 250 + 8 * 10)


def test_generator_rejects_bad_phantom():
    import stripmlem as sm
    sc = sm.Scanner(200, 500, 200, 250, 2, 2, 10, 42)
    try:
        sm.generate_events(sc, [(0, 0, -1, 10, 0, 1.0)], 10)
    except sm.StripError as e:
        assert e.code == -1
    else:
        raise AssertionError("expected StripError")

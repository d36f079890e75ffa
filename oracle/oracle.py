"""TEST INFRASTRUCTURE ONLY: ctypes binding of the C oracle (liboracle.so,
strip_oracle.c) and runners for the reference binaries under oracle/_ref.

Only tests/, bench.py's reference / cpu_baseline arm and
__graft_entry__.smoke() may import this module, and only as the checker.
"""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_RECON = os.path.join(REF_DIR, "2d_strip_reconstruction")
REF_RECON_NOCONTRACT = os.path.join(REF_DIR, "2d_strip_reconstruction_nocontract")

MODE_CPU = 0
MODE_GPU = 1


class Geometry(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_double),
        ("scintillator_length", ctypes.c_double),
        ("n_y_pixels", ctypes.c_int32),
        ("n_z_pixels", ctypes.c_int32),
        ("pixel_height", ctypes.c_double),
        ("pixel_width", ctypes.c_double),
        ("sigma_z", ctypes.c_double),
        ("sigma_dl", ctypes.c_double),
        ("center_y", ctypes.c_double),
        ("center_z", ctypes.c_double),
    ]


def build():
    """Compiles liboracle.so (plain gcc; works on any box of this image)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        f, d, i32, u64, g = (P(ctypes.c_float), P(ctypes.c_double), P(ctypes.c_int32),
                             P(ctypes.c_uint64), P(Geometry))
        c_f, c_d, c_i, c_l = ctypes.c_float, ctypes.c_double, ctypes.c_int, ctypes.c_int64
        sig = {
            "orc_event_box_f32": (None, [g, c_f, c_f, c_f, i32]),
            "orc_event_box_f64": (None, [g, c_d, c_d, c_d, i32]),
            "orc_pixel_set_f32": (c_l, [g, c_f, c_f, c_f, i32, c_l]),
            "orc_pixel_set_stats_f32": (None, [g, f, f, f, c_l, i32, i32, u64]),
            "orc_mix64": (ctypes.c_uint64, [ctypes.c_uint64]),
            "orc_mlem_f32": (None, [g, f, f, f, c_l, f, c_i, c_i]),
            "orc_mlem_f64": (None, [g, f, f, f, c_l, d, c_i, c_i, c_i, c_i, c_i]),
            "orc_forward_f64": (None, [g, f, f, f, c_l, d, c_d, c_d, c_i, d]),
            "orc_adjoint_f64": (None, [g, f, f, f, c_l, d, c_d, c_d, c_i, d]),
            "orc_grad_sigma_f64": (None, [g, f, f, f, c_l, d, d, c_d, c_d, d, d]),
            "orc_gaussian_kernel_f32": (c_f, [c_f] * 8),
            "orc_gaussian_kernel_f64": (c_d, [c_d] * 8),
            "orc_analytic_kernel_f32": (c_f, [c_f] * 8),
            "orc_analytic_kernel_f64": (c_d, [c_d] * 8),
            "orc_bb_y_f64": (c_d, [c_d] * 3),
            "orc_bb_z_f64": (c_d, [c_d] * 3),
            "orc_sensitivity_f64": (c_d, [g, c_d, c_d]),
            "orc_sensitivity_f32": (c_f, [g, c_f, c_f]),
            "orc_pixel_sensitivity_f32": (c_f, [g, ctypes.c_int32, ctypes.c_int32]),
            "orc_sensitivity_image_f32": (None, [g, c_i, f]),
            "orc_pixel_at_f64": (None, [g, c_d, c_d, i32]),
            "orc_pixel_center_f64": (None, [g, ctypes.c_int32, ctypes.c_int32, d]),
            "orc_to_projection_tan_f64": (None, [c_d, c_d, c_d, c_d, d]),
            "orc_from_projection_tan_f64": (None, [c_d, c_d, c_d, c_d, d]),
            "orc_generate_events": (c_i, [g, d, c_i, ctypes.c_uint64, c_l, f, f, f]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def geometry(radius, length, n_y, n_z, p_h, p_w, s_z, s_dl, c_y=0.0, c_z=0.0):
    return Geometry(radius, length, n_y, n_z, p_h, p_w, s_z, s_dl, c_y, c_z)


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _soa(z_u, z_d, dl):
    return (np.ascontiguousarray(z_u, np.float32), np.ascontiguousarray(z_d, np.float32),
            np.ascontiguousarray(dl, np.float32))


def generate_events(g, ellipses, n, seed):
    """n seeded events (z_u, z_d, dl binary32 arrays) of the benchmark's
    counter-based generator; ellipses = rows (z, y, a, b, angle_deg,
    activity).  The same events as the product library's generator, computed
    without it (strip_events.c)."""
    el = np.ascontiguousarray(np.asarray(ellipses, np.float64).reshape(-1, 6))
    out = [np.empty(n, np.float32) for _ in range(3)]
    rc = lib().orc_generate_events(ctypes.byref(g), _dp(el), el.shape[0], int(seed), n,
                                   *(_fp(a) for a in out))
    if rc != 0:
        raise ValueError("orc_generate_events failed")
    return tuple(out)


def event_box(g, z_u, z_d, dl, f64=False):
    out = np.zeros(6, np.int32)
    (lib().orc_event_box_f64 if f64 else lib().orc_event_box_f32)(
        ctypes.byref(g), z_u, z_d, dl, _ip(out))
    return out


def pixel_set(g, z_u, z_d, dl):
    n = lib().orc_pixel_set_f32(ctypes.byref(g), z_u, z_d, dl, None, 0)
    out = np.zeros(max(n, 1), np.int32)
    lib().orc_pixel_set_f32(ctypes.byref(g), z_u, z_d, dl, _ip(out), n)
    return out[:n]


def pixel_set_stats(g, z_u, z_d, dl):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    n = z_u.shape[0]
    nbb = np.zeros(n, np.int32)
    nin = np.zeros(n, np.int32)
    dig = np.zeros(n, np.uint64)
    lib().orc_pixel_set_stats_f32(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), n,
                                  _ip(nbb), _ip(nin),
                                  dig.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return nbb, nin, dig


def mlem_f32(g, z_u, z_d, dl, n_iter, rho=None, mode=MODE_CPU):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    if rho is None:
        rho = np.ones((g.n_y_pixels, g.n_z_pixels), np.float32)
    rho = np.ascontiguousarray(rho, np.float32).copy()
    lib().orc_mlem_f32(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), z_u.shape[0],
                       _fp(rho), n_iter, mode)
    return rho


def mlem_f64(g, z_u, z_d, dl, n_iter, rho=None, mode=MODE_CPU, n_subsets=1,
             sets_f32=True, n_threads=0):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    if rho is None:
        rho = np.ones((g.n_y_pixels, g.n_z_pixels), np.float64)
    rho = np.ascontiguousarray(rho, np.float64).copy()
    lib().orc_mlem_f64(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), z_u.shape[0],
                       _dp(rho), n_iter, mode, n_subsets, int(bool(sets_f32)), n_threads)
    return rho


def forward_f64(g, z_u, z_d, dl, rho, sigma_z, sigma_dl, mode=MODE_CPU):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    r = np.ascontiguousarray(rho, np.float64)
    y = np.zeros(z_u.shape[0], np.float64)
    lib().orc_forward_f64(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), z_u.shape[0],
                          _dp(r), sigma_z, sigma_dl, mode, _dp(y))
    return y


def adjoint_f64(g, z_u, z_d, dl, w, sigma_z, sigma_dl, mode=MODE_CPU):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    wv = np.ascontiguousarray(w, np.float64)
    out = np.zeros((g.n_y_pixels, g.n_z_pixels), np.float64)
    lib().orc_adjoint_f64(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), z_u.shape[0],
                          _dp(wv), sigma_z, sigma_dl, mode, _dp(out))
    return out


def grad_sigma_f64(g, z_u, z_d, dl, rho, w, sigma_z, sigma_dl):
    z_u, z_d, dl = _soa(z_u, z_d, dl)
    r = np.ascontiguousarray(rho, np.float64)
    wv = np.ascontiguousarray(w, np.float64)
    gz = ctypes.c_double()
    gd = ctypes.c_double()
    lib().orc_grad_sigma_f64(ctypes.byref(g), _fp(z_u), _fp(z_d), _fp(dl), z_u.shape[0],
                             _dp(r), _dp(wv), sigma_z, sigma_dl, ctypes.byref(gz),
                             ctypes.byref(gd))
    return gz.value, gd.value


def sensitivity_image_f32(g, five_point=True):
    out = np.zeros((g.n_y_pixels, g.n_z_pixels), np.float32)
    lib().orc_sensitivity_image_f32(ctypes.byref(g), int(five_point), _fp(out))
    return out


# --------------------------------------------------------------------------
# The reference's own binary (compiled from its sources by oracle/Makefile)
# --------------------------------------------------------------------------

def ref_available(nocontract=True):
    return os.access(REF_RECON_NOCONTRACT if nocontract else REF_RECON, os.X_OK)


def write_events_bin(path, z_u, z_d, dl):
    """Reference binary event format: raw little-endian f32 triples
    z_u z_d dl, no header (bstream.h:23-26, reconstruction.h:156-167)."""
    t = np.stack([np.asarray(z_u, np.float32), np.asarray(z_d, np.float32),
                  np.asarray(dl, np.float32)], axis=1)
    t.astype("<f4").tofile(path)


def run_ref(g, z_u, z_d, dl, n_iter, threads=1, nocontract=True, extra=(),
            workdir=None, timeout=3600):
    """Runs the reference 2d_strip_reconstruction on the events; returns
    (image float32 [n_y, n_z], stdout).  Geometry goes through the CLI as
    -r R -l L -p P --n-y-pixels --n-z-pixels --s-z --s-dl (square pixels)."""
    exe = REF_RECON_NOCONTRACT if nocontract else REF_RECON
    if g.pixel_width != g.pixel_height or g.center_y != 0 or g.center_z != 0:
        raise ValueError("the reference CLI has square pixels and a centred scanner")
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        ev = os.path.join(td, "events.bin")
        write_events_bin(ev, z_u, z_d, dl)
        out = os.path.join(td, "r.bin")
        cmd = [exe, ev, "-r", repr(g.radius), "-l", repr(g.scintillator_length),
               "-p", repr(g.pixel_width), "--n-y-pixels", str(g.n_y_pixels),
               "--n-z-pixels", str(g.n_z_pixels), "--s-z", repr(g.sigma_z),
               "--s-dl", repr(g.sigma_dl), "-i", "1", "-I", str(n_iter),
               "-T", str(threads), "-o", out, *extra]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference failed ({p.returncode}): {p.stderr}")
        # output naming: add_index(iteration, n_iterations) -> r_<it>.bin
        files = sorted(f for f in os.listdir(td) if re.match(r"r_\d+\.bin$", f))
        img = np.fromfile(os.path.join(td, files[-1]), dtype="<f4")
        return img.reshape(g.n_y_pixels, g.n_z_pixels), p.stdout + p.stderr


def ref_benchmark(g, events_path, n_iter, threads, timeout=3600):
    """Times the reference CPU path (-vv): returns ms per iteration ('# av')."""
    cmd = [REF_RECON, events_path, "-r", repr(g.radius), "-l", repr(g.scintillator_length),
           "-p", repr(g.pixel_width), "--n-y-pixels", str(g.n_y_pixels),
           "--n-z-pixels", str(g.n_z_pixels), "--s-z", repr(g.sigma_z),
           "--s-dl", repr(g.sigma_dl), "-i", "1", "-I", str(n_iter),
           "-T", str(threads), "-vv"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference failed ({p.returncode}): {p.stderr}")
    m = re.search(r"# av\s+([0-9.]+)", p.stdout)
    if not m:
        raise RuntimeError("no '# av' line in reference output:\n" + p.stdout)
    return float(m.group(1)), p.stdout

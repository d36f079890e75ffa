"""TEST INFRASTRUCTURE ONLY -- Python side of the 3D hybrid oracle.

ctypes binding of libhybrid_oracle.so (the C++ restatement in
hybrid_oracle.cpp of src/3d/hybrid/reconstruction.h) and a runner for the
reference's own 3d_hybrid_reconstruction built under oracle/_ref.  Only
tests/, bench.py's reference arm and __graft_entry__.smoke() use this
module, and only as the checker.
"""
import ctypes
import glob
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libhybrid_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "3d_hybrid_reconstruction")
REF_BIN_NOCONTRACT = os.path.join(HERE, "_ref", "3d_hybrid_reconstruction_nocontract")


class Setup(ctypes.Structure):
    _fields_ = [("n_columns", ctypes.c_int32), ("n_rows", ctypes.c_int32),
                ("n_planes", ctypes.c_int32), ("pixel_size", ctypes.c_float),
                ("z_left", ctypes.c_float), ("length", ctypes.c_float),
                ("sigma_z", ctypes.c_float), ("sigma_dl", ctypes.c_float)]


FRAME = np.dtype([("lor_index", "<i4"), ("plane_begin", "<i2"), ("plane_end", "<i2"),
                  ("info_begin", "<i8"), ("info_end", "<i8"), ("up", "<f4"), ("right", "<f4"),
                  ("tan", "<f4"), ("sec", "<f4")])


class Stats(ctypes.Structure):
    _fields_ = [("used_events", ctypes.c_int64), ("used_pixels", ctypes.c_int64),
                ("used_voxels", ctypes.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "libhybrid_oracle.so"], check=True,
                           capture_output=True)
        _lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        _lib.hyb_soa_from_matrix.restype = ctypes.c_int64
        _lib.hyb_soa_from_matrix.argtypes = [ctypes.POINTER(Setup), ctypes.c_int32, vp,
                                             ctypes.c_int64] + [vp] * 5 + [
            ctypes.c_uint32, vp, ctypes.c_int32] + [vp] * 6
        _lib.hyb_sensitivity.argtypes = [ctypes.POINTER(Setup), ctypes.c_int64, vp, vp, vp]
        _lib.hyb_normalize.argtypes = [ctypes.c_int64, ctypes.POINTER(Setup), vp, vp, vp]
        _lib.hyb_frame_events.restype = ctypes.c_int64
        _lib.hyb_frame_events.argtypes = [ctypes.POINTER(Setup), ctypes.c_int64] + [vp] * 6 + [
            ctypes.c_int64, ctypes.c_int64] + [vp] * 7
        for name in ("hyb_mlem_f32", "hyb_mlem_f64"):
            getattr(_lib, name).argtypes = [ctypes.POINTER(Setup)] + [vp] * 5 + [
                ctypes.c_int64, vp, ctypes.c_int32, ctypes.POINTER(Stats)]
        _lib.hyb_kernel_f32.restype = ctypes.c_float
        _lib.hyb_kernel_f32.argtypes = [ctypes.POINTER(Setup)] + [ctypes.c_float] * 7
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def setup(n_columns, n_rows, n_planes, pixel_size, z_left, length, sigma_z, sigma_dl):
    return Setup(n_columns, n_rows, n_planes, pixel_size, z_left, length, sigma_z, sigma_dl)


def soa_from_matrix(s, centers, matrix, inactive=None):
    """GeometrySOA(matrix, centres, grid, inactive) -> dict of flat arrays."""
    c = np.ascontiguousarray(centers, np.float32)
    nd = len(c)
    n_lors = (nd + 1) * nd // 2
    n = len(matrix)
    seg = np.zeros((n_lors, 9), np.float32)
    pix = np.zeros((n, 2), np.int16)
    pos = np.zeros(n, np.float32)
    w = np.zeros(n, np.float32)
    lb = np.zeros(n_lors, np.int64)
    le = np.zeros(n_lors, np.int64)
    ina = None if inactive is None else np.ascontiguousarray(inactive, np.int16)
    k = lib().hyb_soa_from_matrix(
        ctypes.byref(s), nd, _p(c), n, _p(matrix.lor_a), _p(matrix.lor_b), _p(matrix.px),
        _p(matrix.py), _p(matrix.hits), matrix.n_emissions, _p(ina),
        0 if ina is None else len(ina), _p(seg), _p(pix), _p(pos), _p(w), _p(lb), _p(le))
    if k < 0:
        raise ValueError("invalid matrix")
    return {"seg": seg, "pix": pix[:k].copy(), "pos": pos[:k].copy(), "w": w[:k].copy(),
            "lbeg": lb, "lend": le}


def segments9(seg4):
    """LineSegment(start, end) per LOR in binary32 (line_segment.h:18-27):
    start, end, mid point, direction, length -- the 9-float layout."""
    q = np.asarray(seg4, np.float32).reshape(-1, 4)
    sx, sy, ex, ey = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    vx, vy = ex - sx, ey - sy
    with np.errstate(divide="ignore", invalid="ignore"):
        ln = np.sqrt(vx * vx + vy * vy)
        out = np.stack([sx, sy, ex, ey, (sx + ex) / np.float32(2), (sy + ey) / np.float32(2),
                        vx / ln, vy / ln, np.sqrt(vx * vx + vy * vy)], 1)
    return out.astype(np.float32)


def geo_from_soa(soa):
    """The oracle's geometry dict from flat GeometrySOA arrays."""
    return {"seg": segments9(soa["segments"]), "pix": np.ascontiguousarray(soa["pixels"], np.int16),
            "pos": np.ascontiguousarray(soa["positions"], np.float32),
            "w": np.ascontiguousarray(soa["weights"], np.float32),
            "lbeg": np.asarray(soa["lor_begin"], np.int64),
            "lend": np.asarray(soa["lor_end"], np.int64)}


def sensitivity(s, geo):
    sens = np.zeros((s.n_rows, s.n_columns), np.float32)
    lib().hyb_sensitivity(ctypes.byref(s), len(geo["w"]), _p(geo["pix"]), _p(geo["w"]),
                          _p(sens))
    return sens


def normalize(s, geo, sens):
    w = geo["w"].copy()
    lib().hyb_normalize(len(w), ctypes.byref(s), _p(geo["pix"]), _p(w),
                        _p(np.ascontiguousarray(sens, np.float32)))
    return w


def frame_events(s, geo, w, first, second, z_up, z_dn, dl):
    """-> (frames structured array, keep mask)."""
    n = len(first)
    frames = np.zeros(n, FRAME)
    keep = np.zeros(n, np.uint8)
    a = [np.ascontiguousarray(x, t) for x, t in ((first, np.int16), (second, np.int16),
                                                  (z_up, np.float32), (z_dn, np.float32),
                                                  (dl, np.float32))]
    k = lib().hyb_frame_events(ctypes.byref(s), len(geo["lbeg"]), _p(geo["seg"]),
                               _p(geo["pix"]), _p(geo["pos"]), _p(np.ascontiguousarray(w)),
                               _p(geo["lbeg"]), _p(geo["lend"]), len(geo["pos"]), n,
                               *[_p(x) for x in a], _p(frames), _p(keep))
    return frames[:k].copy(), keep.astype(bool)


def mlem(s, geo, w, sens, frames, n_iter, rho=None, f64=False):
    """n_iter iterations; returns (image (n_planes, n_rows, n_columns), stats)."""
    t = np.float64 if f64 else np.float32
    shape = (s.n_planes, s.n_rows, s.n_columns)
    r = np.ones(shape, t) if rho is None else np.array(rho, t).reshape(shape)
    st = Stats()
    fn = lib().hyb_mlem_f64 if f64 else lib().hyb_mlem_f32
    fn(ctypes.byref(s), _p(geo["seg"]), _p(geo["pix"]), _p(np.ascontiguousarray(w, np.float32)),
       _p(np.ascontiguousarray(sens, np.float32)), _p(frames), len(frames), _p(r), n_iter,
       ctypes.byref(st))
    return r, {"used_events": st.used_events, "used_pixels": st.used_pixels,
               "used_voxels": st.used_voxels}


def reconstruct(s, centers, matrix, responses, n_iter, sens_mode="calculate", f64=False,
                inactive=None):
    """The whole CPU path: geometry, sensitivity, normalisation, frames, MLEM."""
    geo = soa_from_matrix(s, centers, matrix, inactive)
    if sens_mode == "calculate":
        sens = sensitivity(s, geo)
    elif sens_mode == "one":
        sens = np.ones((s.n_rows, s.n_columns), np.float32)
    else:
        sens = np.ascontiguousarray(sens_mode, np.float32).reshape(s.n_rows, s.n_columns)
    w = normalize(s, geo, sens)
    frames, keep = frame_events(s, geo, w, *responses)
    img, st = mlem(s, geo, w, sens, frames, n_iter, f64=f64)
    return {"geo": geo, "sens": sens, "w": w, "frames": frames, "keep": keep, "rho": img,
            "stats": st}


def ref_available(nocontract=True):
    return os.path.exists(REF_BIN_NOCONTRACT if nocontract else REF_BIN)


def run_ref(workdir, matrix_path, detector_path, symmetry_path, responses_path, n_pixels,
            pixel_size, n_planes, z_left, length, sigma_z, sigma_dl, n_iter, threads=1,
            nocontract=True, extra=(), timeout=3600):
    """Runs the reference's 3d_hybrid_reconstruction (--system matrix path)
    and returns the image after n_iter iterations (n_planes, n, n)."""
    exe = REF_BIN_NOCONTRACT if nocontract else REF_BIN
    out = os.path.join(workdir, "rho.bin")
    cmd = [exe, "--system", matrix_path, "--detector-file", detector_path,
           "--detector-file-sym", symmetry_path, "-n", str(n_pixels), "-p", repr(pixel_size),
           "--n-planes", str(n_planes), "--z-left", repr(z_left), "--length", repr(length),
           "--s-z", repr(sigma_z), "--s-dl", repr(sigma_dl), "-i", "1", "-I", str(n_iter),
           "-T", str(threads), "-o", out, *extra, responses_path]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=workdir)
    if p.returncode != 0:
        raise RuntimeError(f"reference failed ({p.returncode}): {p.stderr[-2000:]}")
    files = sorted(f for f in glob.glob(os.path.join(workdir, "rho_*"))
                   if not f.endswith(".nrrd"))
    if not files:
        raise RuntimeError(f"no reference output in {workdir}: {os.listdir(workdir)}")
    img = np.fromfile(files[-1], np.float32)
    return img.reshape(n_planes, n_pixels, n_pixels), p.stderr


def ref_naive(workdir, n_pixels, n_planes):
    """The naive image (event points counted per voxel, int32) that
    run_ref's reference call wrote to rho.bin."""
    return np.fromfile(os.path.join(workdir, "rho.bin"), np.int32).reshape(
        n_planes, n_pixels, n_pixels)


def tempdir():
    return tempfile.mkdtemp(prefix="hybref_")

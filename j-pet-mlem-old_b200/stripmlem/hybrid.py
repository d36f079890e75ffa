"""3D hybrid list-mode TOF MLEM on the B200: the host side of include/hybridmlem.h.

The reference's 3D hybrid reconstruction (src/3d/hybrid/reconstruction.h)
combines the 2D barrel's LOR geometry (a system matrix's pixels per LOR,
flattened into a GeometrySOA, src/2d/barrel/geometry_soa.h) with the strip
TOF kernel along z.  This module holds

* HybridReconstruction -- the device reconstruction (C ABI in
  lib/libstripmlem.so; no CPU fallback);
* the reference's file formats the CLI reads: the full sparse system matrix
  (PETP, src/2d/barrel/sparse_matrix.h:42-68), the detector description file
  (ScannerBuilder::deserialize, src/2d/barrel/scanner_builder.h:21-35), the
  identity symmetry file (SymmetryDescriptor::deserialize,
  symmetry_descriptor.h:111-125) and binary / text responses
  (Scanner::Response, src/3d/hybrid/scanner.h:71-95);
* a ring-of-square-detectors barrel (ScannerBuilder::build_multiple_rings,
  scanner_builder.h:37-230), and seeded synthetic inputs: an analytic system
  matrix (pixels whose centre lies within the LOR's detector width, weights
  falling off linearly with the distance) and responses of emissions in a
  phantom of z-cylinders.  These stand in for the Monte-Carlo matrix of
  2d_barrel_matrix and the events of 3d_hybrid_phantom.
"""
import ctypes
import math
import struct

import numpy as np

from . import _lib

_PETP = struct.unpack("<I", b"PETP")[0]
_PETp = struct.unpack("<I", b"PETp")[0]


class HybridError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_lib.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def _vp(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


# --- barrel ------------------------------------------------------------------

class Barrel:
    """Rings of square detectors (ScannerBuilder::build_multiple_rings).

    Ring 0 holds detector k at angle 2 pi k / n; ring i > 0 is turned by a
    further 2 pi rotation[i] / n, as the reference builds them.  Each
    detector is a w x h rectangle whose inner face lies at the ring's radius.
    `polygons` (n, 4, 2) float32; `centers` (n, 2) float32 is
    PolygonalDetector::center(), the binary32 mean of the four vertices."""

    def __init__(self, radius=(0.4155, 0.458, 0.5655), n_detectors=(48, 48, 96),
                 rotation=(0.0, 0.5, 0.5), w_detector=0.007, h_detector=0.019):
        polys = []
        w, h = float(w_detector), float(h_detector)
        base = np.array([(w / 2, h / 2), (w / 2, -h / 2), (-w / 2, -h / 2), (-w / 2, h / 2)])
        for ring, (r, n) in enumerate(zip(radius, n_detectors)):
            rot = rotation[ring] if ring < len(rotation) else 0.0
            b = base + (0.0, r + h / 2)
            for k in range(n):
                a = 2 * math.pi * k / n - math.pi / 2
                if ring > 0:
                    a += 2 * math.pi * rot / n
                c, s = math.cos(a), math.sin(a)
                polys.append(np.stack([b[:, 0] * c - b[:, 1] * s, b[:, 0] * s + b[:, 1] * c], 1))
        self.polygons = np.asarray(polys, np.float32)
        self.centers = detector_centers(self.polygons)
        self.n_detectors = len(self.polygons)

    def write_detector_file(self, path):
        write_detector_file(path, self.polygons)


def detector_centers(polygons):
    """PolygonalDetector::center() in binary32 (src/2d/geometry/polygon.h:57-68)."""
    p = np.asarray(polygons, np.float32)
    cx = np.zeros(len(p), np.float32)
    cy = np.zeros(len(p), np.float32)
    for k in range(p.shape[1]):
        cx = cx + p[:, k, 0]
        cy = cy + p[:, k, 1]
    n = np.float32(p.shape[1])
    return np.stack([cx / n, cy / n], 1).astype(np.float32)


def write_detector_file(path, polygons):
    """One line per detector: its vertices' x y pairs, to binary32 round trip."""
    with open(path, "w") as f:
        for poly in np.asarray(polygons, np.float32):
            f.write(" ".join(f"{float(x):.9g} {float(y):.9g}" for x, y in poly) + "\n")


def read_detector_file(path):
    polys = []
    with open(path) as f:
        for line in f:
            v = [float(x) for x in line.split()]
            if v:
                polys.append(np.asarray(v, np.float32).reshape(-1, 2))
    return np.asarray(polys, np.float32)


def write_symmetry_file(path, n_detectors):
    """A symmetry descriptor file whose eight symmetries map every detector to
    itself.  The reconstruction never reads the symmetries, but the reader
    stores them at detector * 8 + symmetry whatever count the file declares
    (symmetry_descriptor.h:94-97, :111-125), so the file declares eight."""
    with open(path, "w") as f:
        f.write(f"{n_detectors} 8\n")
        for d in range(n_detectors):
            f.write(f"{d}" + f" {d}" * 8 + "\n")


# --- system matrix ----------------------------------------------------------

class SystemMatrix:
    """A full (PETP) 2D barrel system matrix as flat arrays: element i is the
    pixel (px[i], py[i]) of LOR (lor_a[i], lor_b[i]) with hits[i]."""

    def __init__(self, n_pixels_in_row, n_emissions, n_detectors, lor_a, lor_b, px, py, hits):
        self.n_pixels_in_row = int(n_pixels_in_row)
        self.n_emissions = int(n_emissions)
        self.n_detectors = int(n_detectors)
        self.lor_a = np.ascontiguousarray(lor_a, np.uint16)
        self.lor_b = np.ascontiguousarray(lor_b, np.uint16)
        self.px = np.ascontiguousarray(px, np.uint16)
        self.py = np.ascontiguousarray(py, np.uint16)
        self.hits = np.ascontiguousarray(hits, np.uint32)

    def __len__(self):
        return len(self.hits)

    def write(self, path):
        """SparseMatrix operator<< (sparse_matrix.h:301-347), full form."""
        first = np.maximum(self.lor_a, self.lor_b)
        second = np.minimum(self.lor_a, self.lor_b)
        order = np.lexsort((self.px, self.py, second, first))
        f, s = first[order], second[order]
        x, y, h = self.px[order], self.py[order], self.hits[order]
        key = f.astype(np.int64) * 65536 + s
        starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
        ends = np.r_[starts[1:], len(key)]
        rec = np.zeros(len(h), dtype=[("x", "<u2"), ("y", "<u2"), ("h", "<u4")])
        rec["x"], rec["y"], rec["h"] = x, y, h
        with open(path, "wb") as out:
            out.write(struct.pack("<IIII", _PETP, self.n_pixels_in_row, self.n_emissions,
                                  self.n_detectors))
            for b, e in zip(starts, ends):
                out.write(struct.pack("<HHI", int(f[b]), int(s[b]), int(e - b)))
                out.write(rec[b:e].tobytes())

    @classmethod
    def read(cls, path):
        """SparseMatrix(util::ibstream&) (sparse_matrix.h:163-235), full non-TOF form."""
        data = open(path, "rb").read()
        magic, n_pix, n_em, n_det = struct.unpack_from("<IIII", data, 0)
        if magic == _PETp:
            raise ValueError("matrix must be in full form (2d_barrel_matrix --full)")
        if magic != _PETP:
            raise ValueError("not a full PETP system matrix")
        off = 16
        la, lb, xs, ys, hs = [], [], [], [], []
        rec_t = np.dtype([("x", "<u2"), ("y", "<u2"), ("h", "<u4")])
        while off + 8 <= len(data):
            a, b, count = struct.unpack_from("<HHI", data, off)
            off += 8
            rec = np.frombuffer(data, rec_t, count, off)
            off += 8 * count
            la.append(np.full(count, a, np.uint16))
            lb.append(np.full(count, b, np.uint16))
            xs.append(rec["x"])
            ys.append(rec["y"])
            hs.append(rec["h"])
        cat = (lambda v, t: np.concatenate(v).astype(t) if v else np.zeros(0, t))
        return cls(n_pix, n_em, n_det, cat(la, np.uint16), cat(lb, np.uint16),
                   cat(xs, np.uint16), cat(ys, np.uint16), cat(hs, np.uint32))


def synthetic_matrix(barrel, n_pixels, pixel_size, fov_radius, n_emissions=100000,
                     peak_hits=1000, chunk=256):
    """Analytic stand-in for a Monte-Carlo system matrix.  LOR (i, j) holds
    every pixel inside the field of view whose centre lies within the LOR's
    half-width (the largest vertex distances of its two detectors from the
    line between their centres, as 2d_barrel_geometry measures the LOR
    width, plus half a pixel) strictly between the two centres; its hits
    fall linearly from peak_hits on the line to 1 at the edge."""
    n = int(n_pixels)
    p = np.float64(pixel_size)
    ll = -p * n / 2
    ix, iy = np.meshgrid(np.arange(n), np.arange(n))
    ix, iy = ix.ravel(), iy.ravel()
    cx = ll + (ix + 0.5) * p
    cy = ll + (iy + 0.5) * p
    inside = cx * cx + cy * cy <= fov_radius * fov_radius
    ix, iy, cx, cy = ix[inside], iy[inside], cx[inside], cy[inside]
    cen = barrel.centers.astype(np.float64)
    poly = barrel.polygons.astype(np.float64)
    nd = barrel.n_detectors
    fa, fb = np.tril_indices(nd, -1)  # first > second
    out_a, out_b, out_x, out_y, out_h = [], [], [], [], []
    for s0 in range(0, len(fa), chunk):
        a, b = fa[s0:s0 + chunk], fb[s0:s0 + chunk]
        st, en = cen[b], cen[a]
        v = en - st
        ln = np.hypot(v[:, 0], v[:, 1])
        d = v / ln[:, None]
        nrm = np.stack([-d[:, 1], d[:, 0]], 1)
        off = (st * nrm).sum(1)
        wa = np.abs((poly[a] * nrm[:, None, :]).sum(2) - off[:, None]).max(1)
        wb = np.abs((poly[b] * nrm[:, None, :]).sum(2) - off[:, None]).max(1)
        half = (wa + wb) / 2 + p / 2
        dist = cx[None, :] * nrm[:, 0:1] + cy[None, :] * nrm[:, 1:2] - off[:, None]
        t = ((cx[None, :] - st[:, 0:1]) * d[:, 0:1] + (cy[None, :] - st[:, 1:2]) * d[:, 1:2]) \
            / ln[:, None]
        m = (np.abs(dist) < half[:, None]) & (t > 0) & (t < 1)
        li, pi = np.nonzero(m)
        hits = 1 + np.floor((peak_hits - 1) * (1 - np.abs(dist[li, pi]) / half[li]))
        out_a.append(a[li])
        out_b.append(b[li])
        out_x.append(ix[pi])
        out_y.append(iy[pi])
        out_h.append(hits)
    cat = np.concatenate
    return SystemMatrix(n, n_emissions, nd, cat(out_a), cat(out_b), cat(out_x), cat(out_y),
                        cat(out_h))


# --- responses ---------------------------------------------------------------

_RESP = np.dtype([("first", "<i2"), ("second", "<i2"), ("z_up", "<f4"), ("z_dn", "<f4"),
                  ("dl", "<f4")])


def write_responses(path, first, second, z_up, z_dn, dl):
    """Binary responses as Scanner::Response(util::ibstream&) reads them
    (LOR as two int16, then z_up, z_dn, dl binary32; 16 bytes each)."""
    r = np.zeros(len(first), _RESP)
    r["first"], r["second"], r["z_up"], r["z_dn"], r["dl"] = first, second, z_up, z_dn, dl
    r.tofile(path)


def read_responses_text(path):
    """Text responses `first second z_up z_dn dl` parsed as the reference's
    fast loader parses them (fast_load_txt_events, reconstruction.h:163-186,
    util::text_parser::read_lines: a line counts when it ends in a newline),
    by the library's parser (hybrid_parse_responses_text)."""
    data = open(path, "rb").read()
    n = data.count(b"\n")
    first = np.empty(n, np.int16)
    second = np.empty(n, np.int16)
    zu = np.empty(n, np.float32)
    zd = np.empty(n, np.float32)
    dl = np.empty(n, np.float32)
    got = ctypes.c_int64()
    rc = _lib.load().hybrid_parse_responses_text(data, len(data), n, _vp(first), _vp(second),
                                                 _vp(zu), _vp(zd), _vp(dl), ctypes.byref(got))
    if rc != _lib.STRIP_OK:
        raise ValueError(f"{path}: malformed number on line {got.value + 1}")
    return first, second, zu, zd, dl


def read_responses(path):
    """Binary (16-byte records) or, for *.txt, text lines `first second z_up
    z_dn dl` (parsed as the reference parses them)."""
    if str(path).endswith(".txt"):
        return read_responses_text(path)
    r = np.fromfile(path, _RESP)
    return (r["first"].copy(), r["second"].copy(), r["z_up"].copy(), r["z_dn"].copy(),
            r["dl"].copy())


def generate_responses(barrel, phantom, n, length, sigma_z, sigma_dl, seed=1, device=-1):
    """Seeded synthetic responses (hybrid_generate_responses).  `phantom` is
    a list of z-cylinders (x, y, z, radius, half_length, activity); overlaps
    are exclusive, the first cylinder on top.  Emissions are isotropic; each
    photon is taken by the first detector its 2D line crosses (rings inwards
    out), at the projection of that detector's centre on the line, when it
    lies within |z| <= length / 2.  first = the larger detector index ("up"),
    dl = l_up - l_dn of the 3D path lengths, smeared with N(0, sigma_z) and
    N(0, sigma_dl).  device < 0 runs on the host (OpenMP), otherwise on that
    CUDA device; response i depends only on (seed, i)."""
    lib = _lib.load()
    poly = np.ascontiguousarray(barrel.polygons, np.float32)
    ph = list(phantom)
    cyl = (_lib.HybridCylinder * len(ph))(*[_lib.HybridCylinder(*map(float, c)) for c in ph])
    first = np.empty(n, np.int16)
    second = np.empty(n, np.int16)
    zu = np.empty(n, np.float32)
    zd = np.empty(n, np.float32)
    dl = np.empty(n, np.float32)
    rc = lib.hybrid_generate_responses(len(poly), _vp(poly), cyl, len(ph), length, sigma_z,
                                       sigma_dl, seed, n, device, _vp(first), _vp(second),
                                       _vp(zu), _vp(zd), _vp(dl))
    if rc != _lib.STRIP_OK:
        raise HybridError(rc, "hybrid_generate_responses")
    return first, second, zu, zd, dl


# --- the device reconstruction --------------------------------------------------

class HybridReconstruction:
    """PET3D::Hybrid::Reconstruction on one B200 (include/hybridmlem.h).

    Order of use, as run_reconstruction (reconstruction_cmd.cpp:457-680):
    set_geometry_from_matrix, set_sensitivity, set_responses, then call with
    the number of iterations.  The image (rho) starts at 1; its numpy shape is
    (n_planes, n_rows, n_columns)."""

    def __init__(self, n_columns, n_rows, n_planes, pixel_size, z_left, length, sigma_z,
                 sigma_dl, device=0):
        self.lib = _lib.load()
        self.setup = _lib.HybridSetup(n_columns, n_rows, n_planes, 0, pixel_size, z_left,
                                      length, sigma_z, sigma_dl)
        self.shape = (int(n_planes), int(n_rows), int(n_columns))
        self.device = int(device)
        ctx = ctypes.c_void_p()
        rc = self.lib.hybrid_ctx_create(ctypes.byref(self.setup), device, ctypes.byref(ctx))
        if rc != _lib.STRIP_OK:
            raise HybridError(rc, "hybrid_ctx_create")
        self._ctx = ctx

    def _check(self, rc):
        if rc != _lib.STRIP_OK:
            msg = self.lib.hybrid_last_error(self._ctx) or b""
            raise HybridError(rc, msg.decode(errors="replace"))

    def close(self):
        if getattr(self, "_ctx", None):
            self.lib.hybrid_ctx_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def set_geometry_from_matrix(self, centers, matrix, inactive=None):
        c = np.ascontiguousarray(centers, np.float32)
        ina = None if inactive is None else np.ascontiguousarray(inactive, np.int16)
        self._check(self.lib.hybrid_set_geometry_from_matrix(
            self._ctx, len(c), _vp(c), len(matrix), _vp(matrix.lor_a), _vp(matrix.lor_b),
            _vp(matrix.px), _vp(matrix.py), _vp(matrix.hits), matrix.n_emissions, _vp(ina),
            0 if ina is None else len(ina)))

    def set_geometry_soa(self, n_detectors, segments, pixels, positions, weights, lor_begin,
                         lor_end):
        """A flattened geometry as the reference's GPU run() receives it:
        segments (n_lors, 4) start / end points, pixels (n, 2), positions,
        weights, per-LOR [lor_begin, lor_end)."""
        seg = np.ascontiguousarray(segments, np.float32).reshape(-1, 4)
        pix = np.ascontiguousarray(pixels, np.int16).reshape(-1, 2)
        pos = np.ascontiguousarray(positions, np.float32)
        w = np.ascontiguousarray(weights, np.float32)
        lb = np.ascontiguousarray(lor_begin, np.uint64)
        le = np.ascontiguousarray(lor_end, np.uint64)
        self._check(self.lib.hybrid_set_geometry_soa(self._ctx, n_detectors, _vp(seg), len(pos),
                                                     _vp(pix), _vp(pos), _vp(w), _vp(lb),
                                                     _vp(le)))

    def set_frames(self, lor, info_begin, info_end, plane_begin, plane_end, up, right, tan, sec):
        """Frame events as the reference's GPU run() receives them."""
        a = [np.ascontiguousarray(x, t) for x, t in (
            (lor, np.int32), (info_begin, np.int64), (info_end, np.int64),
            (plane_begin, np.int16), (plane_end, np.int16), (up, np.float32),
            (right, np.float32), (tan, np.float32), (sec, np.float32))]
        self._check(self.lib.hybrid_set_frames(self._ctx, len(a[0]), *[_vp(x) for x in a]))

    def set_sensitivity(self, sensitivity="calculate", given=False):
        """'calculate', 'one' or a 2D map; with given=True the map is used as
        is and the weights are taken as normalised already."""
        if given:
            s = np.ascontiguousarray(sensitivity, np.float32).reshape(-1)
            self._check(self.lib.hybrid_set_sensitivity(self._ctx, _lib.HYBRID_SENS_GIVEN,
                                                        _vp(s)))
            return
        if isinstance(sensitivity, str):
            mode = {"calculate": _lib.HYBRID_SENS_CALCULATE, "one": _lib.HYBRID_SENS_ONE}[sensitivity]
            self._check(self.lib.hybrid_set_sensitivity(self._ctx, mode, None))
        else:
            s = np.ascontiguousarray(sensitivity, np.float32).reshape(-1)
            if s.size != self.shape[1] * self.shape[2]:
                raise ValueError("external sensitivity must be n_rows x n_columns")
            self._check(self.lib.hybrid_set_sensitivity(self._ctx, _lib.HYBRID_SENS_EXTERNAL,
                                                        _vp(s)))

    def set_responses(self, first, second, z_up, z_dn, dl):
        a = np.ascontiguousarray(first, np.int16)
        b = np.ascontiguousarray(second, np.int16)
        zu = np.ascontiguousarray(z_up, np.float32)
        zd = np.ascontiguousarray(z_dn, np.float32)
        d = np.ascontiguousarray(dl, np.float32)
        self._check(self.lib.hybrid_set_responses(self._ctx, _vp(a), _vp(b), _vp(zu), _vp(zd),
                                                  _vp(d), len(a)))

    def __call__(self, n_iterations=1, progress=None):
        cb = _lib.HYBRID_PROGRESS_CB(
            (lambda it, fin, user: progress(it, bool(fin))) if progress else (lambda *a: None))
        self._check(self.lib.hybrid_iterate(self._ctx, n_iterations, cb, None))
        return self

    # split iteration for event-sharded runs (stripmlem.distributed.ShardedHybrid)
    @property
    def n_voxels(self):
        return self.shape[0] * self.shape[1] * self.shape[2]

    @property
    def torch_device(self):
        import torch
        return torch.device("cuda", self.device)

    def set_accumulator(self, acc):
        """acc: a CUDA float32 tensor of n_voxels on this device, or None."""
        ptr = None if acc is None else ctypes.c_void_p(acc.data_ptr())
        self._acc_ref = acc
        self._check(self.lib.hybrid_set_accumulator(self._ctx, ptr))

    def accumulate(self):
        self._check(self.lib.hybrid_accumulate(self._ctx))

    def update(self):
        self._check(self.lib.hybrid_update(self._ctx))

    @property
    def rho(self):
        out = np.empty(self.shape, np.float32)
        self._check(self.lib.hybrid_get_image(self._ctx, _vp(out)))
        return out

    @rho.setter
    def rho(self, value):
        v = np.ascontiguousarray(value, np.float32).reshape(self.shape)
        self._check(self.lib.hybrid_set_image(self._ctx, _vp(v)))

    @property
    def sensitivity(self):
        out = np.empty(self.shape[1:], np.float32)
        self._check(self.lib.hybrid_get_sensitivity(self._ctx, _vp(out)))
        return out

    def stats(self):
        st = _lib.HybridStats()
        self._check(self.lib.hybrid_get_stats(self._ctx, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.HybridStats._fields_ if k != "reserved"}

    def geometry(self):
        st = self.stats()
        nl, ni = st["n_lors"], st["n_pixel_infos"]
        seg = np.empty((nl, 9), np.float32)
        pix = np.empty((ni, 2), np.int16)
        pos = np.empty(ni, np.float32)
        w = np.empty(ni, np.float32)
        lb = np.empty(nl, np.int64)
        le = np.empty(nl, np.int64)
        self._check(self.lib.hybrid_get_geometry(self._ctx, _vp(seg), _vp(pix), _vp(pos), _vp(w),
                                                 _vp(lb), _vp(le)))
        return {"seg": seg, "pix": pix, "pos": pos, "w": w, "lbeg": lb, "lend": le}

    def frames(self):
        n = self.stats()["n_events"]
        out = {"lor": np.empty(n, np.int32), "info_begin": np.empty(n, np.int64),
               "info_end": np.empty(n, np.int64), "plane_begin": np.empty(n, np.int16),
               "plane_end": np.empty(n, np.int16), "index": np.empty(n, np.int64)}
        self._check(self.lib.hybrid_get_frames(
            self._ctx, _vp(out["lor"]), _vp(out["info_begin"]), _vp(out["info_end"]),
            _vp(out["plane_begin"]), _vp(out["plane_end"]), _vp(out["index"])))
        return out


# --- GATE text converters (3d_tool_convert) ---------------------------------------

_CM = 0.01
_C_PS = 299792458.0e-12          # speed of light, m / ps
_C_SCINT_PS = 126000000.0e-12    # signal speed in the scintillator, m / ps


def _contains(polygons, x, y, tol):
    """Polygon::contains(p, tol) (src/2d/geometry/polygon.h:70-83) of every
    point against every detector, binary32 as the reference: -> (n, n_det)."""
    poly = np.asarray(polygons, np.float32)
    px = np.asarray(x, np.float32)[:, None]
    py = np.asarray(y, np.float32)[:, None]
    inside = np.ones((len(px), len(poly)), bool)
    start = poly[:, -1, :]
    for i in range(poly.shape[1]):
        end = poly[:, i, :]
        ex, ey = end[:, 0] - start[:, 0], end[:, 1] - start[:, 1]
        # cw_perpendicular (ey, -ex) . (p - start)
        d = ey[None, :] * (px - start[None, :, 0]) + (-ex)[None, :] * (py - start[None, :, 1])
        inside &= ~(d < np.float32(-tol))
        start = end
    return inside


def convert_warsaw(lines, polygons, length, sigma_z=0.0, sigma_dl=0.0, seed=0, only=0,
                   chunk=65536):
    """3d_tool_convert --warsaw (src/3d/tool/convert_cmd.cpp:86-162): GATE
    hit pairs `x1 y1 z1 t1 x2 y2 z2 t2 ... scatter` (cm, ps; the column count
    from the first line, scatter the last column) -> responses (first,
    second, z_up, z_dn, dl) in metres, binary64 as the reference prints them.
    Pairs with |z| > length / 2 are skipped, as are pairs whose scatter
    differs from `only` (when only != 0) and points inside no detector
    (Polygon::contains with tolerance 1e-4); the larger detector index comes
    first.  The Gaussian errors (sigma_z on z, sigma_dl on dl) are the
    reference's for the same seed: std::normal_distribution over
    std::mt19937_64 in output order (hybrid_smear_responses)."""
    rows = [ln.split() for ln in lines if ln.strip()]
    if not rows:
        z = np.zeros(0)
        return np.zeros(0, np.int16), np.zeros(0, np.int16), z, z, z
    n_col = len(rows[0])
    a = np.array([[float(v) for v in r[:8]] + [float(r[n_col - 1])] for r in rows])
    x1, y1, z1, t1, x2, y2, z2, t2, sc = a.T
    keep = ~((np.abs(z1 * _CM) > length / 2) | (np.abs(z2 * _CM) > length / 2))
    if only:
        keep &= sc.astype(np.int64) == only
    idx = np.flatnonzero(keep)
    d1 = np.full(len(a), -1, np.int64)
    d2 = np.full(len(a), -1, np.int64)
    n_det = len(polygons)
    for s in range(0, len(idx), chunk):
        k = idx[s:s + chunk]
        for pts, dd in (((x1, y1), d1), ((x2, y2), d2)):
            inside = _contains(polygons, pts[0][k] * _CM, pts[1][k] * _CM, 0.0001)
            last = n_det - 1 - np.argmax(inside[:, ::-1], axis=1)  # the last detector wins
            dd[k] = np.where(inside.any(1), last, -1)
    ok = keep & (d1 >= 0) & (d2 >= 0)
    d1, d2, z1, z2, t1, t2 = d1[ok], d2[ok], z1[ok], z2[ok], t1[ok], t2[ok]
    sw = d1 < d2
    d1, d2 = np.where(sw, d2, d1), np.where(sw, d1, d2)
    z1, z2 = np.where(sw, z2, z1), np.where(sw, z1, z2)
    t1, t2 = np.where(sw, t2, t1), np.where(sw, t1, t2)
    dl = np.ascontiguousarray((t1 - t2) * _C_PS)
    zu = np.ascontiguousarray(z1 * _CM)
    zd = np.ascontiguousarray(z2 * _CM)
    rc = _lib.load().hybrid_smear_responses(int(seed), float(sigma_z), float(sigma_dl), len(d1),
                                            _vp(zu), _vp(zd), _vp(dl))
    if rc != _lib.STRIP_OK:
        raise HybridError(rc, "hybrid_smear_responses")
    return d1.astype(np.int16), d2.astype(np.int16), zu, zd, dl


def convert_tbednarski(lines, relative_time=False):
    """3d_tool_convert --tbednarski (convert_cmd.cpp:164-211): records
    `du dd t_ul t_ur t_dl t_dr` (detectors from 1, times in ps).  Default:
    responses (first, second, z_up, z_dn, dl) with the larger detector first
    (its times swapped along), indices from 0, z = c_scint (t_l - t_r) / 2,
    dl = c ((t_ul + t_ur) - (t_dl + t_dr)) / 2.  relative_time: the records
    with every time less the record's smallest, detectors unchanged."""
    rows = [ln.split() for ln in lines if ln.strip()]
    if not rows:
        z = np.zeros(0)
        return (np.zeros(0, np.int64),) * 2 + (z,) * 4 if relative_time else \
            (np.zeros(0, np.int16),) * 2 + (z,) * 3
    du = np.array([int(r[0]) for r in rows])
    dd = np.array([int(r[1]) for r in rows])
    t = np.array([[float(v) for v in r[2:6]] for r in rows])
    tul, tur, tdl, tdr = t.T
    if relative_time:
        tmin = np.minimum(np.minimum(tur, tul), np.minimum(tdr, tdl))
        return du, dd, tul - tmin, tur - tmin, tdl - tmin, tdr - tmin
    sw = du < dd
    du, dd = np.where(sw, dd, du), np.where(sw, du, dd)
    tul, tdl = np.where(sw, tdl, tul), np.where(sw, tul, tdl)
    tur, tdr = np.where(sw, tdr, tur), np.where(sw, tur, tdr)
    zu = 0.5 * _C_SCINT_PS * (tul - tur)
    zd = 0.5 * _C_SCINT_PS * (tdl - tdr)
    dl = 0.5 * _C_PS * ((tul + tur) - (tdl + tdr))
    return (du - 1).astype(np.int16), (dd - 1).astype(np.int16), zu, zd, dl


# --- LOR geometry files (2d_barrel_geometry output, the --geometry input) ---------

_PETg = struct.unpack("<I", b"PETg")[0]
_PIXEL_INFO = np.dtype([("x", "<i2"), ("y", "<i2"), ("t", "<f4"), ("distance", "<f4"),
                        ("fill", "<f4"), ("weight", "<f4")])


def read_geometry(path):
    """A binary32 LOR geometry file (Geometry(util::ibstream&),
    src/2d/barrel/geometry.h: magic "PETg", n_detectors, the pixel grid,
    then per LOR its pair, segment start / end, width and pixel infos
    (pixel, t, distance, fill, weight)) -> dict with 'n_detectors',
    'grid' (n_columns, n_rows, pixel_size, lower_left x, y) and 'lors'
    {lor index: (segment (4,), width, pixel-info array)}."""
    data = open(path, "rb").read()
    magic, = struct.unpack_from("<I", data, 0)
    if magic != _PETg:
        raise ValueError("unknown binary geometry file")
    n_det, nc, nr, p, llx, lly = struct.unpack_from("<hhhfff", data, 4)
    off = 4 + 2 + 2 + 2 + 12
    lors = {}
    while off + 32 <= len(data):
        first, second, sx, sy, ex, ey, width, n = struct.unpack_from("<hhfffffQ", data, off)
        off += 32
        infos = np.frombuffer(data, _PIXEL_INFO, n, off).copy()
        off += 20 * n
        lors[first * (first + 1) // 2 + second] = (np.array([sx, sy, ex, ey], np.float32),
                                                   np.float32(width), infos)
    return {"n_detectors": int(n_det), "grid": (int(nc), int(nr), float(p), float(llx),
                                                 float(lly)), "lors": lors}


def write_geometry(path, n_detectors, grid, lors):
    """The inverse of read_geometry: every LOR of the table in index order
    (empty ones included, as Geometry's operator<< writes them)."""
    nc, nr, p, llx, lly = grid
    n_lors = (n_detectors + 1) * n_detectors // 2
    with open(path, "wb") as out:
        out.write(struct.pack("<Ihhhfff", _PETg, n_detectors, nc, nr, p, llx, lly))
        for first in range(n_detectors):
            for second in range(first + 1):
                li = first * (first + 1) // 2 + second
                seg, width, infos = lors.get(li, (np.zeros(4, np.float32), 0.0,
                                                  np.zeros(0, _PIXEL_INFO)))
                out.write(struct.pack("<hhfffffQ", first, second, *[float(v) for v in seg],
                                      float(width), len(infos)))
                out.write(np.asarray(infos, _PIXEL_INFO).tobytes())


def geometry_soa_from_file(geom, matrix=None):
    """GeometrySOA(Geometry) (geometry_soa.h:184-205: LORs in index order,
    pixel infos as stored, positions t, weights as stored) and, with a
    matrix, load_weights_from_matrix_file (geometry_soa.h:207-260: weights
    zeroed, then hits / n_emissions added to the info of each matrix element's
    pixel in its LOR) -> dict of flat arrays for HybridReconstruction.set_geometry_soa."""
    nd = geom["n_detectors"]
    n_lors = (nd + 1) * nd // 2
    seg = np.zeros((n_lors, 4), np.float32)
    lb = np.zeros(n_lors, np.uint64)
    le = np.zeros(n_lors, np.uint64)
    parts = []
    size = 0
    for li in range(n_lors):
        if li in geom["lors"]:
            sg, _, infos = geom["lors"][li]
            seg[li] = sg
            lb[li] = size
            parts.append(infos)
            size += len(infos)
            le[li] = size
    infos = np.concatenate(parts) if parts else np.zeros(0, _PIXEL_INFO)
    pix = np.stack([infos["x"], infos["y"]], 1).astype(np.int16)
    pos = infos["t"].astype(np.float32)
    w = infos["weight"].astype(np.float32).copy()
    if matrix is not None:
        w[:] = 0
        f32 = np.float32
        n_em = f32(matrix.n_emissions)
        first = np.maximum(matrix.lor_a, matrix.lor_b).astype(np.int64)
        second = np.minimum(matrix.lor_a, matrix.lor_b).astype(np.int64)
        order = np.lexsort((matrix.px, matrix.py, second, first))
        cur, idx, k, k_end = -1, None, 0, 0
        for e in order:
            li = int(first[e] * (first[e] + 1) // 2 + second[e])
            if li != cur:
                cur = li
                b0, b1 = int(lb[li]), int(le[li])
                idx = b0 + np.lexsort((pix[b0:b1, 0], pix[b0:b1, 1]))  # by y then x
                k, k_end = 0, b1 - b0
            px, py = int(matrix.px[e]), int(matrix.py[e])
            while k < k_end and (pix[idx[k], 1], pix[idx[k], 0]) < (py, px):
                k += 1
            if k == k_end or (py, px) < (pix[idx[k], 1], pix[idx[k], 0]):
                continue
            w[idx[k]] = f32(w[idx[k]] + f32(f32(matrix.hits[e]) / n_em))
    return {"n_detectors": nd, "segments": seg, "pixels": pix, "positions": pos, "weights": w,
            "lor_begin": lb, "lor_end": le}

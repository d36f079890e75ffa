"""Python host side of the B200 strip list-mode TOF MLEM library.

Mirrors the reference's operator interface for the 2D strip path
(JPETTomography/j-pet-mlem-old):

* ``Scanner``        -- Scanner<F, S> constructor arguments (src/2d/strip/scanner.h:39-67)
* ``Reconstruction`` -- Reconstruction<F, Kernel>: ``rho``, ``sensitivity``,
  ``responses`` and ``__call__(progress, n_iterations, n_iterations_so_far)``
  (src/2d/strip/reconstruction.h:42-154)
* ``run``            -- PET2D::Strip::GPU::Reconstruction::run with its output /
  progress / device-name callbacks (src/2d/strip/cuda/reconstruction.cu:32-113)

Everything calls the C ABI of lib/libstripmlem.so (include/stripmlem.h); the
arithmetic runs in the library's sm_100a kernels.  Errors raise StripError.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import (ACCUM_FP32, ACCUM_FP64, ACCUM_KAHAN, MODE_CPU, MODE_GPU,
                   STRIP_OK)

__all__ = [
    "Scanner", "Reconstruction", "StripError", "run", "generate_events",
    "MODE_CPU", "MODE_GPU", "ACCUM_FP32", "ACCUM_KAHAN", "ACCUM_FP64",
]


class StripError(RuntimeError):
    def __init__(self, code, message=""):
        self.code = code
        name = _lib.ERROR_NAMES.get(code, f"error {code}")
        super().__init__(f"{name}: {message}" if message else name)


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Scanner:
    """Scanner parameters (scanner.h:39-67 argument order).

    ``Scanner(radius, scintillator_length, n_y_pixels, n_z_pixels,
    pixel_height, pixel_width, sigma_z, sigma_dl, center_y=0, center_z=0)``
    """

    def __init__(self, radius, scintillator_length, n_y_pixels, n_z_pixels,
                 pixel_height, pixel_width, sigma_z, sigma_dl, center_y=0.0,
                 center_z=0.0):
        self.radius = float(radius)
        self.scintillator_length = float(scintillator_length)
        self.n_y_pixels = int(n_y_pixels)
        self.n_z_pixels = int(n_z_pixels)
        self.pixel_height = float(pixel_height)
        self.pixel_width = float(pixel_width)
        self.sigma_z = float(sigma_z)
        self.sigma_dl = float(sigma_dl)
        self.center_y = float(center_y)
        self.center_z = float(center_z)

    @classmethod
    def from_cli(cls, radius, length, s_pixel, s_z, s_dl, n_z_pixels=None,
                 n_y_pixels=None, n_pixels=None):
        """calculate_scanner_options + PET2D_STRIP_SCANNER_CL
        (options.cpp:106-124, options.h:42-50)."""
        import math
        if n_pixels:
            n_z_pixels = n_y_pixels = n_pixels
        if not n_z_pixels:
            n_z_pixels = int(math.ceil(length / s_pixel))
        if not n_y_pixels:
            n_y_pixels = int(math.ceil(2 * radius / s_pixel))
        return cls(radius, length, n_y_pixels, n_z_pixels, s_pixel, s_pixel,
                   s_z, s_dl)

    @property
    def total_n_pixels(self):
        return self.n_y_pixels * self.n_z_pixels

    def geometry(self):
        return _lib.Geometry(self.radius, self.scintillator_length,
                             self.n_y_pixels, self.n_z_pixels,
                             self.pixel_height, self.pixel_width,
                             self.sigma_z, self.sigma_dl, self.center_y,
                             self.center_z)

    def as_dict(self):
        return dict(vars(self))


class Reconstruction:
    """List-mode MLEM on the strip scanner, run by the library's kernels.

    ``mode`` selects the reference's CPU semantics (MODE_CPU: GaussianKernel,
    no sensitivity) or its ``--gpu`` semantics (MODE_GPU: AnalyticKernel with
    the 5-point pixel sensitivity in the denominator).
    """

    def __init__(self, scanner, device=0, mode=MODE_CPU, accumulation=ACCUM_KAHAN):
        self.lib = _lib.load()
        self.scanner = scanner
        self.mode = mode
        self._geom = scanner.geometry()
        ctx = ctypes.c_void_p()
        rc = self.lib.strip_ctx_create(ctypes.byref(self._geom), int(device),
                                       ctypes.byref(ctx))
        if rc != STRIP_OK:
            raise StripError(rc, "strip_ctx_create")
        self._ctx = ctx
        self.device = int(device)
        self.torch_device = f"cuda:{self.device}"
        self.n_events = 0
        self.n_subsets = 1
        self._check(self.lib.strip_set_accumulation(self._ctx, accumulation))

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc):
        if rc != STRIP_OK:
            buf = ctypes.create_string_buffer(512)
            if self._ctx:
                self.lib.strip_last_error(self._ctx, buf, 512)
            raise StripError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "_ctx", None):
            self.lib.strip_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def device_name(self):
        buf = ctypes.create_string_buffer(256)
        self._check(self.lib.strip_device_name(self._ctx, buf, 256))
        return buf.value.decode()

    def stats(self):
        s = _lib.Stats()
        self._check(self.lib.strip_get_stats(self._ctx, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def set_accumulation(self, accum):
        self._check(self.lib.strip_set_accumulation(self._ctx, int(accum)))

    # -- events -----------------------------------------------------------
    def set_events(self, z_u, z_d, dl, n_subsets=1):
        z_u = np.ascontiguousarray(z_u, dtype=np.float32)
        z_d = np.ascontiguousarray(z_d, dtype=np.float32)
        dl = np.ascontiguousarray(dl, dtype=np.float32)
        n = z_u.shape[0]
        if z_d.shape[0] != n or dl.shape[0] != n:
            raise StripError(_lib.STRIP_E_INVALID, "z_u, z_d, dl sizes differ")
        self._check(self.lib.strip_set_events(self._ctx, _fp(z_u), _fp(z_d),
                                              _fp(dl), n, int(n_subsets)))
        self.n_events = n
        self.n_subsets = int(n_subsets)

    def set_events_device(self, z_u, z_d, dl, n_subsets=1):
        """Device tensors (torch, float32, contiguous, same device)."""
        n = int(z_u.numel())
        self._check(self.lib.strip_set_events_device(
            self._ctx, z_u.data_ptr(), z_d.data_ptr(), dl.data_ptr(), n,
            int(n_subsets)))
        self.n_events = n
        self.n_subsets = int(n_subsets)

    @property
    def responses(self):
        raise AttributeError("responses live on the device; keep the host copy")

    @responses.setter
    def responses(self, triples):
        t = np.ascontiguousarray(triples, dtype=np.float32).reshape(-1, 3)
        self._check(self.lib.strip_set_responses(self._ctx, _fp(t), t.shape[0],
                                                 self.n_subsets))
        self.n_events = t.shape[0]

    # -- image ------------------------------------------------------------
    @property
    def rho(self):
        out = np.empty((self.scanner.n_y_pixels, self.scanner.n_z_pixels), np.float32)
        self._check(self.lib.strip_get_image(self._ctx, _fp(out)))
        return out

    @rho.setter
    def rho(self, image):
        img = np.ascontiguousarray(image, dtype=np.float32).reshape(
            self.scanner.n_y_pixels, self.scanner.n_z_pixels)
        self._check(self.lib.strip_set_image(self._ctx, _fp(img)))

    def sensitivity(self, five_point=False):
        out = np.empty((self.scanner.n_y_pixels, self.scanner.n_z_pixels), np.float32)
        self._check(self.lib.strip_get_sensitivity(self._ctx, int(bool(five_point)), _fp(out)))
        return out

    # -- reconstruction ---------------------------------------------------
    def __call__(self, progress=None, n_iterations=1, n_iterations_so_far=0,
                 n_subsets=None, mode=None):
        """Reconstruction::operator() (reconstruction.h:109-154)."""
        if n_subsets is None:
            n_subsets = self.n_subsets
        if mode is None:
            mode = self.mode
        if progress is None:
            cb = _lib.PROGRESS_CB()
        else:
            def _cb(completed, finished, _user):
                r = progress(completed, bool(finished))
                return 1 if r is True else 0
            cb = _lib.PROGRESS_CB(_cb)
        self._check(self.lib.strip_iterate(self._ctx, int(n_iterations), int(mode),
                                           int(n_subsets), int(n_iterations_so_far),
                                           cb, None))
        self.n_subsets = int(n_subsets)

    iterate = __call__

    # -- schedule -----------------------------------------------------------
    def autotune(self, mode=None):
        """Times the tile-kernel schedules on this context's events and keeps
        the fastest (strip_autotune); returns {'tile', 'grab', 'ms'}."""
        t = _lib.Tuning()
        self._check(self.lib.strip_autotune(self._ctx, self.mode if mode is None else mode,
                                            ctypes.byref(t)))
        self.n_subsets = 1
        return {"tile": t.tile, "grab": t.grab, "ms": t.ms}

    def set_schedule(self, tile=32, grab=32):
        self._check(self.lib.strip_set_schedule(self._ctx, int(tile), int(grab)))

    def load_responses_file(self, path, first=0, n=-1, n_subsets=1):
        """Reads a binary event file (raw f32 triples z_u z_d dl) straight to
        the device and bins the events (strip_load_responses_file); returns
        the number of events read."""
        got = ctypes.c_int64()
        self._check(self.lib.strip_load_responses_file(
            self._ctx, os.fsencode(os.fspath(path)), int(first), int(n), int(n_subsets),
            ctypes.byref(got)))
        self.n_events = got.value
        self.n_subsets = int(n_subsets)
        return got.value

    def set_item_events(self, max_events=0):
        """Largest tile work item in events (1..8000), or 0 to let each
        binning choose (strip_set_item_events)."""
        self._check(self.lib.strip_set_item_events(self._ctx, int(max_events)))

    # -- split iteration (events sharded over processes) -------------------
    def set_accumulator(self, acc):
        """Makes ``acc`` (a float64 CUDA tensor of n_y * n_z values on this
        context's device) the backprojection accumulator and zero-fills it;
        None returns to the context's own buffer."""
        if acc is None:
            self._check(self.lib.strip_set_accumulator(self._ctx, None))
            self._acc = None
            return
        if (acc.dtype.itemsize != 8 or not acc.is_cuda or not acc.is_contiguous()
                or acc.numel() != self.scanner.total_n_pixels):
            raise StripError(_lib.STRIP_E_INVALID,
                             "accumulator must be a contiguous float64 CUDA tensor "
                             "of n_y * n_z values")
        self._check(self.lib.strip_set_accumulator(self._ctx, acc.data_ptr()))
        self._acc = acc  # keeps the buffer alive while the context uses it

    def accumulate(self, subset=0, n_subsets=1, mode=None):
        """acc_j += sum over the subset's events of P_ej / D_e (no update)."""
        mode = self.mode if mode is None else mode
        self._check(self.lib.strip_accumulate(self._ctx, int(mode), int(n_subsets),
                                              int(subset)))
        self.n_subsets = int(n_subsets)

    def update(self, scale=1.0):
        """rho_j <- rho_j * acc_j * scale; acc_j <- 0."""
        self._check(self.lib.strip_update(self._ctx, float(scale)))

    # -- projections ------------------------------------------------------
    def forward(self, rho, sigma_z=None, sigma_dl=None, mode=None):
        sz = self.scanner.sigma_z if sigma_z is None else float(sigma_z)
        sdl = self.scanner.sigma_dl if sigma_dl is None else float(sigma_dl)
        img = np.ascontiguousarray(rho, dtype=np.float32)
        y = np.empty(self.n_events, np.float64)
        self._check(self.lib.strip_forward(self._ctx, _fp(img), sz, sdl,
                                           self.mode if mode is None else mode, _dp(y)))
        return y

    def adjoint(self, w, sigma_z=None, sigma_dl=None, mode=None):
        sz = self.scanner.sigma_z if sigma_z is None else float(sigma_z)
        sdl = self.scanner.sigma_dl if sigma_dl is None else float(sigma_dl)
        wv = np.ascontiguousarray(w, dtype=np.float64)
        g = np.empty((self.scanner.n_y_pixels, self.scanner.n_z_pixels), np.float64)
        self._check(self.lib.strip_adjoint(self._ctx, _dp(wv), sz, sdl,
                                           self.mode if mode is None else mode, _dp(g)))
        return g

    def grad_sigma(self, rho, w, sigma_z=None, sigma_dl=None):
        sz = self.scanner.sigma_z if sigma_z is None else float(sigma_z)
        sdl = self.scanner.sigma_dl if sigma_dl is None else float(sigma_dl)
        img = np.ascontiguousarray(rho, dtype=np.float32)
        wv = np.ascontiguousarray(w, dtype=np.float64)
        gz = ctypes.c_double()
        gd = ctypes.c_double()
        self._check(self.lib.strip_grad_sigma(self._ctx, _fp(img), _dp(wv), sz, sdl,
                                              ctypes.byref(gz), ctypes.byref(gd)))
        return gz.value, gd.value

    # -- parity -----------------------------------------------------------
    def pixel_sets(self, z_u, z_d, dl):
        z_u = np.ascontiguousarray(z_u, dtype=np.float32)
        z_d = np.ascontiguousarray(z_d, dtype=np.float32)
        dl = np.ascontiguousarray(dl, dtype=np.float32)
        n = z_u.shape[0]
        nbb = np.empty(n, np.int32)
        nin = np.empty(n, np.int32)
        dig = np.empty(n, np.uint64)
        P = ctypes.POINTER
        self._check(self.lib.strip_debug_pixel_sets(
            self._ctx, _fp(z_u), _fp(z_d), _fp(dl), n,
            nbb.ctypes.data_as(P(ctypes.c_int32)),
            nin.ctypes.data_as(P(ctypes.c_int32)),
            dig.ctypes.data_as(P(ctypes.c_uint64))))
        return nbb, nin, dig


class Batch:
    """Several Reconstructions (each with its own geometry, events and
    image) advanced together: per MLEM step, a tile launch of its own for
    every member with at least two work items per SM (on side streams), one
    persistent tile launch over the others' items and one update launch,
    replayed from a CUDA graph (strip_batch_*).
    Re-create the batch after set_events on a member."""

    def __init__(self, reconstructions, mode=MODE_CPU):
        self.lib = _lib.load()
        self.members = list(reconstructions)
        arr = (ctypes.c_void_p * len(self.members))(*[r._ctx.value for r in self.members])
        h = ctypes.c_void_p()
        rc = self.lib.strip_batch_create(arr, len(self.members), int(mode), ctypes.byref(h))
        if rc != STRIP_OK:
            msgs = []
            for r in self.members:
                buf = ctypes.create_string_buffer(512)
                self.lib.strip_last_error(r._ctx, buf, 512)
                if buf.value:
                    msgs.append(buf.value.decode(errors="replace"))
            raise StripError(rc, "; ".join(msgs) or "strip_batch_create")
        self._h = h
        for r in self.members:
            r.n_subsets = 1

    def _check(self, rc):
        if rc != STRIP_OK:
            buf = ctypes.create_string_buffer(512)
            self.lib.strip_batch_last_error(self._h, buf, 512)
            raise StripError(rc, buf.value.decode(errors="replace"))

    def __call__(self, n_iterations=1):
        self._check(self.lib.strip_batch_iterate(self._h, int(n_iterations)))

    iterate = __call__

    def stats(self):
        ms = ctypes.c_double()
        ne = ctypes.c_int64()
        items = ctypes.c_int32()
        launches = ctypes.c_int32()
        self._check(self.lib.strip_batch_stats(self._h, ctypes.byref(ms), ctypes.byref(ne),
                                               ctypes.byref(items), ctypes.byref(launches)))
        return {"last_iterate_ms": ms.value, "n_events": ne.value,
                "n_work_items": items.value, "launches_per_iteration": launches.value}

    def close(self):
        if getattr(self, "_h", None):
            self.lib.strip_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def generate_events(scanner, ellipses, n, seed=1):
    """Seeded synthetic events (strip_generate_events); returns z_u, z_d, dl.

    ``ellipses``: iterable of (z, y, a, b, angle_deg, activity), the
    reference's phantom-file ellipse fields, first on top.
    """
    lib = _lib.load()
    el = list(ellipses)
    arr = (_lib.Ellipse * len(el))(*[_lib.Ellipse(*map(float, e)) for e in el])
    zu = np.empty(n, np.float32)
    zd = np.empty(n, np.float32)
    dl = np.empty(n, np.float32)
    g = scanner.geometry()
    rc = lib.strip_generate_events(ctypes.byref(g), arr, len(el), int(seed), int(n),
                                   _fp(zu), _fp(zd), _fp(dl))
    if rc != STRIP_OK:
        raise StripError(rc, "strip_generate_events")
    return zu, zd, dl


def generate_events_device(scanner, ellipses, n, seed=1, device=0):
    """generate_events on the GPU (strip_generate_events_device): returns
    three float32 CUDA tensors on ``device`` holding the same events."""
    import torch
    lib = _lib.load()
    el = list(ellipses)
    arr = (_lib.Ellipse * len(el))(*[_lib.Ellipse(*map(float, e)) for e in el])
    out = [torch.empty(int(n), dtype=torch.float32, device=f"cuda:{device}")
           for _ in range(3)]
    g = scanner.geometry()
    with torch.cuda.device(device):
        torch.cuda.current_stream().synchronize()
        rc = lib.strip_generate_events_device(ctypes.byref(g), arr, len(el), int(seed),
                                              int(n), *(t.data_ptr() for t in out))
    if rc != STRIP_OK:
        raise StripError(rc, "strip_generate_events_device")
    return tuple(out)


def generate_events_image_device(scanner, rho, n, seed=1, uniform_angle=False, device=0):
    """generate_events_image on the GPU (strip_generate_events_image_device)."""
    import torch
    lib = _lib.load()
    img = np.ascontiguousarray(rho, dtype=np.float32)
    if img.size != scanner.n_y_pixels * scanner.n_z_pixels:
        raise ValueError("rho must hold n_y_pixels * n_z_pixels values")
    out = [torch.empty(int(n), dtype=torch.float32, device=f"cuda:{device}")
           for _ in range(3)]
    g = scanner.geometry()
    with torch.cuda.device(device):
        torch.cuda.current_stream().synchronize()
        rc = lib.strip_generate_events_image_device(
            ctypes.byref(g), _fp(img), int(seed), int(n), int(bool(uniform_angle)),
            *(t.data_ptr() for t in out))
    if rc != STRIP_OK:
        raise StripError(rc, "strip_generate_events_image_device")
    return tuple(out)


def generate_events_image(scanner, rho, n, seed=1, uniform_angle=False):
    """Seeded synthetic events emitted from an activity image
    (strip_generate_events_image); returns z_u, z_d, dl.  ``uniform_angle``
    draws the emission angle uniformly (the strip kernel's model) instead of
    tan(theta) uniformly over the acceptance."""
    lib = _lib.load()
    img = np.ascontiguousarray(rho, dtype=np.float32)
    if img.size != scanner.n_y_pixels * scanner.n_z_pixels:
        raise ValueError("rho must hold n_y_pixels * n_z_pixels values")
    zu = np.empty(n, np.float32)
    zd = np.empty(n, np.float32)
    dl = np.empty(n, np.float32)
    g = scanner.geometry()
    rc = lib.strip_generate_events_image(ctypes.byref(g), _fp(img), int(seed), int(n),
                                         int(bool(uniform_angle)), _fp(zu), _fp(zd), _fp(dl))
    if rc != STRIP_OK:
        raise StripError(rc, "strip_generate_events_image")
    return zu, zd, dl


def run(scanner, responses, rho, n_blocks, n_iterations_in_block, output=None,
        progress=None, device=0, device_name=None, mode=MODE_GPU):
    """GPU::Reconstruction::run (cuda/reconstruction.cu:32-113): runs
    n_blocks x n_iterations_in_block iterations, calls output(-1, sensitivity)
    first, output(i + 1, rho) after iterations 1-5, 10, 15, 20, 30, 50, 100 of
    the first block and output((block + 1) * n, rho) after each block; rho is
    updated in place."""
    with Reconstruction(scanner, device=device, mode=mode) as rec:
        if device_name is not None:
            device_name(rec.device_name)
        if output is not None:
            output(-1, rec.sensitivity(five_point=True))
        t = np.ascontiguousarray(responses, dtype=np.float32).reshape(-1, 3)
        rec.set_events(t[:, 0], t[:, 1], t[:, 2])
        rec.rho = rho
        for block in range(n_blocks):
            for i in range(n_iterations_in_block):
                it = block * n_iterations_in_block + i
                rec(progress, 1, it)
                if (output is not None and block == 0 and i < n_iterations_in_block - 1
                        and (i < 5 or i in (9, 14, 19, 29, 49, 99))):
                    output(i + 1, rec.rho)
            if output is not None:
                output((block + 1) * n_iterations_in_block, rec.rho)
        rho[...] = rec.rho.reshape(rho.shape)
        if progress is not None:
            progress(n_blocks * n_iterations_in_block, False)
    return rho

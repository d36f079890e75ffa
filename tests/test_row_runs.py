"""The closed-form row runs of the device kernels, restated in binary32 numpy,
against the oracle's brute-force pixel sets (every box pixel tested with the
reference's in_ellipse, reconstruction.h:255-264).

The kernels never test every box pixel: per row they take the run ends from
the ellipse's closed form and settle each end with one exact test of the
nearest column (strip_rows.cuh row_run).  These cases check that argument on
the CPU for geometries from coarse pixels up to sigma_z = 20 pixels, all
tan over the acceptance and the tips / empty rows of the boxes; the GPU
parity tests check the CUDA code itself on the same kind of inputs."""
import math

import numpy as np
import pytest

from oracle import oracle as orc

f32 = np.float32


def fma(a, b, c):
    return f32(np.float64(a) * np.float64(b) + np.float64(c))


class Scan:
    """ScannerF as make_scanner() fills it (binary32 where the device uses it)."""

    def __init__(self, R, L, ny, nz, ph, pw, sz, sdl):
        self.R, self.pw, self.ph = f32(R), f32(pw), f32(ph)
        self.n_y, self.n_z = ny, nz
        size_y = f32(ny) * self.ph
        size_z = f32(nz) * self.pw
        self.tl_y = f32(0) + size_y / f32(2)
        self.tl_z = f32(0) - size_z / f32(2)
        self.tl_y_half_h = self.tl_y - self.ph / f32(2)
        self.tl_z_half_w = self.tl_z + self.pw / f32(2)
        self.ipsz = f32(1) / (f32(sz) * f32(sz))
        self.ipsdl = f32(1) / (f32(sdl) * f32(sdl))
        self.inv_pw = f32(1) / self.pw
        self.inv2z = f32(0.5) / self.ipsz
        cpw2 = 2.0 * float(self.ipsz) * float(self.pw) ** 2
        self.min_closed_hw = f32(max(0.0, 2e-3 / cpw2 - 0.25))


def event(s, zu, zd, dl):
    """tan, y, z, sec, A, B, C of event_setup (binary32, no contraction)."""
    zu, zd, dl = f32(zu), f32(zd), f32(dl)
    tan = (zu - zd) / (f32(2) * s.R)
    tt = tan * tan
    y = f32(-0.5) * (dl / np.sqrt(f32(1) + tt))
    z = f32(0.5) * ((zu + zd) + (f32(2) * y) * tan)
    sec = np.sqrt(f32(1) + tt)
    A = ((f32(4) * sec) * sec) * s.ipsdl + (f32(2) * tt) * s.ipsz
    B = (f32(-4) * tan) * s.ipsz
    C = f32(2) * s.ipsz
    return tan, y, z, sec, A, B, C


def row_run(s, ev, iy, tlx, brx):
    """strip_rows.cuh row_run: (lo, len) of row iy within [tlx, brx)."""
    tan, y, z, sec, A, B, C = ev
    py = s.tl_y_half_h - f32(iy) * s.ph
    dy = py - y
    Ady2 = (A * dy) * dy
    Bdy = B * dy

    def inside(iz):
        dz = (s.tl_z_half_w + f32(iz) * s.pw) - z
        return (Ady2 + Bdy * dz) + (C * dz) * dz <= f32(9)

    k4 = ((f32(4) * sec) * sec) * s.ipsdl
    x0 = (z - s.tl_z_half_w) * s.inv_pw
    cmin, cmax = tlx, brx - 1
    u = fma(-k4 * dy, dy, f32(9))
    hw = np.sqrt(max(u, f32(0)) * s.inv2z) * s.inv_pw
    xv = fma(tan * dy, s.inv_pw, x0)
    xl, xh = xv - hw, xv + hw
    if hw >= s.min_closed_hw and abs(xv) < 1e7:
        ml, mh = int(np.rint(xl)), int(np.rint(xh))
        lo = ml if inside(ml) else ml + 1
        hi = mh if inside(mh) else mh - 1
        lo, hi = max(lo, cmin), min(hi, cmax)
        return lo, max(hi - lo + 1, 0)
    if not (abs(xl) < 1e8 and abs(xh) < 1e8):
        lo, hi = cmin, cmax
    else:
        xl = min(max(xl, f32(cmin - 2)), f32(cmax + 2))
        xh = min(max(xh, f32(cmin - 2)), f32(cmax + 2))
        lo = max(int(math.ceil(xl)) - 1, cmin)
        hi = min(int(math.floor(xh)) + 1, cmax)
    while lo <= hi and not inside(lo):
        lo += 1
    while hi >= lo and not inside(hi):
        hi -= 1
    if lo <= hi:
        while lo > cmin and inside(lo - 1):
            lo -= 1
        while hi < cmax and inside(hi + 1):
            hi += 1
    return lo, max(hi - lo + 1, 0)


# (R, L, n_y, n_z, pixel, sigma_z, sigma_dl, events): sigma_z from 2 to 20 pixels
GEOMETRIES = [
    (400.0, 800.0, 400, 800, 1.0, 5.0, 25.0, 1500),   # the 800 x 400 benchmark geometry
    (200.0, 500.0, 200, 250, 2.0, 10.0, 42.0, 1500),  # the 250 x 200 geometry
    (150.0, 300.0, 100, 100, 3.0, 12.0, 50.0, 1000),
    (80.0, 240.0, 40, 60, 4.0, 8.0, 30.0, 1000),
    (100.0, 200.0, 400, 400, 0.5, 10.0, 30.0, 250),   # sigma_z = 20 pixels
    (100.0, 200.0, 200, 200, 1.0, 3.0, 9.0, 1500),    # narrow kernel, tilted ellipses
]


@pytest.mark.parametrize("geom", GEOMETRIES, ids=lambda g: f"p{g[4]}_sz{g[5]}")
def test_closed_form_runs_equal_brute_force_sets(geom):
    import stripmlem as sm
    R, L, ny, nz, p, sz, sdl, n = geom
    sc = sm.Scanner(R, L, ny, nz, p, p, sz, sdl)
    g = orc.geometry(R, L, ny, nz, p, p, sz, sdl)
    size_z, size_y = nz * p, ny * p
    phantom = [(0.0, 0.0, 0.45 * size_z, 0.45 * size_y, 0.0, 1.0),
               (0.25 * size_z, 0.2 * size_y, 0.1 * size_z, 0.1 * size_y, 30.0, 2.0)]
    zu, zd, dl = sm.generate_events(sc, phantom, n, seed=17)
    s = Scan(R, L, ny, nz, p, p, sz, sdl)
    rows_checked = narrow = 0
    for i in range(len(zu)):
        box = orc.event_box(g, float(zu[i]), float(zd[i]), float(dl[i]))
        tlx, tly, brx, bry = int(box[2]), int(box[3]), int(box[4]), int(box[5])
        ref = orc.pixel_set(g, float(zu[i]), float(zd[i]), float(dl[i]))
        cols = {}
        for q in ref:
            cols.setdefault(int(q) // nz, []).append(int(q) % nz)
        ev = event(s, zu[i], zd[i], dl[i])
        for iy in range(tly, bry):
            lo, ln = row_run(s, ev, iy, tlx, brx)
            narrow += ln <= 2
            want = sorted(cols.get(iy, []))
            got = list(range(lo, lo + ln))
            assert got == want, (i, iy, got[:3], want[:3], len(got), len(want))
            rows_checked += 1
    assert rows_checked > 10 * len(zu)
    assert narrow > len(zu) // 4  # tips and empty box rows are among the cases
    assert float(s.min_closed_hw) < 0.5  # the closed form settles nearly every row


def test_min_closed_half_width_grows_for_wide_kernels():
    assert float(Scan(400, 800, 400, 800, 1, 1, 5, 25).min_closed_hw) == 0.0
    assert float(Scan(100, 200, 400, 400, 0.5, 0.5, 10, 30).min_closed_hw) > 0.0
    assert float(Scan(100, 200, 400, 400, 0.1, 0.1, 10, 30).min_closed_hw) > 4.0

"""The FP64 oracle's sigma gradient against central differences of its own
forward projection, and the quadrature grid of the sigma fit.  CPU only."""
import numpy as np

from conftest import C1, C1_PHANTOM
from oracle import oracle as orc


def c1_case(n=3000):
    import stripmlem as sm
    sc = sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                    C1["s_z"], C1["s_dl"])
    g = orc.geometry(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                     C1["s_z"], C1["s_dl"])
    ev = sm.generate_events(sc, C1_PHANTOM, n, seed=31)
    rng = np.random.default_rng(6)
    rho = rng.lognormal(0.0, 0.5, size=(g.n_y_pixels, g.n_z_pixels))
    w = rng.uniform(0.5, 1.5, size=n)
    return sc, g, ev, rho, w


def test_grad_sigma_matches_central_differences():
    _, g, (zu, zd, dl), rho, w = c1_case()
    sz, sdl = 9.0, 40.0
    gz, gdl = orc.grad_sigma_f64(g, zu, zd, dl, rho, w, sz, sdl)

    def f(a, b):
        return float(np.dot(w, orc.forward_f64(g, zu, zd, dl, rho, a, b)))
    hz, hd = 1e-4 * sz, 1e-4 * sdl
    fz = (f(sz + hz, sdl) - f(sz - hz, sdl)) / (2 * hz)
    fd = (f(sz, sdl + hd) - f(sz, sdl - hd)) / (2 * hd)
    assert abs(gz - fz) <= 1e-6 * abs(fz)
    assert abs(gdl - fd) <= 1e-6 * abs(fd)


def test_quadrature_grid_covers_the_event_box():
    import stripmlem as sm
    from stripmlem.autograd import quadrature_events
    sc = sm.Scanner(100.0, 200.0, 100, 100, 2.0, 2.0, 15.0, 60.0)
    zu, zd, dl, vol = quadrature_events(sc, 4.0, 8.0)
    assert zu.min() > -100 and zu.max() < 100 and zd.min() > -100 and zd.max() < 100
    nd = len(np.unique(dl))
    assert len(zu) == 50 * 50 * nd
    dmax = 2 * 100 * np.sqrt(2.0) + 6 * 60
    assert dl.max() >= dmax - 8 and -dl.min() >= dmax - 8
    assert vol == 4.0 * 4.0 * 8.0

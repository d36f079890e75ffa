"""Differentiable projection on the GPU: the sigma-gradient kernel, the
device-buffer projections and the torch.autograd.Function, against the FP64
oracle, against central differences, and in a sigma fit."""
import numpy as np
import pytest

from conftest import C1, C1_PHANTOM
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    import stripmlem as sm
    sc = sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                    C1["s_z"], C1["s_dl"])
    g = orc.geometry(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                     C1["s_z"], C1["s_dl"])
    n = 30_000
    ev = sm.generate_events(sc, C1_PHANTOM, n, seed=32)
    rng = np.random.default_rng(7)
    rho = rng.lognormal(0.0, 0.5, size=(g.n_y_pixels, g.n_z_pixels)).astype(np.float32)
    # weights that make d(w'y)/dsigma large: the kernel integrates to nearly
    # the same total at every sigma, so uniform weights would leave only a
    # small residual (and a cancellation-dominated test); w ~ y weighs the
    # kernel cores, whose height falls as sigma grows
    y0 = orc.forward_f64(g, *ev, rho, C1["s_z"], C1["s_dl"])
    w = y0 / y0.mean() * rng.uniform(0.9, 1.1, size=n)
    return sc, g, ev, rho, w


def test_grad_sigma_vs_fp64(case):
    import stripmlem as sm
    sc, g, ev, rho, w = case
    with sm.Reconstruction(sc) as rec:
        rec.set_events(*ev)
        for sz, sdl in ((10.0, 42.0), (9.0, 40.0), (6.0, 30.0)):
            gz, gdl = rec.grad_sigma(rho, w, sz, sdl)
            oz, odl = orc.grad_sigma_f64(g, *ev, rho.astype(np.float64), w, sz, sdl)
            assert abs(gz - oz) <= REL_TOL * abs(oz), (sz, sdl, gz, oz)
            assert abs(gdl - odl) <= REL_TOL * abs(odl), (sz, sdl, gdl, odl)


def test_grad_sigma_vs_central_differences_of_the_kernels(case):
    import stripmlem as sm
    sc, g, ev, rho, w = case
    sz, sdl = 9.0, 40.0
    with sm.Reconstruction(sc) as rec:
        rec.set_events(*ev)
        gz, gdl = rec.grad_sigma(rho, w, sz, sdl)

        def f(a, b):
            return float(np.dot(w, rec.forward(rho, a, b, mode=0)))
        # binary32 forward values carry ~1e-7 relative noise (ex2.approx,
        # rounding), so the step is 1 % of sigma and the bar 0.5 %; the FP64
        # oracle's gradient meets its own differences to 1e-6
        # (tests/test_oracle_grad.py)
        hz, hd = 1e-2 * sz, 1e-2 * sdl
        fz = (f(sz + hz, sdl) - f(sz - hz, sdl)) / (2 * hz)
        fd = (f(sz, sdl + hd) - f(sz, sdl - hd)) / (2 * hd)
    assert abs(gz - fz) <= 5e-3 * abs(fz)
    assert abs(gdl - fd) <= 5e-3 * abs(fd)


@pytest.mark.parametrize("mode", [0, 1])
def test_autograd_function_vs_fp64(case, mode):
    import torch
    import stripmlem as sm
    from stripmlem.autograd import project
    sc, g, ev, rho, w = case
    with sm.Reconstruction(sc, mode=mode) as rec:
        rec.set_events(*ev)
        r = torch.tensor(rho, device="cuda:0", requires_grad=True)
        s = torch.tensor([9.0, 40.0], dtype=torch.float64, requires_grad=(mode == 0))
        y = project(rec, r, s)
        loss = (torch.tensor(w, device="cuda:0") * y).sum()
        loss.backward()
        yo = orc.forward_f64(g, *ev, rho, 9.0, 40.0, mode=mode)
        assert rel(y.detach().cpu().numpy(), yo) < REL_TOL
        go = orc.adjoint_f64(g, *ev, w, 9.0, 40.0, mode=mode)
        assert rel(r.grad.cpu().numpy(), go) < REL_TOL
        if mode == 0:
            oz, odl = orc.grad_sigma_f64(g, *ev, rho.astype(np.float64), w, 9.0, 40.0)
            assert rel(s.grad.numpy(), [oz, odl]) < REL_TOL
        # the device entry points agree with the host ones
        assert rel(y.detach().cpu().numpy(), rec.forward(rho, 9.0, 40.0)) < 1e-12


def test_sigma_gradient_refused_for_analytic_kernel(case):
    import torch
    import stripmlem as sm
    from stripmlem.autograd import project
    sc, g, ev, rho, w = case
    with sm.Reconstruction(sc, mode=1) as rec:
        rec.set_events(*(a[:1000] for a in ev))
        r = torch.tensor(rho, device="cuda:0")
        s = torch.tensor([9.0, 40.0], dtype=torch.float64, requires_grad=True)
        y = project(rec, r, s)
        with pytest.raises(sm.StripError):
            y.sum().backward()


def test_sigma_fit_recovers_the_model_sigmas():
    """Self-consistent fit: the data density is the model's own at
    (8, 30) mm (quadrature events weighted by v_c * y_c(8, 30)), so the
    extended likelihood peaks at (8, 30) exactly; Adam on log sigma from
    (15, 60) must get there."""
    import torch
    import stripmlem as sm
    from stripmlem import autograd as sa
    n = 100
    rng = np.random.default_rng(4)
    rho = np.exp(0.5 * rng.standard_normal((n, n))).astype(np.float32)
    model = sm.Scanner(100.0, 200.0, n, n, 2.0, 2.0, 15.0, 60.0)
    rho_t = torch.from_numpy(rho).cuda()
    qu, qd, ql, vol = sa.quadrature_events(model, 3.0, 6.0)
    with sm.Reconstruction(model) as rq:
        rq.set_events(qu, qd, ql)
        with torch.no_grad():
            yq = sa.project(rq, rho_t, torch.tensor([8.0, 30.0], dtype=torch.float64), 0)
        s, hist = sa.fit_sigma(rq, rq, vol, rho_t, (15.0, 60.0), weights=vol * yq)
    assert abs(float(s[0]) - 8.0) < 0.04 and abs(float(s[1]) - 30.0) < 0.15, hist[-5:]


@pytest.mark.parametrize("uniform_angle,expected", [(True, (10.90, 31.77)),
                                                    (False, (9.22, 32.00))])
def test_sigma_fit_on_simulated_events_lands_where_the_kernel_is_best(uniform_angle,
                                                                       expected):
    """The fit on physically simulated events: 1e7 events emitted from a
    log-normal (sigma 0.5) activity image on the 400 x 400 1 mm geometry
    (R 200 mm, L 400 mm), detected on their exact hits and smeared with
    sigma_z = 8 mm, sigma_dl = 30 mm; L-BFGS on the extended likelihood from
    (15, 60) mm.  It does not return (8, 30): the reference's GaussianKernel
    is not a normalised density of the smeared events -- its integral over
    the detected event space drifts with sigma (test_oracle_kernel_norm.py:
    -0.8 % for sigmas 25 % larger at the centre pixel) -- so the likelihood
    peaks where the kernel approximates the events best.  Pinned: the landing
    point for uniform emission angles (the kernel's own angular model) and
    for tan(theta) uniform over the acceptance."""
    import torch
    import stripmlem as sm
    from stripmlem import autograd as sa
    n = 400
    rng = np.random.default_rng(4)
    rho = np.exp(0.5 * rng.standard_normal((n, n))).astype(np.float32)
    model = sm.Scanner(200.0, 400.0, n, n, 1.0, 1.0, 15.0, 60.0)
    truth = sm.Scanner(200.0, 400.0, n, n, 1.0, 1.0, 8.0, 30.0)
    ev = sm.generate_events_image_device(truth, rho, 10_000_000, seed=7,
                                         uniform_angle=uniform_angle)
    qu, qd, ql, vol = sa.quadrature_events(model, 3.0, 6.0)
    with sm.Reconstruction(model) as rd, sm.Reconstruction(model) as rq:
        rd.set_events_device(*ev)
        rq.set_events(qu, qd, ql)
        s, hist = sa.fit_sigma(rd, rq, vol, torch.from_numpy(rho).cuda(), (15.0, 60.0))
    assert abs(float(s[0]) - expected[0]) < 0.15, hist[-3:]
    assert abs(float(s[1]) - expected[1]) < 0.3, hist[-3:]
    # far from the simulated sigmas: the bias is the model's, not the optimiser's
    assert abs(float(s[0]) - 8.0) > 1.0

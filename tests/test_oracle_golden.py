"""The oracle against the reference's own unit-test golden values for the
strip path (src/2d/strip/*_test.cpp).  CPU only."""
import math

import numpy as np
import pytest

from oracle import oracle as orc


def approx(a, b, eps):
    # Catch v1 Approx: |a - b| < eps * (1 + max(|a|, |b|))
    return abs(a - b) < eps * (1.0 + max(abs(a), abs(b)))


# gaussian_kernel_test.cpp:11-50 -- GaussianKernel<float>(0.01, 0.04), R = 0.35
@pytest.mark.parametrize("angle,y,dz,dy,ref", [
    (math.pi / 6, 0.1, 0.0, 0.0, 184.304974530866),
    (math.pi / 6, 0.1, 0.05, 0.1, 5.272096361578383e-6),
    (math.pi / 6, 0.1, -0.05, -0.05, 0.0338473429952690),
    (math.pi / 4, -0.3, 0.0, 0.0, 95.87658397191050),
    (math.pi / 4, -0.3, 0.05, 0.1, 0.0),
    (math.pi / 4, -0.3, -0.05, -0.05, 0.1719727908599724),
])
def test_gaussian_kernel_golden(angle, y, dz, dy, ref):
    L = orc.lib()
    a = np.float32(angle)
    sec = np.float32(1.0) / np.float32(math.cos(a))
    tan = np.float32(math.tan(a))
    v = L.orc_gaussian_kernel_f32(0.01, 0.04, y, tan, sec, 0.35, dz, dy)
    assert approx(v, ref, 1e-6), (v, ref)
    v64 = L.orc_gaussian_kernel_f64(0.01, 0.04, y, math.tan(angle),
                                    1 / math.cos(angle), 0.35, dz, dy)
    assert approx(v64, ref, 1e-6), (v64, ref)


# kernel_test.cpp:31-49 -- Scanner<double, short>::sensitivity
@pytest.mark.parametrize("R,L,pt,ref", [
    (500, 1000, (0, 0), 0.5),
    (500, 1000, (50, 0), 0.46652458328685176),
    (500, 1000, (-50, 100), 0.4410019151324715),
    (500, 1000, (-450, -200), 0.07526632771111386),
    (450, 200, (0, 0), 0.1392089745461279),
    (450, 200, (50, 0), 0.07044657495455454),
    (450, 200, (-50, 100), 0.07402517367717103),
    (450, 200, (-70, -200), 0.05269621503719814),
])
def test_sensitivity_golden(R, L, pt, ref):
    g = orc.geometry(R, L, 200, 200, 5, 5, 10, 63)
    v = orc.lib().orc_sensitivity_f64(g, pt[0], pt[1])
    assert approx(v, ref, 1e-13), (v, ref)


# kernel_test.cpp:81-113 -- bb_y / bb_z for sigma_z 10, sigma_dl 63
@pytest.mark.parametrize("angle,bby,bbz", [
    (0.0470448, 94.3954, 21.6737),
    (-0.594145, 78.3053, 56.9959),
    (0.20029, 92.6108, 28.3458),
    (-0.571667, 79.4745, 55.3539),
    (-0.420542, 86.266, 44.0276),
])
def test_bbox_golden(angle, bby, bbz):
    ipdl = 1.0 / (63.0 * 63.0)
    ipz = 1.0 / (10.0 * 10.0)
    A = (4.0 / (math.cos(angle) ** 2)) * ipdl + 2.0 * math.tan(angle) ** 2 * ipz
    B = -4.0 * math.tan(angle) * ipz
    C = 2.0 * ipz
    B_2 = (B / 2.0) ** 2
    L = orc.lib()
    assert approx(L.orc_bb_y_f64(A, C, B_2), bby, 1e-4)
    assert approx(L.orc_bb_z_f64(A, C, B_2), bbz, 1e-4)


# scanner_test.cpp:15-37 -- pixel_at incl. boundaries (truncation toward zero)
@pytest.mark.parametrize("pt,px", [
    ((0.0, 0.0), (100, 100)),
    ((-0.00001, 0.00001), (99, 99)),
    ((-500.0, 500.0), (0, 0)),
    ((500.0, 500.0), (200, 0)),
    ((-500.0, -500.0), (0, 200)),
    ((500.0, -500.0), (200, 200)),
    ((-499.99999, 499.99999), (0, 0)),
    ((499.99999, 499.99999), (199, 0)),
    ((-499.99999, -499.99999), (0, 199)),
    ((499.99999, -499.99999), (199, 199)),
])
def test_pixel_at_golden(pt, px):
    g = orc.geometry(500, 1000, 200, 200, 5, 5, 10, 63)
    out = np.zeros(2, np.int32)
    orc.lib().orc_pixel_at_f64(g, pt[0], pt[1], orc._ip(out))
    assert tuple(out) == px


# scanner_test.cpp:39-66 -- pixel_center and reversibility
def test_pixel_center_golden():
    L = orc.lib()
    # Scanner(100, 200, 200, 200, 10, 63): pixel size 2R/n_y = 1, L/n_z = 1
    g = orc.geometry(100, 200, 200, 200, 1, 1, 10, 63)
    pt = np.zeros(2)
    for px, ref in [((100, 100), (0.5, -0.5)), ((99, 99), (-0.5, 0.5)),
                    ((0, 0), (-99.5, 99.5))]:
        L.orc_pixel_center_f64(g, px[0], px[1], orc._dp(pt))
        assert tuple(pt) == ref
        back = np.zeros(2, np.int32)
        L.orc_pixel_at_f64(g, pt[0], pt[1], orc._ip(back))
        assert tuple(back) == px
    g = orc.geometry(500, 1000, 200, 200, 5, 5, 10, 63)
    for p, ref in [((0.0, 0.0), (2.5, -2.5)), ((-6.0, 3.0), (-7.5, 2.5)),
                   ((6.0, 3.0), (7.5, 2.5)), ((-6.0, -3.0), (-7.5, -2.5)),
                   ((6.0, -3.0), (7.5, -2.5))]:
        px = np.zeros(2, np.int32)
        L.orc_pixel_at_f64(g, p[0], p[1], orc._ip(px))
        L.orc_pixel_center_f64(g, int(px[0]), int(px[1]), orc._dp(pt))
        assert tuple(pt) == ref


# response_test.cpp:11-55 -- image <-> projection space at 1e-13
@pytest.mark.parametrize("y,z,tan,zu,zd,dl", [
    (10.0, 20.0, 0.1227845609029046, 74.02520679727803, -36.480898015336116,
     -20.15019650917697),
    (-10.0, 37.0, -0.08748866352592401, -3.244785221925042, 75.49501195140655,
     20.076396750866948),
])
def test_projection_conversions_golden(y, z, tan, zu, zd, dl):
    L = orc.lib()
    assert approx(math.tan(math.radians(7.0 if y > 0 else -5.0)), tan, 1e-13)
    out = np.zeros(3)
    L.orc_to_projection_tan_f64(450.0, y, z, tan, orc._dp(out))
    assert approx(out[0], zu, 1e-13) and approx(out[1], zd, 1e-13)
    assert approx(out[2], dl, 1e-13)
    back = np.zeros(3)
    L.orc_from_projection_tan_f64(450.0, out[0], out[1], out[2], orc._dp(back))
    assert approx(back[1], y, 1e-13) and approx(back[2], z, 1e-13)

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "j-pet-mlem-old_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from stripmlem import _lib
    return _lib.load()


# Scanner of the small parity configuration: C1 geometry (two 500 mm strips at
# y = +-200 mm, 250 x 200 pixels of 2 mm, sigma_z 10 mm, sigma_dl 42 mm).
C1 = dict(radius=200.0, length=500.0, n_y=200, n_z=250, p=2.0, s_z=10.0, s_dl=42.0)
# C1 phantom: hot and cold ellipses listed before the body so that, with the
# reference's exclusive overlaps (first on top), each keeps its own activity.
C1_PHANTOM = [(40, 30, 30, 20, 0, 3.0), (-50, -20, 25, 40, 0, 0.3), (0, 0, 150, 100, 0, 1.0)]
# C2 geometry: 800 mm strips at y = +-400 mm, 800 x 400 pixels of 1 mm.
C2 = dict(radius=400.0, length=800.0, n_y=400, n_z=800, p=1.0, s_z=5.0, s_dl=25.0)
C2_PHANTOM = [
    (-150, 60, 40, 25, 20, 2.0),
    (150, -60, 50, 30, -30, 0.1),
    (0, 100, 60, 20, 0, 1.5),
    (0, -110, 70, 25, 10, 0.5),
    (-250, -40, 30, 30, 0, 1.8),
    (250, 50, 35, 20, 45, 0.3),
    (80, 40, 20, 15, 0, 2.0),
    (-80, -60, 25, 15, -15, 0.8),
    (0, 0, 300, 150, 0, 1.0),
    (0, 0, 360, 175, 0, 0.2),
]

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running")


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


class GoldenScene:
    """A scene rebuilt from a golden fixture (inputs exactly as the reference read them)."""

    def __init__(self, g):
        self.nx, self.ny, self.nz = [int(v) for v in g["shape"]]
        self.dx = float(g["dx"])
        self.dt = float(g["dt"])
        self.tol = float(g["tol"])
        self.g = g
        self.solid_phi = g["solid"] if int(g["has_solid"]) else None
        self.solid_active = g["solid_active"] if int(g["has_solid"]) else None
        self.fluid_active = g["fluid_active"]
        self.velocity_active = [g["u_in_active"], g["v_in_active"], g["w_in_active"]]
        self.solid_velocity = [g["us"], g["vs"], g["ws"]]

    def fluid_effective(self):
        return self.g["fluid"].astype(np.float32)

    def solid_effective(self):
        return self.g["solid"].astype(np.float32)

    def velocity_effective(self):
        return [self.g["u_in"].astype(np.float32), self.g["v_in"].astype(np.float32), self.g["w_in"].astype(np.float32)]

    def solid_velocity_effective(self):
        return [a.astype(np.float32) for a in self.solid_velocity]


@pytest.fixture(params=golden_names() if os.path.isdir(GOLDEN) else [])
def golden(request):
    return request.param, load_golden(request.param)

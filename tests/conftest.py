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


def golden_names(prefix: str = ""):
    """Fixtures of plain projections, or (prefix "term_") of projections with
    one optional term on, or (prefix "ext_") of the velocity extension after a
    projection, or (prefix "splat_") of the FLIP splat before one."""
    names = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    if prefix:
        return [n for n in names if n.startswith(prefix)]
    return [n for n in names if not n.startswith(("term_", "ext_", "splat_"))]


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


@pytest.fixture(params=golden_names("term_") if os.path.isdir(GOLDEN) else [])
def golden_term(request):
    return request.param, load_golden(request.param)


@pytest.fixture(params=golden_names("ext_") if os.path.isdir(GOLDEN) else [])
def golden_ext(request):
    return request.param, load_golden(request.param)


@pytest.fixture(params=golden_names("splat_") if os.path.isdir(GOLDEN) else [])
def golden_splat(request):
    return request.param, load_golden(request.param)


def splat_particles(g):
    """The particle records of a splat_ fixture as a structured array."""
    from shiokaze_b200.scenes import PARTICLE_DTYPE
    return np.ascontiguousarray(g["particles"]).view(PARTICLE_DTYPE).reshape(-1)


def term_options(g):
    """Keyword options of oracle.project / the B200 solver for a term_ fixture."""
    opt = {}
    if float(g["kappa"]):
        opt["kappa"] = float(g["kappa"])
    if "density_u" in g:
        opt["density"] = [g["density_u"], g["density_v"], g["density_w"]]
    if float(g["volume"][1]):
        opt["volume"] = (float(g["volume"][0]), float(g["volume"][1]), 0.0, float(g["gain"]))
    if int(g["warm_start"]):
        opt["warm_start"] = True
    opt["tile"] = int(g["tile"])
    opt["repeat"] = int(g["repeat"])
    return opt

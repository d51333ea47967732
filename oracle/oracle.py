"""ctypes front end of the C restatement in ``shkz_oracle.c``.

TEST INFRASTRUCTURE ONLY: the product never imports this module. Tests, the
smoke check and the benchmark's CPU-baseline leg use it as the checker.

``project(scene)`` reproduces ``macpressuresolver3::project``
(src/projection/macpressuresolver3.cpp:54-299) on the CPU: face fractions,
labelling, assembly into a row-sorted CSR, PCG (identity as shipped, or
MIC(0) applied), pressure scatter and velocity update.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess
import time
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libshkz_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "shkz_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.shkzo_get_area.restype = ctypes.c_double
        L.shkzo_get_area.argtypes = [P]
        L.shkzo_fraction.restype = ctypes.c_double
        L.shkzo_fraction.argtypes = [ctypes.c_double, ctypes.c_double]
        L.shkzo_fractions.argtypes = [ctypes.c_int] * 3 + [P, P, P, P, ctypes.c_double, ctypes.c_double,
                                                          ctypes.c_int, ctypes.c_int, P, P, P]
        L.shkzo_label.restype = ctypes.c_longlong
        L.shkzo_label.argtypes = [ctypes.c_int] * 4 + [P, P, P, P]
        L.shkzo_assemble.restype = ctypes.c_longlong
        L.shkzo_assemble.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_double, P, P, P, P, P, P,
                                                          ctypes.c_longlong, P, P, P, P]
        L.shkzo_spmv.argtypes = [ctypes.c_longlong, P, P, P, P, P]
        L.shkzo_mic0_apply.argtypes = [ctypes.c_longlong, P, P, P, ctypes.c_double, ctypes.c_double, P, P, P]
        L.shkzo_pcg.restype = ctypes.c_int
        L.shkzo_pcg.argtypes = [ctypes.c_longlong, P, P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, P]
        L.shkzo_update_velocity.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_double, P, P, P, P, P, P,
                                                                P]
        L.shkzo_splat.restype = ctypes.c_int
        L.shkzo_splat.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_longlong, P] + \
            [ctypes.c_int] * 7 + [P] * 5
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _ptr3(arrs):
    t = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])
    return t


@dataclasses.dataclass
class System:
    index: np.ndarray      # (nz,ny,nx) int64, -1 where no unknown
    n: int
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    rhs: np.ndarray

    def matrix(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.data, self.indices, self.indptr), shape=(self.n, self.n))


@dataclasses.dataclass
class OracleResult:
    area: list
    rho: list
    system: System
    x: np.ndarray
    iterations: int
    reresid: float
    pressure: np.ndarray
    pressure_active: np.ndarray
    velocity: list
    velocity_active: list
    solve_s: float
    total_s: float
    volume_rhs_correct: float = 0.0
    y_prev: Optional[float] = None
    warm_prev: Optional[np.ndarray] = None


def _opt3(arrs):
    return _ptr3(arrs) if arrs is not None else None


def fractions(scene, eps_solid=1e-2, eps_fluid=1e-2, second_order_fluid=True, second_order_solid=True,
              density=None):
    """Face solid areas and liquid fractions; ``density`` (three face arrays)
    applies set_solid_density (macpressuresolver3.cpp:75-80)."""
    nx, ny, nz = scene.nx, scene.ny, scene.nz
    solid = np.ascontiguousarray(scene.solid_effective(), np.float32)
    sact = (np.ascontiguousarray(scene.solid_active, np.uint8) if scene.solid_active is not None
            else np.zeros(solid.shape, np.uint8))
    fluid = np.ascontiguousarray(scene.fluid_effective(), np.float32)
    fact = np.ascontiguousarray(scene.fluid_active, np.uint8)
    fshapes = [(nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)]
    area = [np.zeros(s, np.float32) for s in fshapes]
    rho = [np.zeros(s, np.float32) for s in fshapes]
    dens = [np.ascontiguousarray(d, np.float32) for d in density] if density is not None else None
    lib().shkzo_fractions(nx, ny, nz, _p(solid), _p(sact), _p(fluid), _p(fact), eps_solid, eps_fluid,
                          int(second_order_fluid), int(second_order_solid), _ptr3(area), _ptr3(rho), _opt3(dens))
    return area, rho


def surface_tension(scene, rho, kappa: float, vel: list, vact: list) -> None:
    """Velocity += surface tension force, in place (macpressuresolver3.cpp:98-128):
    curvature = 7-point Laplacian of the liquid level set with clamped
    neighbours (six neighbours summed in FP32 as the float operands are, then
    FP64), and on active faces with 0 < rho < 1
    u += float(-sgn*dt/(dx*rho)*kappa*(theta*c_i + (1-theta)*c_{i-1}))."""
    fl = np.ascontiguousarray(scene.fluid_effective(), np.float32)
    dx, dt = float(scene.dx), float(scene.dt)
    pad = np.pad(fl, 1, mode="edge")
    s6 = pad[1:-1, 1:-1, :-2] + pad[1:-1, 1:-1, 2:]
    s6 = s6 + pad[1:-1, :-2, 1:-1]
    s6 = s6 + pad[1:-1, 2:, 1:-1]
    s6 = s6 + pad[:-2, 1:-1, 1:-1]
    s6 = s6 + pad[2:, 1:-1, 1:-1]
    curv = ((s6.astype(np.float64) - 6.0 * fl.astype(np.float64)) / (dx * dx)).astype(np.float32)
    nz, ny, nx = fl.shape
    for d in range(3):
        fz, fy, fx = vel[d].shape
        kk, jj, ii = np.meshgrid(np.arange(fz), np.arange(fy), np.arange(fx), indexing="ij")
        c1 = (np.minimum(kk, nz - 1), np.minimum(jj, ny - 1), np.minimum(ii, nx - 1))
        c0 = (np.clip(kk - (d == 2), 0, nz - 1), np.clip(jj - (d == 1), 0, ny - 1), np.clip(ii - (d == 0), 0, nx - 1))
        r = rho[d].astype(np.float64)
        m = vact[d].astype(bool) & (r != 0.0) & (r < 1.0)
        sgn = np.where(fl[c1] < 0.0, -1.0, 1.0)
        theta = np.where(sgn < 0, 1.0 - r, r)
        face_c = theta * curv[c1].astype(np.float64) + (1.0 - theta) * curv[c0].astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            inc = (-sgn * dt / (dx * r) * kappa * face_c).astype(np.float32)
        vel[d][m] = vel[d][m] + inc[m]


def assemble(scene, area, rho, tile=8, vel=None, rhs_add: float = 0.0):
    """Label (indices in the reference's tile-major order for tile edge
    ``tile``) and assemble; ``vel`` overrides the scene's face velocities and
    ``rhs_add`` is the volume correction added to every row."""
    nx, ny, nz = scene.nx, scene.ny, scene.nz
    fluid = np.ascontiguousarray(scene.fluid_effective(), np.float32)
    index = np.empty((nz, ny, nx), np.int64)
    n = lib().shkzo_label(nx, ny, nz, tile, _p(fluid), _ptr3(area), _ptr3(rho), _p(index))
    vel = [np.ascontiguousarray(v, np.float32) for v in (vel if vel is not None else scene.velocity_effective())]
    svel = [np.ascontiguousarray(v, np.float32) for v in scene.solid_velocity_effective()]
    indptr = np.zeros(n + 1, np.int64)
    indices = np.zeros(max(1, 7 * n), np.int64)
    data = np.zeros(max(1, 7 * n), np.float64)
    rhs = np.zeros(max(1, n), np.float64)
    nnz = lib().shkzo_assemble(nx, ny, nz, scene.dx, scene.dt, _p(fluid), _ptr3(area), _ptr3(rho), _ptr3(vel),
                               _ptr3(svel), _p(index), n, _p(indptr), _p(indices), _p(data), _p(rhs))
    rhs = rhs[:n].copy()
    if rhs_add:
        rhs += rhs_add
    return System(index=index, n=int(n), indptr=indptr, indices=indices[:nnz].copy(), data=data[:nnz].copy(),
                  rhs=rhs)


def pcg(system: System, tol: float, max_iterations: int = 30000, mic0: bool = True,
        omega: float = 0.97, min_ratio: float = 0.25):
    n = system.n
    x = np.zeros(max(1, n), np.float64)
    rr = ctypes.c_double(0.0)
    it = lib().shkzo_pcg(n, _p(system.indptr), _p(system.indices), _p(system.data), _p(system.rhs), _p(x),
                         tol, max_iterations, int(mic0), omega, min_ratio, ctypes.byref(rr))
    return x[:n], int(it), float(rr.value)


def mic0_apply(system: System, r: np.ndarray, omega=0.97, min_ratio=0.25):
    z = np.zeros(max(1, system.n), np.float64)
    inv = np.zeros(max(1, system.n), np.float64)
    r = np.ascontiguousarray(r, np.float64)
    lib().shkzo_mic0_apply(system.n, _p(system.indptr), _p(system.indices), _p(system.data), omega, min_ratio,
                           _p(r), _p(z), _p(inv))
    return z[:system.n], inv[:system.n]


def spmv(system: System, x: np.ndarray) -> np.ndarray:
    y = np.zeros(max(1, system.n), np.float64)
    x = np.ascontiguousarray(x, np.float64)
    lib().shkzo_spmv(system.n, _p(system.indptr), _p(system.indices), _p(system.data), _p(x), _p(y))
    return y[:system.n]


def volume_correction(n: int, dt: float, current: float, target: float, y_prev: float, gain: float = 1.0):
    """(rhs correction, new y_prev) of the PI volume controller
    (macpressuresolver3.cpp:219-234); (0, y_prev) when it does not run."""
    if not (n and gain and target):
        return 0.0, y_prev
    x = (current - target) / target
    y = y_prev + x * dt
    kp = gain * 2.3 / (25.0 * 0.01)
    ki = kp * kp / 16.0
    return -(kp * x + ki * y) / (x + 1.0), y


def project(scene, tol: Optional[float] = None, mic0: bool = True, tile: int = 8,
            max_iterations: int = 30000, eps_solid=1e-2, eps_fluid=1e-2, surface_tension_kappa: float = 0.0,
            density=None, volume=None, warm_prev=None, warm_start: bool = False) -> OracleResult:
    """macpressuresolver3::project on the CPU. Optional terms: surface tension
    coefficient, per-face solid density, volume = (current, target, y_prev,
    gain), and warm start from ``warm_prev`` (the previous solution by unknown
    number, numbered with tile edge ``tile``)."""
    t0 = time.perf_counter()
    nx, ny, nz = scene.nx, scene.ny, scene.nz
    area, rho = fractions(scene, eps_solid, eps_fluid, density=density)
    vel = [np.ascontiguousarray(v, np.float32).copy() for v in scene.velocity_effective()]
    vact = [np.ascontiguousarray(m, np.uint8).copy() for m in scene.velocity_active]
    if surface_tension_kappa:
        surface_tension(scene, rho, surface_tension_kappa, vel, vact)
    system = assemble(scene, area, rho, tile, vel=vel)
    rhs_add, y_prev = 0.0, None
    if volume is not None:
        rhs_add, y_prev = volume_correction(system.n, float(scene.dt), *volume)
        if rhs_add:
            system.rhs += rhs_add
    x0 = None
    if (warm_start or warm_prev is not None) and system.n:
        x0 = np.zeros(system.n)
        if warm_prev is not None:
            m = min(system.n, len(warm_prev))
            x0[:m] = warm_prev[:m]
        system.rhs -= spmv(system, x0)
    t1 = time.perf_counter()
    x, it, rr = pcg(system, scene.tol if tol is None else tol, max_iterations, mic0)
    if x0 is not None:
        x = x + x0
    t2 = time.perf_counter()
    pressure = np.zeros((nz, ny, nx), np.float32)
    mask = system.index >= 0
    pressure[mask] = x[system.index[mask]].astype(np.float32)
    svel = [np.ascontiguousarray(v, np.float32) for v in scene.solid_velocity_effective()]
    dens = [np.ascontiguousarray(d, np.float32) for d in density] if density is not None else None
    if system.n:
        lib().shkzo_update_velocity(nx, ny, nz, scene.dx, scene.dt, _p(pressure), _ptr3(area), _ptr3(rho),
                                    _ptr3(svel), _ptr3(vel), _ptr3(vact), _opt3(dens))
    t3 = time.perf_counter()
    return OracleResult(area=area, rho=rho, system=system, x=x, iterations=it, reresid=rr, pressure=pressure,
                        pressure_active=mask.astype(np.uint8), velocity=vel, velocity_active=vact,
                        solve_s=t2 - t1, total_s=t3 - t0, volume_rhs_correct=rhs_add, y_prev=y_prev,
                        warm_prev=x.copy() if x0 is not None else None)


def splat(nx: int, ny: int, nz: int, dx: float, particles: np.ndarray, velocity: list, velocity_active: list,
          apic: bool = True, splat_bullet: bool = False):
    """FLIP splat and combined grid velocity (``shkzo_splat``) on particle
    records in the reference's layout (``shiokaze_b200.scenes.PARTICLE_DTYPE``).
    Returns (velocity, velocity_active, mass, momentum, splat_active), lists of
    three face grids; the inputs are not modified."""
    P = np.ascontiguousarray(particles)
    dt = P.dtype
    vel = [np.ascontiguousarray(v, np.float32).copy() for v in velocity]
    act = [np.ascontiguousarray(a, np.uint8).copy() for a in velocity_active]
    mass = [np.zeros_like(v) for v in vel]
    mom = [np.zeros_like(v) for v in vel]
    sact = [np.zeros_like(a) for a in act]
    off = lambda k: dt.fields[k][1]
    rc = lib().shkzo_splat(nx, ny, nz, dx, len(P), _p(P), dt.itemsize, off("p"), off("velocity"), off("mass"),
                           off("c") if apic else -1, off("bullet"), int(splat_bullet),
                           _ptr3(vel), _ptr3(act), _ptr3(mass), _ptr3(mom), _ptr3(sact))
    if rc:
        raise MemoryError("shkzo_splat")
    return vel, act, mass, mom, sact

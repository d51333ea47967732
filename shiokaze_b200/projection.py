"""Host-side mirror of Shiokaze's ``macproject3_interface`` for the B200 solver.

``MacPressureSolver3`` has the reference module's API and meaning
(include/shiokaze/projection/macproject3_interface.h:42-113,
src/projection/macpressuresolver3.cpp):

* ``configure(config)`` reads the same keys (``Residual``, ``MaxIterations``,
  ``ModifiedIC``, ``MinDiagRatio``, ``EpsFluid``, ``EpsSolid``,
  ``SecondOrderAccurateFluid``, ``SecondOrderAccurateSolid``) plus ``B200.*``
  keys for the device solver;
* ``initialize(shape, dx)`` as the private initialize the module receives;
* ``project(dt, velocity, solid, solid_velocity, fluid, surface_tension)``
  updates the face velocities (values and active bits) in place and keeps
  the pressure;
* ``set_target_volume(current, target)`` and ``set_solid_density(density)``
  as the interface's setters; ``Gain``, ``WarmStart`` and ``TileSize`` (the
  grids' tile edge, which numbers the warm-start vector) are read like the
  reference module reads them;
* ``serialize()`` / ``initialize_from(state)`` carry the fields the module
  serialises (macpressuresolver3.cpp:320-342);
* ``get_pressure()`` returns the pressure grid.

Grids are ``Grid`` (``array3``: values as the reference reads them plus active
bits) and ``MacGrid`` (``macarray3``: three face grids). Every call goes
through the C ABI (``include/shkz_b200.h``) to the CUDA library; there is no
CPU path.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import numpy as np

from . import native


@dataclasses.dataclass
class Grid:
    """Stand-in for ``array3<float>``: values (as read) and active bits, shape (nz,ny,nx)."""
    values: np.ndarray
    active: np.ndarray

    @staticmethod
    def zeros(shape_zyx):
        return Grid(np.zeros(shape_zyx, np.float32), np.zeros(shape_zyx, np.uint8))


@dataclasses.dataclass
class MacGrid:
    """Stand-in for ``macarray3<float>``: face grids for x, y, z."""
    values: list
    active: list


def _c(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, ctypes.c_void_p(a.ctypes.data)


class MacPressureSolver3:
    LONG_NAME = "MAC Pressure Solver 3D (B200)"
    ARGUMENT_NAME = "Projection"

    def __init__(self, config: Optional[dict] = None):
        self.cfg = native.default_config()
        self.shape = None
        self.dx = None
        self.pressure: Optional[Grid] = None
        self.last_result: Optional[dict] = None
        self._ctx: Optional[native.Context] = None
        self.solid_density: Optional[list] = None
        self._volume = [0.0, 0.0, 0.0]  # target, current, y_prev
        if config:
            self.configure(config)

    # -- module hooks --------------------------------------------------
    def configure(self, config: dict) -> None:
        c = self.cfg
        g = config.get
        c.residual = float(g("Residual", c.residual))
        c.max_iterations = int(g("MaxIterations", c.max_iterations))
        c.mic_omega = float(g("ModifiedIC", c.mic_omega))
        c.mic_min_diag_ratio = float(g("MinDiagRatio", c.mic_min_diag_ratio))
        c.eps_fluid = float(g("EpsFluid", c.eps_fluid))
        c.eps_solid = float(g("EpsSolid", c.eps_solid))
        c.second_order_fluid = int(bool(g("SecondOrderAccurateFluid", c.second_order_fluid)))
        c.second_order_solid = int(bool(g("SecondOrderAccurateSolid", c.second_order_solid)))
        pre = g("B200.Preconditioner", None)
        if pre is not None:
            c.preconditioner = {"none": native.PRECOND_NONE, "mic0": native.PRECOND_MIC0,
                                "learned": native.PRECOND_LEARNED}.get(str(pre).lower(), int(pre) if str(pre).isdigit() else c.preconditioner)
        c.refine = int(bool(g("B200.Refine", c.refine)))
        c.fp64_reference = int(bool(g("B200.FP64Reference", c.fp64_reference)))
        c.fp64_tol = float(g("B200.FP64Tolerance", c.fp64_tol))
        c.check_interval = int(g("B200.CheckInterval", c.check_interval))
        c.stall_window = int(g("B200.StallWindow", c.stall_window))
        c.device = int(g("B200.Device", c.device))
        c.mic_block = int(g("B200.MICBlock", c.mic_block))
        c.gain = float(g("Gain", c.gain))
        c.warm_start = int(bool(g("WarmStart", c.warm_start)))
        c.index_tile = int(g("TileSize", c.index_tile))
        c.spin_limit = int(g("B200.SpinLimit", c.spin_limit))
        c.fault_skip_publish = int(g("B200.FaultSkipPublish", c.fault_skip_publish))
        c.device_mem_limit_mb = int(g("B200.DeviceMemoryLimitMB", c.device_mem_limit_mb))
        if self._ctx is not None:
            self._ctx.set_config(c)

    def initialize(self, shape, dx: float) -> None:
        self.shape = tuple(int(s) for s in shape)
        self.dx = float(dx)
        self.post_initialize()

    def post_initialize(self) -> None:
        nx, ny, nz = self.shape
        self.pressure = Grid.zeros((nz, ny, nx))
        self._volume = [0.0, 0.0, 0.0]
        if self._ctx is not None:
            self._push_volume()

    def set_target_volume(self, current_volume: float, target_volume: float) -> None:
        if self._ctx is not None:
            self._pull_volume()  # keep the controller state (y_prev) the projections advanced
        self._volume[0] = float(target_volume)
        self._volume[1] = float(current_volume)
        self._push_volume()

    def set_solid_density(self, density) -> None:
        """Per-face solid density: a MacGrid, three face arrays, or None."""
        if density is None:
            self.solid_density = None
            return
        vals = density.values if isinstance(density, MacGrid) else density
        self.solid_density = [np.ascontiguousarray(v, np.float32) for v in vals]

    def _push_volume(self) -> None:
        st = (ctypes.c_double * 3)(*self._volume)
        self.context.check(native.load().shkz_b200_set_volume_state(self.context.handle, st), "set_volume_state")

    def _pull_volume(self) -> None:
        st = (ctypes.c_double * 3)()
        self.context.check(native.load().shkz_b200_get_volume_state(self.context.handle, st), "get_volume_state")
        self._volume = list(st)

    def warm_start_vector(self) -> np.ndarray:
        """The previous solution by unknown number (m_prev_pressure)."""
        L = native.load()
        n = L.shkz_b200_warm_start_size(self.context.handle)
        out = np.zeros(max(0, n), np.float64)
        self.context.check(L.shkz_b200_get_warm_start(self.context.handle, out.ctypes.data, out.size),
                           "get_warm_start")
        return out

    def set_warm_start_vector(self, prev: np.ndarray) -> None:
        prev = np.ascontiguousarray(prev, np.float64)
        self.context.check(native.load().shkz_b200_set_warm_start(self.context.handle, prev.ctypes.data, prev.size),
                           "set_warm_start")

    def serialize(self) -> dict:
        """shape, dx, target/current volume, y_prev and (with WarmStart) the
        previous solution, as macpressuresolver3::serialize writes them."""
        self._pull_volume()
        st = {"shape": self.shape, "dx": self.dx, "target_volume": self._volume[0],
              "current_volume": self._volume[1], "y_prev": self._volume[2]}
        if self.cfg.warm_start:
            st["prev_pressure"] = self.warm_start_vector()
        return st

    def initialize_from(self, st: dict) -> None:
        self.shape = tuple(st["shape"])
        self.dx = float(st["dx"])
        nx, ny, nz = self.shape
        self.pressure = Grid.zeros((nz, ny, nx))
        self._volume = [float(st["target_volume"]), float(st["current_volume"]), float(st["y_prev"])]
        self._push_volume()
        if self.cfg.warm_start and "prev_pressure" in st:
            self.set_warm_start_vector(st["prev_pressure"])

    @property
    def context(self) -> native.Context:
        if self._ctx is None:
            self._ctx = native.Context(self.cfg)
            self._push_volume()
        return self._ctx

    # -- macproject3_interface ------------------------------------------
    def project(self, dt: float, velocity: MacGrid, solid: Optional[Grid], solid_velocity: Optional[MacGrid],
                fluid: Grid, surface_tension: float = 0.0, rigidbodies=None) -> dict:
        if self.shape is None:
            raise RuntimeError("initialize(shape, dx) must be called before project()")
        nx, ny, nz = self.shape
        args = native.ProjectArgs()
        args.nx, args.ny, args.nz = nx, ny, nz
        args.dx, args.dt = self.dx, float(dt)
        keep = []
        f, args.fluid = _c(fluid.values, np.float32); keep.append(f)
        fa, args.fluid_active = _c(fluid.active, np.uint8); keep.append(fa)
        if solid is not None:
            s, args.solid = _c(solid.values, np.float32); keep.append(s)
            sa, args.solid_active = _c(solid.active, np.uint8); keep.append(sa)
        vel, vact = [], []
        for d in range(3):
            v = np.ascontiguousarray(velocity.values[d], np.float32)
            m = np.ascontiguousarray(velocity.active[d], np.uint8)
            vel.append(v); vact.append(m)
            args.velocity[d] = v.ctypes.data
            args.velocity_active[d] = m.ctypes.data
            if solid_velocity is not None:
                sv, p = _c(solid_velocity.values[d], np.float32)
                keep.append(sv)
                args.solid_velocity[d] = p.value
        args.surface_tension = float(surface_tension)
        if self.solid_density is not None:
            for d in range(3):
                keep.append(self.solid_density[d])
                args.solid_density[d] = self.solid_density[d].ctypes.data
        pressure = np.zeros((nz, ny, nx), np.float32)
        pact = np.zeros((nz, ny, nx), np.uint8)
        args.pressure = pressure.ctypes.data
        args.pressure_active = pact.ctypes.data
        res = native.Result()
        rc = native.load().shkz_b200_project_host(self.context.handle, ctypes.byref(args), ctypes.byref(res))
        if rc not in (0, -4, -5):
            self.context.check(rc, "shkz_b200_project_host")
        for d in range(3):
            velocity.values[d] = vel[d]
            velocity.active[d] = vact[d]
        self.pressure = Grid(pressure, pact)
        self.last_result = res.as_dict()
        return self.last_result

    def get_pressure(self) -> Grid:
        return self.pressure

    # -- inspection of the last system (tests) ---------------------------
    def inspect(self, what: int) -> np.ndarray:
        nx, ny, nz = self.shape
        dtype = np.float64 if what >= 5 else np.float32
        out = np.zeros((nz, ny, nx), dtype)
        rc = native.load().shkz_b200_inspect(self.context.handle, what, out.ctypes.data, out.nbytes)
        self.context.check(rc, "shkz_b200_inspect")
        return out

    def apply_preconditioner(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float32)
        z = np.zeros_like(r)
        rc = native.load().shkz_b200_apply_preconditioner(self.context.handle, r.ctypes.data, z.ctypes.data)
        self.context.check(rc, "shkz_b200_apply_preconditioner")
        return z

    # -- learned preconditioner ------------------------------------------
    def learned_init(self, seed: int = 0) -> None:
        self.context.check(native.load().shkz_b200_learned_init(self.context.handle, seed), "learned_init")

    def learned_params(self, gradients: bool = False) -> np.ndarray:
        L = native.load()
        n = L.shkz_b200_learned_param_count(self.context.handle)
        out = np.zeros(n, np.float32)
        self.context.check(L.shkz_b200_learned_get_params(self.context.handle, out.ctypes.data, n, int(gradients)),
                           "learned_get_params")
        return out

    def learned_set_params(self, blob: np.ndarray) -> None:
        blob = np.ascontiguousarray(blob, np.float32)
        self.context.check(native.load().shkz_b200_learned_set_params(self.context.handle, blob.ctypes.data, blob.size),
                           "learned_set_params")

    def learned_apply(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float32)
        z = np.zeros_like(r)
        self.context.check(native.load().shkz_b200_learned_apply(self.context.handle, r.ctypes.data, z.ctypes.data),
                           "learned_apply")
        return z

    def learned_dims(self):
        d = (ctypes.c_int * 3)()
        self.context.check(native.load().shkz_b200_learned_dims(self.context.handle, d), "learned_dims")
        return tuple(d)

    TENSORS = ["X0", "A1", "S1", "P1", "A2", "S2", "P2", "A3", "B3", "C2", "D2", "C1", "D1", "Z"]

    def learned_tensor(self, which, grad: bool = False) -> np.ndarray:
        """Stored activation of the last network application (name or index);
        "Z" is the raw output; grad=True gives the gradient w.r.t. the tensor."""
        if isinstance(which, str):
            which = self.TENSORS.index(which)
        if grad:
            which += 14
        L = native.load()
        shp = (ctypes.c_int * 4)()
        self.context.check(L.shkz_b200_learned_tensor(self.context.handle, which, None, 0, shp), "learned_tensor")
        out = np.zeros(tuple(shp), np.float32)
        self.context.check(L.shkz_b200_learned_tensor(self.context.handle, which, out.ctypes.data, out.size, shp),
                           "learned_tensor")
        return out[..., 0] if which == 13 else out

    def learned_backward(self, gZ: np.ndarray) -> np.ndarray:
        gZ = np.ascontiguousarray(gZ, np.float32)
        self.context.check(native.load().shkz_b200_learned_backward(self.context.handle, gZ.ctypes.data, gZ.size),
                           "learned_backward")
        return self.learned_params(gradients=True)

    def learned_train(self, steps: int, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(1, steps), np.float64)
        self.context.check(native.load().shkz_b200_learned_train(self.context.handle, steps, lr, seed,
                                                                 losses.ctypes.data), "learned_train")
        return losses[:steps]

    def learned_save(self, path: str) -> None:
        self.context.check(native.load().shkz_b200_learned_save(self.context.handle, path.encode()), "learned_save")

    def learned_load(self, path: str) -> None:
        self.context.check(native.load().shkz_b200_learned_load(self.context.handle, path.encode()), "learned_load")

    def apply_matrix(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros_like(x)
        rc = native.load().shkz_b200_apply_matrix(self.context.handle, x.ctypes.data, y.ctypes.data)
        self.context.check(rc, "shkz_b200_apply_matrix")
        return y


def grids_from_scene(scene):
    """(velocity, solid, solid_velocity, fluid) grids of a ``scenes.Scene``."""
    fluid = Grid(scene.fluid_effective(), np.ascontiguousarray(scene.fluid_active, np.uint8))
    solid = None
    if scene.solid_phi is not None:
        solid = Grid(scene.solid_effective(), np.ascontiguousarray(scene.solid_active, np.uint8))
    velocity = MacGrid([v.copy() for v in scene.velocity_effective()],
                       [np.ascontiguousarray(m, np.uint8).copy() for m in scene.velocity_active])
    solid_velocity = None
    if scene.solid_velocity is not None:
        solid_velocity = MacGrid(scene.solid_velocity_effective(),
                                 [np.ones_like(m) for m in scene.velocity_active])
    return velocity, solid, solid_velocity, fluid

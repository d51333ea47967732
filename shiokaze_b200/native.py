"""ctypes binding of the C ABI in ``include/shkz_b200.h``.

Loads the in-tree ``libshkz_b200.so``; importing this module on a machine
without the built library or without a CUDA device raises instead of falling
back to anything else.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libshkz_b200.so")

PRECOND_NONE = 0
PRECOND_MIC0 = 1
PRECOND_LEARNED = 2

ERRORS = {
    0: "ok", -1: "invalid argument", -2: "CUDA runtime error", -3: "device allocation failed",
    -4: "a bounded device wait gave up", -5: "NaN in the system or the iterates",
    -6: "no usable sm_100 device", -7: "invalid call order", -8: "size beyond a documented limit",
}


class Config(ctypes.Structure):
    _fields_ = [
        ("residual", ctypes.c_double),
        ("max_iterations", ctypes.c_int),
        ("preconditioner", ctypes.c_int),
        ("mic_omega", ctypes.c_double),
        ("mic_min_diag_ratio", ctypes.c_double),
        ("eps_fluid", ctypes.c_double),
        ("eps_solid", ctypes.c_double),
        ("second_order_fluid", ctypes.c_int),
        ("second_order_solid", ctypes.c_int),
        ("refine", ctypes.c_int),
        ("fp64_reference", ctypes.c_int),
        ("fp64_tol", ctypes.c_double),
        ("check_interval", ctypes.c_int),
        ("stall_window", ctypes.c_int),
        ("device", ctypes.c_int),
        ("mic_block", ctypes.c_int),
        ("gain", ctypes.c_double),
        ("warm_start", ctypes.c_int),
        ("index_tile", ctypes.c_int),
        ("spin_limit", ctypes.c_int),
        ("fault_skip_publish", ctypes.c_int),
        ("device_mem_limit_mb", ctypes.c_int),
        ("csr_preconditioner", ctypes.c_int),
    ]


class ProjectArgs(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dt", ctypes.c_double),
        ("fluid", ctypes.c_void_p), ("fluid_active", ctypes.c_void_p),
        ("solid", ctypes.c_void_p), ("solid_active", ctypes.c_void_p),
        ("velocity", ctypes.c_void_p * 3), ("velocity_active", ctypes.c_void_p * 3),
        ("solid_velocity", ctypes.c_void_p * 3),
        ("pressure", ctypes.c_void_p), ("pressure_active", ctypes.c_void_p),
        ("surface_tension", ctypes.c_double),
        ("solid_density", ctypes.c_void_p * 3),
    ]


class ExtendArgs(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_double),
        ("width", ctypes.c_int), ("constrain", ctypes.c_int),
        ("solid", ctypes.c_void_p), ("solid_active", ctypes.c_void_p),
        ("velocity", ctypes.c_void_p * 3), ("velocity_active", ctypes.c_void_p * 3),
    ]


class SplatArgs(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_double),
        ("count", ctypes.c_longlong), ("particles", ctypes.c_void_p), ("stride", ctypes.c_int),
        ("offset_position", ctypes.c_int), ("offset_velocity", ctypes.c_int), ("offset_mass", ctypes.c_int),
        ("offset_apic", ctypes.c_int), ("offset_bullet", ctypes.c_int), ("splat_bullet", ctypes.c_int),
        ("velocity", ctypes.c_void_p * 3), ("velocity_active", ctypes.c_void_p * 3),
        ("mass", ctypes.c_void_p * 3), ("momentum", ctypes.c_void_p * 3), ("splat_active", ctypes.c_void_p * 3),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("iterations", ctypes.c_int), ("outer_steps", ctypes.c_int),
        ("fallbacks", ctypes.c_int), ("unknowns", ctypes.c_longlong), ("tiles", ctypes.c_longlong),
        ("reresid", ctypes.c_double), ("reresid_l2", ctypes.c_double), ("err_fp64_inf", ctypes.c_double),
        ("fp64_reresid", ctypes.c_double), ("ms_assemble", ctypes.c_double), ("ms_solve", ctypes.c_double),
        ("ms_update", ctypes.c_double), ("ms_total", ctypes.c_double), ("ms_h2d", ctypes.c_double),
        ("ms_d2h", ctypes.c_double), ("kernel_launches", ctypes.c_longlong),
        ("volume_rhs_correct", ctypes.c_double), ("ms_fractions", ctypes.c_double),
        ("ms_labelling", ctypes.c_double), ("ms_build", ctypes.c_double), ("reserved", ctypes.c_double * 3),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


EXPORTS = [
    "shkz_b200_default_config", "shkz_b200_create", "shkz_b200_destroy", "shkz_b200_set_config",
    "shkz_b200_errstr", "shkz_b200_last_error", "shkz_b200_project_host", "shkz_b200_project_device",
    "shkz_b200_stream", "shkz_b200_solve_csr", "shkz_b200_inspect", "shkz_b200_apply_preconditioner",
    "shkz_b200_apply_matrix", "shkz_b200_time_kernel",
    "shkz_b200_learned_init", "shkz_b200_learned_param_count", "shkz_b200_learned_set_params",
    "shkz_b200_learned_get_params", "shkz_b200_learned_apply", "shkz_b200_learned_dims",
    "shkz_b200_learned_tensor", "shkz_b200_learned_backward", "shkz_b200_learned_train",
    "shkz_b200_learned_save", "shkz_b200_learned_load", "shkz_b200_conv3d", "shkz_b200_conv3d_noalloc",
    "shkz_b200_host_alloc", "shkz_b200_host_free",
    "shkz_b200_set_target_volume", "shkz_b200_get_volume_state", "shkz_b200_set_volume_state",
    "shkz_b200_warm_start_size", "shkz_b200_get_warm_start", "shkz_b200_set_warm_start",
    "shkz_b200_learned_flops", "shkz_b200_extend_velocity_host", "shkz_b200_extend_velocity_device",
    "shkz_b200_splat_host", "shkz_b200_splat_device",
]

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises OSError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is not built; run `python -m shiokaze_b200.build`")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    L.shkz_b200_default_config.argtypes = [ctypes.POINTER(Config)]
    L.shkz_b200_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(Config)]
    L.shkz_b200_create.restype = ctypes.c_int
    L.shkz_b200_destroy.argtypes = [P]
    L.shkz_b200_set_config.argtypes = [P, ctypes.POINTER(Config)]
    L.shkz_b200_errstr.argtypes = [ctypes.c_int]
    L.shkz_b200_errstr.restype = ctypes.c_char_p
    L.shkz_b200_last_error.argtypes = [P]
    L.shkz_b200_last_error.restype = ctypes.c_char_p
    L.shkz_b200_project_host.argtypes = [P, ctypes.POINTER(ProjectArgs), ctypes.POINTER(Result)]
    L.shkz_b200_project_device.argtypes = [P, ctypes.POINTER(ProjectArgs), ctypes.POINTER(Result)]
    L.shkz_b200_extend_velocity_host.argtypes = [P, ctypes.POINTER(ExtendArgs)]
    L.shkz_b200_extend_velocity_device.argtypes = [P, ctypes.POINTER(ExtendArgs)]
    L.shkz_b200_splat_host.argtypes = [P, ctypes.POINTER(SplatArgs)]
    L.shkz_b200_splat_device.argtypes = [P, ctypes.POINTER(SplatArgs)]
    L.shkz_b200_stream.argtypes = [P]
    L.shkz_b200_stream.restype = P
    L.shkz_b200_solve_csr.argtypes = [P, ctypes.c_longlong, P, P, P, P, P, ctypes.POINTER(Result)]
    L.shkz_b200_inspect.argtypes = [P, ctypes.c_int, P, ctypes.c_size_t]
    L.shkz_b200_set_target_volume.argtypes = [P, ctypes.c_double, ctypes.c_double]
    L.shkz_b200_get_volume_state.argtypes = [P, P]
    L.shkz_b200_set_volume_state.argtypes = [P, P]
    L.shkz_b200_learned_flops.argtypes = [P]
    L.shkz_b200_learned_flops.restype = ctypes.c_double
    L.shkz_b200_warm_start_size.argtypes = [P]
    L.shkz_b200_warm_start_size.restype = ctypes.c_longlong
    L.shkz_b200_get_warm_start.argtypes = [P, P, ctypes.c_size_t]
    L.shkz_b200_set_warm_start.argtypes = [P, P, ctypes.c_size_t]
    L.shkz_b200_apply_preconditioner.argtypes = [P, P, P]
    L.shkz_b200_apply_matrix.argtypes = [P, P, P]
    L.shkz_b200_time_kernel.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_longlong)]
    L.shkz_b200_learned_init.argtypes = [P, ctypes.c_uint]
    L.shkz_b200_learned_param_count.argtypes = [P]
    L.shkz_b200_learned_param_count.restype = ctypes.c_longlong
    L.shkz_b200_learned_set_params.argtypes = [P, P, ctypes.c_size_t]
    L.shkz_b200_learned_get_params.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int]
    L.shkz_b200_learned_apply.argtypes = [P, P, P]
    L.shkz_b200_learned_dims.argtypes = [P, P]
    L.shkz_b200_learned_tensor.argtypes = [P, ctypes.c_int, P, ctypes.c_size_t, P]
    L.shkz_b200_learned_backward.argtypes = [P, P, ctypes.c_size_t]
    L.shkz_b200_learned_train.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_uint, P]
    L.shkz_b200_learned_save.argtypes = [P, ctypes.c_char_p]
    L.shkz_b200_learned_load.argtypes = [P, ctypes.c_char_p]
    L.shkz_b200_conv3d.argtypes = [ctypes.c_int] * 7 + [P, P, P, P, ctypes.c_int, P]
    L.shkz_b200_conv3d_noalloc.argtypes = [ctypes.c_int] * 7 + [P, P, P, P, ctypes.c_int, P, P]
    L.shkz_b200_host_alloc.argtypes = [ctypes.c_size_t]
    L.shkz_b200_host_alloc.restype = P
    L.shkz_b200_host_free.argtypes = [P]
    L.shkz_b200_host_free.restype = None
    _lib = L
    return L


def default_config() -> Config:
    c = Config()
    load().shkz_b200_default_config(ctypes.byref(c))
    return c


class ShkzError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code}) {detail}".strip())


class Context:
    """Owns one device context (``shkz_b200_create`` / ``shkz_b200_destroy``)."""

    def __init__(self, config: Config | None = None):
        L = load()
        self.config = config if config is not None else default_config()
        h = ctypes.c_void_p()
        rc = L.shkz_b200_create(ctypes.byref(h), ctypes.byref(self.config))
        if rc != 0:
            raise ShkzError(rc, "shkz_b200_create")
        self.handle = h

    def set_config(self, config: Config):
        self.config = config
        rc = load().shkz_b200_set_config(self.handle, ctypes.byref(config))
        if rc != 0:
            raise ShkzError(rc, "shkz_b200_set_config")

    def close(self):
        if getattr(self, "handle", None):
            load().shkz_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return load().shkz_b200_last_error(self.handle).decode()

    def check(self, rc: int, where: str):
        if rc != 0:
            raise ShkzError(rc, where, self.last_error())

    @property
    def stream(self) -> int:
        return load().shkz_b200_stream(self.handle)


def extend_velocity(ctx: Context, velocity, velocity_active, solid, solid_active, dx: float, width: int,
                    constrain: bool = True):
    """The velocity extension the liquid solver runs right after a projection
    (macliquid3::extend_both, src/liquid/macliquid3.cpp:330-340), on host
    numpy grids through ``shkz_b200_extend_velocity_host``: ``width``
    extrapolation passes, then (``constrain``) constrain_velocity. Face grids
    are [k, j, i] float32 with uint8 masks; solid is the nodal level set (or
    None). Returns new (velocity, velocity_active) lists."""
    import numpy as np
    vel = [np.ascontiguousarray(v, np.float32).copy() for v in velocity]
    act = [np.ascontiguousarray(m, np.uint8).copy() for m in velocity_active]
    nz, ny, nx = vel[0].shape[0], vel[0].shape[1], vel[0].shape[2] - 1
    a = ExtendArgs()
    a.nx, a.ny, a.nz, a.dx, a.width, a.constrain = nx, ny, nz, float(dx), int(width), int(bool(constrain))
    keep = []
    if solid is not None:
        s = np.ascontiguousarray(solid, np.float32)
        sa = np.ascontiguousarray(solid_active, np.uint8)
        keep += [s, sa]
        a.solid, a.solid_active = s.ctypes.data, sa.ctypes.data
    for d in range(3):
        a.velocity[d] = vel[d].ctypes.data
        a.velocity_active[d] = act[d].ctypes.data
    ctx.check(load().shkz_b200_extend_velocity_host(ctx.handle, ctypes.byref(a)), "shkz_b200_extend_velocity_host")
    return vel, act


def splat_args(nx: int, ny: int, nz: int, dx: float, particles, count: int, record_dtype, apic: bool = True,
               splat_bullet: bool = False) -> SplatArgs:
    """shkz_b200_splat_args for particle records of a numpy structured dtype
    with fields p, velocity, mass, c and bullet (the reference's layout is
    ``shiokaze_b200.scenes.PARTICLE_DTYPE``) at address ``particles``; the
    grid pointers are left for the caller."""
    a = SplatArgs()
    a.nx, a.ny, a.nz, a.dx = nx, ny, nz, float(dx)
    a.count, a.particles, a.stride = int(count), particles, record_dtype.itemsize
    off = lambda k: record_dtype.fields[k][1]
    a.offset_position, a.offset_velocity, a.offset_mass = off("p"), off("velocity"), off("mass")
    a.offset_apic = off("c") if apic else -1
    a.offset_bullet = off("bullet") if "bullet" in record_dtype.fields else -1
    a.splat_bullet = int(bool(splat_bullet))
    return a


def splat(ctx: Context, nx: int, ny: int, nz: int, dx: float, particles, velocity, velocity_active,
          apic: bool = True, splat_bullet: bool = False, outputs: bool = True):
    """The FLIP splat and combined grid velocity the FLIP liquid solver runs
    right before a projection (macflipliquid3.cpp:135-151), on host numpy data
    through ``shkz_b200_splat_host``. ``particles`` is a structured array of
    particle records. Returns (velocity, velocity_active, mass, momentum,
    splat_active), lists of three face grids (the last three None without
    ``outputs``)."""
    import numpy as np
    P = np.ascontiguousarray(particles)
    vel = [np.ascontiguousarray(v, np.float32).copy() for v in velocity]
    act = [np.ascontiguousarray(m, np.uint8).copy() for m in velocity_active]
    a = splat_args(nx, ny, nz, dx, P.ctypes.data if len(P) else None, len(P), P.dtype, apic, splat_bullet)
    mass = mom = sact = None
    if outputs:
        mass = [np.zeros_like(v) for v in vel]
        mom = [np.zeros_like(v) for v in vel]
        sact = [np.zeros_like(m) for m in act]
    for d in range(3):
        a.velocity[d], a.velocity_active[d] = vel[d].ctypes.data, act[d].ctypes.data
        if outputs:
            a.mass[d], a.momentum[d], a.splat_active[d] = mass[d].ctypes.data, mom[d].ctypes.data, sact[d].ctypes.data
    ctx.check(load().shkz_b200_splat_host(ctx.handle, ctypes.byref(a)), "shkz_b200_splat_host")
    return vel, act, mass, mom, sact

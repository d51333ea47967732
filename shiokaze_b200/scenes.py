"""Seeded synthetic scenes for the pressure projection.

Each scene produces the inputs of ``macproject3_interface::project``
(include/shiokaze/projection/macproject3_interface.h:84-91): a cell-centred
liquid level set, a nodal solid level set, three face-velocity grids and three
solid face-velocity grids, on an ``nx*ny*nz`` grid with ``dx = 1/nx``.

The narrow-band rules follow ``macutility3::assign_initial_variables``
(src/utility/macutility3.cpp:314-416):

* a liquid cell holds a value (is active) only where ``|phi| < sqrt(3)*dx``;
  the liquid is pushed out of solids with ``phi = max(phi, -(solid+dx))``;
  the grid is then a level set with background ``+sqrt(3)*dx`` and fill
  value ``-sqrt(3)*dx`` (``array3::set_as_levelset``,
  include/shiokaze/array/array3.h:261-266);
* the nodal solid grid is cleared to 1 and holds ``min(1, solid(p))`` only
  inside the same band;
* a face velocity is set only where the liquid level set at the face centre is
  ``<= sqrt(3)*dx`` (``fluid_velocity->set_touch_only_actives`` path).

"Effective" arrays are what the reference's ``array3::operator()`` returns
for every cell: the stored value on active cells, the fill value on inactive
cells inside the level set and the background value elsewhere. Inactive
cells are classified inside/outside by the sign of the analytic level set,
which is what the reference flood fill (src/array/tiledarray3.cpp:214-289)
recovers for a band of this width; the test suite checks this against the
compiled reference.

All grids are numpy arrays of shape ``(nz, ny, nx)`` (x fastest in memory),
float32 values rounded once from float64 so that every consumer sees the same
bits. No public dataset is involved; scenes are procedural from a seed.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import Callable, Optional

import numpy as np

SQRT3 = math.sqrt(3.0)


@dataclasses.dataclass
class Scene:
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    dt: float
    tol: float
    fluid_phi: np.ndarray          # (nz,ny,nx) f32 analytic values (unbanded)
    fluid_active: np.ndarray       # (nz,ny,nx) u8
    solid_phi: Optional[np.ndarray]  # (nz+1,ny+1,nx+1) f32 or None
    solid_active: Optional[np.ndarray]
    velocity: list                 # [u (nz,ny,nx+1), v (nz,ny+1,nx), w (nz+1,ny,nx)] f32
    velocity_active: list          # u8 masks, same shapes
    solid_velocity: Optional[list] = None
    fluid_band: float = 0.0
    solid_band: float = 0.0

    # ------------------------------------------------------------------
    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def fluid_effective(self) -> np.ndarray:
        return effective(self.fluid_phi, self.fluid_active, self.fluid_band)

    def solid_effective(self) -> np.ndarray:
        if self.solid_phi is None:
            return np.ones((self.nz + 1, self.ny + 1, self.nx + 1), np.float32)
        return effective(self.solid_phi, self.solid_active, self.solid_band)

    def velocity_effective(self) -> list:
        return [np.where(m != 0, u, np.float32(0)).astype(np.float32)
                for u, m in zip(self.velocity, self.velocity_active)]

    def solid_velocity_effective(self) -> list:
        if self.solid_velocity is None:
            return [np.zeros_like(u) for u in self.velocity]
        return [u.astype(np.float32) for u in self.solid_velocity]

    # ------------------------------------------------------------------
    def write_reference_input(self, path: str) -> None:
        """Write the dense input file read by the reference harness."""
        with open(path, "wb") as f:
            f.write(b"SHKZIN01")
            f.write(struct.pack("<5i", self.nx, self.ny, self.nz,
                                int(self.solid_phi is not None),
                                int(self.solid_velocity is not None)))
            f.write(struct.pack("<4d", self.dx, self.dt, self.fluid_band, self.solid_band))
            f.write(self.fluid_phi.astype(np.float64).tobytes())
            f.write(self.fluid_active.astype(np.uint8).tobytes())
            if self.solid_phi is not None:
                f.write(self.solid_phi.astype(np.float64).tobytes())
                f.write(self.solid_active.astype(np.uint8).tobytes())
            for u, m in zip(self.velocity, self.velocity_active):
                f.write(u.astype(np.float64).tobytes())
                f.write(m.astype(np.uint8).tobytes())
            if self.solid_velocity is not None:
                for u in self.solid_velocity:
                    f.write(u.astype(np.float64).tobytes())


def effective(phi: np.ndarray, active: np.ndarray, band: float) -> np.ndarray:
    """Value the reference reads at every cell of a banded level set."""
    b = np.float32(band)
    return np.where(active != 0, phi, np.where(phi < 0, -b, b)).astype(np.float32)


# ----------------------------------------------------------------------
# signed distance helpers (float64, numpy broadcasting)

def _grid_coords(n: tuple, dx: float, offset: tuple):
    nx, ny, nz = n
    x = (np.arange(nx, dtype=np.float64) + offset[0]) * dx
    y = (np.arange(ny, dtype=np.float64) + offset[1]) * dx
    z = (np.arange(nz, dtype=np.float64) + offset[2]) * dx
    return x[None, None, :], y[None, :, None], z[:, None, None]


def sdf_box(x, y, z, lo, hi):
    qx = np.maximum(lo[0] - x, x - hi[0])
    qy = np.maximum(lo[1] - y, y - hi[1])
    qz = np.maximum(lo[2] - z, z - hi[2])
    outside = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2 + np.maximum(qz, 0) ** 2)
    inside = np.minimum(np.maximum(np.maximum(qx, qy), qz), 0.0)
    return outside + inside


def sdf_sphere(x, y, z, c, r):
    return np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r


def _union_spheres(phi, coords, spheres, band_cells, dx):
    """phi = min(phi, sphere_k) over spheres, touching only each bounding box."""
    x, y, z = coords
    nz, ny, nx = phi.shape
    for (c, r) in spheres:
        lo = [max(0, int(math.floor((c[d] - r) / dx - band_cells - 2))) for d in range(3)]
        hi = [min(s, int(math.ceil((c[d] + r) / dx + band_cells + 2))) for d, s in enumerate((nx, ny, nz))]
        if lo[0] >= hi[0] or lo[1] >= hi[1] or lo[2] >= hi[2]:
            continue
        sub = sdf_sphere(x[:, :, lo[0]:hi[0]], y[:, lo[1]:hi[1], :], z[lo[2]:hi[2], :, :], c, r)
        view = phi[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        np.minimum(view, sub, out=view)
    return phi


# ----------------------------------------------------------------------

def _finish(name, n, dx, dt, tol, fluid_fn: Callable, solid_fn: Optional[Callable],
            vel_fn: Callable, rng, solid_velocity_fn: Optional[Callable] = None) -> Scene:
    nx, ny, nz = n
    band = SQRT3 * dx
    cx, cy, cz = _grid_coords(n, dx, (0.5, 0.5, 0.5))
    phi = fluid_fn(cx, cy, cz)
    solid_phi = solid_active = None
    if solid_fn is not None:
        sx, sy, sz = _grid_coords((nx + 1, ny + 1, nz + 1), dx, (0.0, 0.0, 0.0))
        s64 = np.minimum(1.0, solid_fn(sx, sy, sz))
        solid_phi = s64.astype(np.float32)
        solid_active = (np.abs(solid_phi.astype(np.float64)) < band).astype(np.uint8)
        # liquid is pushed out of the solid: value = max(value, -(solid(p)+dx))
        scell = solid_fn(cx, cy, cz)
        phi = np.maximum(phi, -(scell + dx))
    phi32 = phi.astype(np.float32)
    fluid_active = (np.abs(phi32.astype(np.float64)) < band).astype(np.uint8)
    # face velocities: set only where the liquid level set at the face is <= band
    velocity, velocity_active, solid_velocity = [], [], None
    offsets = [(0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)]
    for dim in range(3):
        fshape = (nx + (dim == 0), ny + (dim == 1), nz + (dim == 2))
        fx, fy, fz = _grid_coords(fshape, dx, offsets[dim])
        fphi = fluid_fn(fx, fy, fz)
        if solid_fn is not None:
            fphi = np.maximum(fphi, -(solid_fn(fx, fy, fz) + dx))
        mask = (fphi <= band)
        vals = vel_fn(rng, (fshape[2], fshape[1], fshape[0])).astype(np.float32)
        velocity.append(np.where(mask, vals, np.float32(0)).astype(np.float32))
        velocity_active.append(mask.astype(np.uint8))
    if solid_velocity_fn is not None:
        solid_velocity = []
        for dim in range(3):
            fshape = (nx + (dim == 0), ny + (dim == 1), nz + (dim == 2))
            solid_velocity.append(solid_velocity_fn(rng, (fshape[2], fshape[1], fshape[0])).astype(np.float32))
    return Scene(name=name, nx=nx, ny=ny, nz=nz, dx=dx, dt=dt, tol=tol,
                 fluid_phi=phi32, fluid_active=fluid_active,
                 solid_phi=solid_phi, solid_active=solid_active,
                 velocity=velocity, velocity_active=velocity_active,
                 solid_velocity=solid_velocity, fluid_band=band, solid_band=band)


def _random_boxes(rng, count, edge_lo, edge_hi, centre_lo=0.15, centre_hi=0.85):
    boxes = []
    for _ in range(count):
        c = rng.uniform(centre_lo, centre_hi, size=3)
        e = rng.uniform(edge_lo, edge_hi, size=3)
        boxes.append((c - 0.5 * e, c + 0.5 * e))
    return boxes


def _boxes_fn(boxes):
    def fn(x, y, z):
        out = None
        for lo, hi in boxes:
            v = sdf_box(x, y, z, lo, hi)
            out = v if out is None else np.minimum(out, v)
        return out
    return fn


def dambreak_sphere(n: int = 64, seed: int = 0, tol: float = 1e-4, dt: float = 0.01,
                    solid_velocity: bool = False) -> Scene:
    """Plain CPU-runnable projection: dam-break box (x<0.4, y<0.6) united with
    a sphere (r=0.15 at (0.5,0.75,0.5)), one seeded random box obstacle,
    face velocities uniform in [-1,1]."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    boxes = _random_boxes(rng, 1, 0.1, 0.25, 0.3, 0.7)

    def fluid(x, y, z):
        box = sdf_box(x, y, z, (-1.0, -1.0, -1.0), (0.4, 0.6, 2.0))
        return np.minimum(box, sdf_sphere(x, y, z, (0.5, 0.75, 0.5), 0.15))

    svel = (lambda r, s: r.uniform(-0.5, 0.5, size=s)) if solid_velocity else None
    return _finish("dambreak_sphere", (n, n, n), dx, dt, tol, fluid, _boxes_fn(boxes),
                   lambda r, s: r.uniform(-1.0, 1.0, size=s), rng, svel)


def sloshing_tank(n: int = 256, seed: int = 0, tol: float = 1e-6, dt: float = 0.005) -> Scene:
    """Free surface y = 0.5 + 0.1 sin(2 pi x) cos(2 pi z), eight seeded boxes
    with edges in [0.05,0.2], Gaussian face velocities (sigma 0.5)."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    boxes = _random_boxes(rng, 8, 0.05, 0.2)

    def fluid(x, y, z):
        return y - (0.5 + 0.1 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * z))

    return _finish("sloshing_tank", (n, n, n), dx, dt, tol, fluid, _boxes_fn(boxes),
                   lambda r, s: r.normal(0.0, 0.5, size=s), rng)


def splash(n: int = 384, seed: int = 0, tol: float = 1e-6, dt: float = 0.005, spheres: int = 200) -> Scene:
    """Pool below y=0.3 plus seeded spheres (r in [0.02,0.08]) in y in
    [0.4,0.9]; face velocities uniform in [-2,2]; no obstacle."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    sph = []
    for _ in range(spheres):
        r = rng.uniform(0.02, 0.08)
        c = (rng.uniform(0.1, 0.9), rng.uniform(0.4, 0.9), rng.uniform(0.1, 0.9))
        sph.append((c, r))

    def fluid(x, y, z):
        phi = np.broadcast_to(y - 0.3, np.broadcast_shapes(x.shape, y.shape, z.shape)).copy()
        return _union_spheres(phi, (x, y, z), sph, 3, dx)

    return _finish("splash", (n, n, n), dx, dt, tol, fluid, None,
                   lambda r, s: r.uniform(-2.0, 2.0, size=s), rng)


def dambreak_rain(n: int = 512, seed: int = 0, tol: float = 1e-6, dt: float = 0.005, spheres: int = 100) -> Scene:
    """Dam-break column (resources/liquid/dambreak3.cpp:32-49 geometry) plus
    seeded falling spheres; Gaussian face velocities."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    width, height, level, depth = 0.232, 0.432, 0.095, 0.2532
    sph = []
    for _ in range(spheres):
        r = rng.uniform(0.02, 0.06)
        c = (rng.uniform(0.35, 0.9), rng.uniform(0.5, 0.9), rng.uniform(0.1, 0.9))
        sph.append((c, r))

    def fluid(x, y, z):
        v = np.maximum(np.maximum(x - width, y - height), np.abs(z - 0.5) - depth)
        v = np.minimum(v, y - level)
        v = np.broadcast_to(v, np.broadcast_shapes(x.shape, y.shape, z.shape)).copy()
        return _union_spheres(v, (x, y, z), sph, 3, dx)

    return _finish("dambreak_rain", (n, n, n), dx, dt, tol, fluid, None,
                   lambda r, s: r.normal(0.0, 0.5, size=s), rng)


def training_scene(n: int = 128, seed: int = 0, dt: float = 0.005) -> Scene:
    """Random scene for learned-preconditioner data: pool height U[0.2,0.5],
    1-50 spheres, 0-8 solid boxes, Gaussian face velocities."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    pool = rng.uniform(0.2, 0.5)
    ns = int(rng.integers(1, 51))
    nb = int(rng.integers(0, 9))
    sph = [((rng.uniform(0.1, 0.9), rng.uniform(pool + 0.05, 0.9), rng.uniform(0.1, 0.9)),
            rng.uniform(0.02, 0.1)) for _ in range(ns)]
    boxes = _random_boxes(rng, nb, 0.05, 0.2)

    def fluid(x, y, z):
        phi = np.broadcast_to(y - pool, np.broadcast_shapes(x.shape, y.shape, z.shape)).copy()
        return _union_spheres(phi, (x, y, z), sph, 3, dx)

    return _finish("training", (n, n, n), dx, dt, 1e-6, fluid, _boxes_fn(boxes) if nb else None,
                   lambda r, s: r.normal(0.0, 0.5, size=s), rng)


def analytic_sphere(n: int, r: float = 0.4, band_cells: float = 2.0):
    """accuracytest3 set-up (src/examples/accuracytest3-example.cpp:88-106):
    sphere of radius r at (0.5,0.5,0.5), u = grad |x-c|^2, dt = 1, no solid.
    Returns a Scene (band 2 dx) and the analytic pressure |x-c|^2 - r^2."""
    dx = 1.0 / n
    band = band_cells * dx
    cx, cy, cz = _grid_coords((n, n, n), dx, (0.5, 0.5, 0.5))
    d = np.sqrt((cx - 0.5) ** 2 + (cy - 0.5) ** 2 + (cz - 0.5) ** 2) - r
    phi = np.broadcast_to(d, (n, n, n)).astype(np.float32)
    active = (np.abs(phi.astype(np.float64)) < band).astype(np.uint8)
    velocity, velocity_active = [], []
    offsets = [(0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)]
    for dim in range(3):
        fshape = (n + (dim == 0), n + (dim == 1), n + (dim == 2))
        fx, fy, fz = _grid_coords(fshape, dx, offsets[dim])
        comp = [fx, fy, fz][dim]
        u = np.broadcast_to(2.0 * (comp - 0.5), (fshape[2], fshape[1], fshape[0])).astype(np.float32)
        velocity.append(u.copy())
        velocity_active.append(np.ones(u.shape, np.uint8))
    exact = (cx - 0.5) ** 2 + (cy - 0.5) ** 2 + (cz - 0.5) ** 2 - r * r
    sc = Scene(name="analytic_sphere", nx=n, ny=n, nz=n, dx=dx, dt=1.0, tol=1e-12,
               fluid_phi=phi, fluid_active=active, solid_phi=None, solid_active=None,
               velocity=velocity, velocity_active=velocity_active, solid_velocity=None,
               fluid_band=band, solid_band=SQRT3 * dx)
    return sc, np.broadcast_to(exact, (n, n, n)).copy()


# FLIP particle records in the reference's own layout (macnbflip3::Particle,
# src/flip/macnbflip3.h:128-139: vec3r p; vec3r c[3]; vec3r velocity; Real
# mass, r; char bullet; Real bullet_time, sizing_value; unsigned live_count),
# 84 bytes each; the splat reads p, c, velocity, mass and bullet.
PARTICLE_DTYPE = np.dtype({
    "names": ["p", "c", "velocity", "mass", "r", "bullet", "bullet_time", "sizing_value", "live_count"],
    "formats": [("<f4", (3,)), ("<f4", (3, 3)), ("<f4", (3,)), "<f4", "<f4", "u1", "<f4", "<f4", "<u4"],
    "offsets": [0, 12, 48, 60, 64, 68, 72, 76, 80],
    "itemsize": 84,
})


def flip_particles(scene: Scene, per_cell: int = 8, seed: int = 0, bullet_fraction: float = 0.02,
                   edge_cases: bool = True, band: Optional[float] = None) -> np.ndarray:
    """Seeded FLIP particles for a scene: ``per_cell`` jittered particles in
    every liquid cell (effective level set < 0; with ``band``, only cells whose
    analytic level set is above ``-band * dx``, the narrow band macnbflip3
    keeps particles in: Narrowband = 3 cells by default, macnbflip3.h:108, at
    8 to 12 particles per cell, mass 1/8 each), a smooth velocity field plus
    noise, APIC matrices of a few 1/s, masses around the reference's default
    1/8 (macnbflip3.cpp:42) and a fraction flagged bullet. With
    ``edge_cases``, also particles exactly on cell faces and nodes, one float
    step either side of them, and particles pushed up to 0.45 cells outside
    the domain on every side (collisions leave such particles in the
    reference too)."""
    rng = np.random.default_rng(seed)
    dx = scene.dx
    phi = scene.fluid_effective()
    inside = phi < 0
    if band is not None:
        inside &= scene.fluid_phi > -band * dx   # the analytic (unbanded) level set
    k, j, i = np.nonzero(inside)
    cells = np.repeat(np.stack([i, j, k], 1), per_cell, axis=0).astype(np.float64)
    pos = (cells + rng.random(cells.shape)) * dx
    extra = []
    if edge_cases and len(cells):
        n3 = np.array([scene.nx, scene.ny, scene.nz], np.float64)
        pick = cells[rng.integers(0, len(cells), 96)]
        on = np.floor(pick) * dx
        on[:32, 1:] += 0.5 * dx
        extra.append(on)
        f = on.astype(np.float32)
        extra.append(np.nextafter(f, np.float32(np.inf)).astype(np.float64))
        extra.append(np.nextafter(f, np.float32(-np.inf)).astype(np.float64))
        for axis in range(3):
            for side in (0, 1):
                q = pos[rng.integers(0, len(pos), 16)].copy()
                off = rng.random(16) * 0.45 * dx
                q[:, axis] = -off if side == 0 else n3[axis] * dx + off
                extra.append(q)
    if extra:
        pos = np.concatenate([pos] + extra, 0)
    n = len(pos)
    P = np.zeros(n, PARTICLE_DTYPE)
    P["p"] = pos.astype(np.float32)
    x, y, z = (pos[:, a] for a in range(3))
    vel = np.stack([0.6 * np.sin(2 * np.pi * y) * np.cos(np.pi * z),
                    -0.8 * np.sin(np.pi * x) + 0.3 * np.cos(2 * np.pi * z),
                    0.4 * np.cos(2 * np.pi * x) * np.sin(np.pi * y)], 1)
    vel += 0.05 * rng.standard_normal(vel.shape)
    P["velocity"] = vel.astype(np.float32)
    P["c"] = (2.0 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    P["mass"] = (0.125 * rng.uniform(0.5, 1.5, n)).astype(np.float32)
    P["r"] = np.float32(0.25 * dx)
    P["bullet"] = (rng.random(n) < bullet_fraction).astype(np.uint8)
    P["live_count"] = rng.integers(0, 8, n).astype(np.uint32)
    return P


SCENES = {
    "dambreak_sphere": dambreak_sphere,
    "sloshing_tank": sloshing_tank,
    "splash": splash,
    "dambreak_rain": dambreak_rain,
    "training": training_scene,
}


def make_scene(name: str, **kw) -> Scene:
    return SCENES[name](**kw)

"""Run the compiled reference projection (oracle/_ref) on a scene.

Test infrastructure only: the product never imports this module. It writes a
scene with ``Scene.write_reference_input``, runs ``shkz_ref_harness`` from
``oracle/_ref/<variant>/`` (built by ``oracle/ref/Makefile`` from the
reference's own sources) and reads back what the reference grids hold after
``macpressuresolver3::project`` (src/projection/macpressuresolver3.cpp:54-299).
"""
from __future__ import annotations

import dataclasses
import os
import re
import struct
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ref_available(variant: str = "float") -> bool:
    return os.path.exists(os.path.join(REF_DIR, variant, "shkz_ref_harness"))


@dataclasses.dataclass
class RefResult:
    fluid: np.ndarray
    fluid_active: np.ndarray
    solid: np.ndarray
    solid_active: np.ndarray
    velocity_in: list
    velocity_in_active: list
    pressure: np.ndarray
    pressure_active: np.ndarray
    velocity: list
    velocity_active: list
    projection_ms: float
    iterations: Optional[int] = None
    console_solves: list = dataclasses.field(default_factory=list)
    reresid: Optional[float] = None
    solve_ms: Optional[float] = None
    system: Optional[dict] = None
    stdout: str = ""


def _read_cells(f, shape_zyx):
    n = int(np.prod(shape_zyx))
    v = np.frombuffer(f.read(8 * n), dtype=np.float64).reshape(shape_zyx)
    m = np.frombuffer(f.read(n), dtype=np.uint8).reshape(shape_zyx)
    return v, m


def read_system(path: str) -> dict:
    with open(path, "rb") as f:
        n, nnz = struct.unpack("<2Q", f.read(16))
        indptr = np.frombuffer(f.read(8 * (n + 1)), dtype=np.uint64).astype(np.int64)
        indices = np.frombuffer(f.read(8 * nnz), dtype=np.uint64).astype(np.int64)
        data = np.frombuffer(f.read(8 * nnz), dtype=np.float64)
        rhs = np.frombuffer(f.read(8 * n), dtype=np.float64)
    return {"n": n, "indptr": indptr, "indices": indices, "data": data, "rhs": rhs}


def run_reference(scene, variant: str = "float", mode: str = "mic0", tol: Optional[float] = None,
                  threads: Optional[int] = None, tile_size: int = 8, dump_system: bool = True,
                  repeat: int = 1, extra: Optional[dict] = None, linsolver: str = "refmic0",
                  extra_libpath: Optional[list] = None, density: Optional[list] = None) -> RefResult:
    exe = os.path.join(REF_DIR, variant, "shkz_ref_harness")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    nx, ny, nz = scene.nx, scene.ny, scene.nz
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        out = os.path.join(td, "out.bin")
        scene.write_reference_input(inp)
        args = [exe, inp, out, f"LinSolver={linsolver}", f"RefMode={mode}",
                f"Residual={tol if tol is not None else scene.tol}", f"TileSize={tile_size}",
                f"Threads={threads or os.cpu_count()}", f"HarnessRepeat={repeat}"]
        for k, v in (extra or {}).items():
            args.append(f"{k}={v}")
        if density is not None:
            dpath = os.path.join(td, "density.bin")
            with open(dpath, "wb") as f:
                for d in range(3):
                    f.write(np.ascontiguousarray(density[d], np.float64).tobytes())
            args.append(f"HarnessDensity={dpath}")
        env = dict(os.environ)
        env["LD_LIBRARY_PATH"] = ":".join(list(extra_libpath or []) + [os.path.join(REF_DIR, variant),
                                                                          env.get("LD_LIBRARY_PATH", "")])
        dump = os.path.join(td, "dump")
        env["SHKZ_REF_DUMP"] = dump if dump_system else ""
        proc = subprocess.run(args, cwd=td, env=env, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed ({proc.returncode}):\n{proc.stdout[-3000:]}\n{proc.stderr[-3000:]}")
        with open(out, "rb") as f:
            assert f.read(8) == b"SHKZOUT1"
            hx, hy, hz, real_bytes = struct.unpack("<4i", f.read(16))
            cs = (nz, ny, nx)
            ns = (nz + 1, ny + 1, nx + 1)
            fs = [(nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)]
            fluid, fluid_m = _read_cells(f, cs)
            solid, solid_m = _read_cells(f, ns)
            vin = [_read_cells(f, s) for s in fs]
            p, pm = _read_cells(f, cs)
            vout = [_read_cells(f, s) for s in fs]
            ms = struct.unpack("<d", f.read(8))[0]
        # the reference module's own console line per solve: "Took N iterations, Reresid=X"
        solves = re.findall(r"Took (\d+) iterations, Reresid=([-+]?(?:nan|inf|[0-9]+(?:\.[0-9]*)?(?:[eE][-+]?[0-9]+)?))", proc.stdout)
        res = RefResult(fluid=fluid, fluid_active=fluid_m, solid=solid, solid_active=solid_m,
                        velocity_in=[v for v, _ in vin], velocity_in_active=[m for _, m in vin],
                        pressure=p, pressure_active=pm,
                        velocity=[v for v, _ in vout], velocity_active=[m for _, m in vout],
                        projection_ms=ms,
                        console_solves=[(int(a), float(b)) for a, b in solves], stdout=proc.stdout)
        if dump_system and os.path.exists(dump + ".solve.txt"):
            it, rr, sms = open(dump + ".solve.txt").read().split()
            res.iterations, res.reresid, res.solve_ms = int(it), float(rr), float(sms)
        if dump_system and os.path.exists(dump + ".system.bin"):
            res.system = read_system(dump + ".system.bin")
        return res


def run_reference_splat(nx: int, ny: int, nz: int, dx: float, particles: np.ndarray, velocity: list,
                        velocity_active: list, apic: bool = True, splat_bullet: bool = False,
                        time: float = 0.0, variant: str = "float", module: Optional[str] = None,
                        extra_libpath=None) -> dict:
    """Run the compiled reference FLIP splat (``shkz_ref_splat``: macnbflip3::splat
    then the combined grid velocity of macflipliquid3) on particle records in
    the reference's layout. Returns face grids (lists over dim) under
    ``mass``, ``momentum``, ``splat_active``, ``velocity``, ``velocity_active``,
    and the reference's wall times ``hash_ms``, ``splat_ms``, ``combine_ms``.
    With ``module``, the splat is that FLIP module's (FLIP=<module>, found on
    ``extra_libpath``), loaded by the reference's module loader."""
    exe = os.path.join(REF_DIR, variant, "shkz_ref_splat")
    P = np.ascontiguousarray(particles)
    n = len(P)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(b"SHKZSP01")
            f.write(struct.pack("<3i2dq", nx, ny, nz, dx, time, n))
            f.write(np.ascontiguousarray(P["p"], np.float32).tobytes())
            f.write(np.ascontiguousarray(P["c"], np.float32).tobytes())
            f.write(np.ascontiguousarray(P["velocity"], np.float32).tobytes())
            f.write(np.ascontiguousarray(P["mass"], np.float32).tobytes())
            f.write((np.asarray(P["bullet"]) != 0).astype(np.uint8).tobytes())
            for v, a in zip(velocity, velocity_active):
                f.write(np.ascontiguousarray(v, np.float32).tobytes())
                f.write(np.ascontiguousarray(a, np.uint8).tobytes())
        env = dict(os.environ)
        env["LD_LIBRARY_PATH"] = ":".join(list(extra_libpath or []) + [os.path.join(REF_DIR, variant),
                                                                       env.get("LD_LIBRARY_PATH", "")])
        args = [exe, fin, fout, "APIC=" + ("Yes" if apic else "No"),
                "SplatBulletParticle=" + ("Yes" if splat_bullet else "No")]
        if module:
            args.append("FLIP=" + module)
        proc = subprocess.run(args, cwd=td, env=env, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"reference splat failed ({proc.returncode}):\n{proc.stdout[-2000:]}\n{proc.stderr[-2000:]}")
        out = {k: [] for k in ("mass", "momentum", "splat_active", "velocity", "velocity_active")}
        if not os.path.exists(fout):
            # the module loader ends the process with status 0 when a module is missing
            raise RuntimeError(f"reference splat wrote no output:\n{proc.stdout[-2000:]}\n{proc.stderr[-2000:]}")
        m = re.search(r"hash_ms ([0-9.]+) splat_ms ([0-9.]+) combine_ms ([0-9.]+)", proc.stdout)
        if m:
            out["hash_ms"], out["splat_ms"], out["combine_ms"] = (float(x) for x in m.groups())
        with open(fout, "rb") as f:
            for d in range(3):
                shp = (nz + (d == 2), ny + (d == 1), nx + (d == 0))
                nf = int(np.prod(shp))
                for k, dt_ in (("mass", np.float32), ("momentum", np.float32), ("splat_active", np.uint8),
                               ("velocity", np.float32), ("velocity_active", np.uint8)):
                    w = np.dtype(dt_).itemsize
                    out[k].append(np.frombuffer(f.read(w * nf), dtype=dt_).reshape(shp).copy())
    return out

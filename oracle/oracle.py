"""ctypes bindings of the oracle libraries. TEST INFRASTRUCTURE ONLY.

* ``libhidem_oracle.so`` — the plain-C restatement (oracle/hidem_oracle.c), always built.
* ``_ref/libhidem_ref_{mixed,fp64}.so`` — the reference's own CPU hot path compiled from
  its sources by oracle/Makefile (IEEE flags), when the reference tree was available at
  build time; ``_ref/libhidem_ref_fast_*.so`` — the same with the reference's own
  optimisation flags, used only to time the CPU baseline.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from hidem_b200 import abi

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libhidem_oracle.so"
REF_DIR = HERE / "_ref"

_i64 = C.c_int64
_P = C.POINTER


class _quiet_stdout:
    """Sends C-level stdout to /dev/null while the reference code runs: its Logger prints
    progress lines (e.g. NeighbourGrid::generate, PLiB/NeighbourGrid.cpp:67) that would
    mix into a caller's machine-readable output."""

    def __enter__(self):
        import os
        import sys
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        import os
        C.CDLL(None).fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)


def _bind(lib, prefix: str):
    getattr(lib, prefix + "_cells").argtypes = [_P(abi.HidemParams), _P(abi.HidemParticleSoA), _i64,
                                                C.c_void_p, C.c_void_p, C.c_void_p, _P(_i64),
                                                _P(C.c_double)]
    getattr(lib, prefix + "_neighbours").argtypes = [_P(abi.HidemParams), _P(abi.HidemParticleSoA),
                                                     _i64, C.c_void_p, C.c_void_p, _i64, _P(_i64)]
    getattr(lib, prefix + "_run").argtypes = [
        _P(abi.HidemParams), _P(abi.HidemParticleSoA), _i64, _P(abi.HidemLinkSoA), _i64, _i64,
        C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, _i64, _P(_i64), C.c_void_p, _i64, _P(_i64),
        _P(C.c_double)]
    for name in ("_cells", "_neighbours", "_run"):
        getattr(lib, prefix + name).restype = C.c_int
    getattr(lib, prefix + "_threads").restype = C.c_int
    return lib


class CpuPath:
    """One CPU implementation of the hot path: the C restatement ('port') or the
    reference's own code ('reference')."""

    def __init__(self, path: Path, prefix: str, kind: str, precision: int | None = None):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        self.lib = _bind(C.CDLL(str(path)), prefix)
        self.prefix = prefix
        self.kind = kind
        self.path = path
        self.fixed_precision = precision

    def threads(self) -> int:
        return int(getattr(self.lib, self.prefix + "_threads")())

    def set_maps(self, bed=None, friction=None, ext=None) -> None:
        """Bed / friction / external force maps (abi.map2d structs) of the next runs; the
        caller keeps the data arrays alive."""
        f = getattr(self.lib, self.prefix + "_set_maps")
        f.argtypes = [_P(abi.HidemMap2d), _P(abi.HidemMap2d), _P(abi.HidemMap2d)]
        f.restype = None
        extarr = (abi.HidemMap2d * 6)(*ext) if ext is not None else None
        f(C.byref(bed) if bed is not None else None, C.byref(friction) if friction is not None else None,
          extarr)

    def set_mesh(self, mesh=None) -> None:
        """Collision mesh (an abi.mesh struct) of the next runs; the caller keeps its arrays
        alive."""
        f = getattr(self.lib, self.prefix + "_set_mesh")
        f.argtypes = [_P(abi.HidemMesh)]
        f.restype = None
        with _quiet_stdout():
            f(C.byref(mesh) if mesh is not None else None)
        self._mesh_tris = int(mesh.triangles) if mesh is not None else 0

    def mesh_face_forces(self, precision: int) -> np.ndarray:
        """[triangles][3] face forces of the last run with a mesh."""
        lp = abi.lp_dtype(precision)
        out = [np.zeros(self._mesh_tris, lp) for _ in range(3)]
        f = getattr(self.lib, self.prefix + "_mesh_face_forces")
        f.argtypes = [C.c_void_p] * 3
        f.restype = C.c_int
        rc = f(*[a.ctypes.data for a in out])
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_mesh_face_forces failed ({rc})")
        return np.stack(out, axis=1)

    def mesh_accel(self, precision: int) -> dict:
        """The MeshAccel grid of the set mesh (the contract of hidem_get_mesh_accel)."""
        from hidem_b200.hidemlib import _mesh_accel
        f = getattr(self.lib, self.prefix + "_mesh_accel")
        port = self.prefix == "hidem_oracle"  # the port builds the grid in either precision
        f.argtypes = ([C.c_int32] if port else []) + [C.c_void_p] * 6 + [_i64, _P(_i64)]
        f.restype = C.c_int

        def call(*a):
            rc = f(precision, *a) if port else f(*a)
            if rc != 0:
                raise RuntimeError(f"{self.prefix}_mesh_accel failed ({rc})")
        return _mesh_accel(call)

    def _prec(self, params) -> int:
        p = int(params.precision)
        if self.fixed_precision is not None and p != self.fixed_precision:
            raise ValueError(f"{self.path.name} is built for precision {self.fixed_precision}")
        return p

    def cells(self, params, particles: dict):
        prec = self._prec(params)
        n = particles["xCord"].shape[0]
        soa = abi.particle_soa(particles, prec, n)
        ix, iy, iz = (np.zeros(n, np.int32) for _ in range(3))
        dims = (_i64 * 3)()
        mins = (C.c_double * 3)()
        with _quiet_stdout():
            rc = getattr(self.lib, self.prefix + "_cells")(C.byref(params), C.byref(soa), n,
                                                           ix.ctypes.data, iy.ctypes.data,
                                                           iz.ctypes.data, dims, mins)
        if rc:
            raise RuntimeError(f"{self.prefix}_cells -> {rc}")
        return ix, iy, iz, tuple(dims), tuple(mins)

    def neighbours(self, params, particles: dict):
        prec = self._prec(params)
        n = particles["xCord"].shape[0]
        soa = abi.particle_soa(particles, prec, n)
        counts = np.zeros(n, np.int32)
        total = _i64()
        f = getattr(self.lib, self.prefix + "_neighbours")
        with _quiet_stdout():
            rc = f(C.byref(params), C.byref(soa), n, counts.ctypes.data, None, 0, C.byref(total))
        if rc:
            raise RuntimeError(f"{self.prefix}_neighbours -> {rc}")
        lst = np.zeros(max(total.value, 1), np.int32)
        with _quiet_stdout():
            rc = f(C.byref(params), C.byref(soa), n, counts.ctypes.data, lst.ctypes.data,
                   lst.shape[0], C.byref(total))
        if rc:
            raise RuntimeError(f"{self.prefix}_neighbours -> {rc}")
        return counts, lst[: total.value]

    def run(self, params, particles: dict, links: dict, nsteps: int, start_step: int = 0):
        """Runs the timestep loop on copies of the inputs. Returns (particles, links,
        forces[6,n] of the last step, events (link, step), regen steps, seconds)."""
        prec = self._prec(params)
        p = {k: v.copy() for k, v in particles.items()}
        l = {k: v.copy() for k, v in links.items()}
        n = p["xCord"].shape[0]
        L = l["globalKeyEndA"].shape[0]
        psoa = abi.particle_soa(p, prec, n)
        lsoa = abi.link_soa(l, prec, L)
        lp = abi.lp_dtype(prec)
        F = np.zeros((6, n), lp)
        fptr = (C.c_void_p * 6)(*[F[k].ctypes.data for k in range(6)])
        cap = max(L, 1)
        ev_l = np.zeros(cap, np.int64)
        ev_s = np.zeros(cap, np.int64)
        nev = _i64()
        rcap = nsteps + 1
        rg = np.zeros(rcap, np.int64)
        nrg = _i64()
        secs = C.c_double()
        with _quiet_stdout():
            rc = getattr(self.lib, self.prefix + "_run")(
                C.byref(params), C.byref(psoa), n, C.byref(lsoa), L, start_step, nsteps, fptr,
                ev_l.ctypes.data, ev_s.ctypes.data, cap, C.byref(nev), rg.ctypes.data, rcap,
                C.byref(nrg), C.byref(secs))
        if rc:
            raise RuntimeError(f"{self.prefix}_run -> {rc}")
        k = min(nev.value, cap)
        order = np.lexsort((ev_l[:k], ev_s[:k]))
        events = np.stack([ev_l[:k][order], ev_s[:k][order]], axis=1)
        return p, l, F, events, rg[: min(nrg.value, rcap)], secs.value


def port() -> CpuPath:
    return CpuPath(ORACLE_LIB, "hidem_oracle", "port")


def reference(precision: int, fast: bool = False) -> CpuPath:
    tag = ("fast_" if fast else "") + ("mixed" if precision == abi.PREC_MIXED else "fp64")
    return CpuPath(REF_DIR / f"libhidem_ref_{tag}.so", "hidem_ref", "reference", precision)


def reference_available(precision: int, fast: bool = False) -> bool:
    tag = ("fast_" if fast else "") + ("mixed" if precision == abi.PREC_MIXED else "fp64")
    return (REF_DIR / f"libhidem_ref_{tag}.so").exists()


class RefSession:
    """A persistent run of the reference's CPU timestep loop (oracle/_ref), so steps can be
    timed without its setup: ``advance(k)`` returns the seconds of k timesteps, excluding
    the rebuild of the first one."""

    def __init__(self, params, particles: dict, links: dict, fast: bool = True, start_step: int = 0):
        prec = int(params.precision)
        tag = ("fast_" if fast else "") + ("mixed" if prec == abi.PREC_MIXED else "fp64")
        path = REF_DIR / f"libhidem_ref_{tag}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        lib = C.CDLL(str(path))
        lib.hidem_ref_open.restype = C.c_void_p
        lib.hidem_ref_open.argtypes = [_P(abi.HidemParams), _P(abi.HidemParticleSoA), _i64,
                                       _P(abi.HidemLinkSoA), _i64, _i64]
        lib.hidem_ref_advance.restype = C.c_int
        lib.hidem_ref_advance.argtypes = [C.c_void_p, C.c_int32, _P(C.c_double)]
        lib.hidem_ref_close.argtypes = [C.c_void_p]
        lib.hidem_ref_threads.restype = C.c_int
        self.lib = lib
        self.path = path
        self.params = params
        n = particles["xCord"].shape[0]
        L = links["globalKeyEndA"].shape[0]
        psoa = abi.particle_soa(particles, prec, n)
        lsoa = abi.link_soa(links, prec, L)
        self.n = n
        with _quiet_stdout():
            self.h = lib.hidem_ref_open(C.byref(params), C.byref(psoa), n, C.byref(lsoa), L,
                                        start_step)

    def threads(self) -> int:
        return int(self.lib.hidem_ref_threads())

    def advance(self, nsteps: int) -> float:
        secs = C.c_double()
        with _quiet_stdout():
            rc = self.lib.hidem_ref_advance(self.h, nsteps, C.byref(secs))
        if rc:
            raise RuntimeError(f"hidem_ref_advance -> {rc}")
        return secs.value

    def close(self):
        if self.h:
            self.lib.hidem_ref_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

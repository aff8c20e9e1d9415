"""Python host mirror of the reference's ``HiDEMLib`` operator surface over the C ABI.

Method names follow ``HiDEMLib<PDataT, LDataT>`` (HiDEMLib/HiDEMLib.h): ``gridService``
(533-628), ``computePartForce`` (316-382) with the default contact and beam functors,
``applyForce`` (303-314) with the sample integrate step, ``linkUpdate`` (256-269) with the
default break functor, ``finalizeTs`` (495-530), ``getCurrentTimestep`` (245-247), ``run``
(234-240). ``step(n)`` runs n whole timesteps of the sample main loop
(HiDEM/MeshBlock/MainMeshBlock.cpp:274-323) on the device, each as the context's step kernel
(one fused kernel, or the two-pass step's passes).

Errors follow the C ABI: every failing call raises ``HidemError`` carrying the status and
``hidem_last_error`` text (the reference would print and ``exit(1)``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class HiDEMLib:
    def __init__(self, params: abi.HidemParams, device: int = 0, end_timestep: int | None = None):
        self._lib = abi.load()
        self.params = params
        self._mesh_tris = 0
        self.device = int(device)
        self.precision = int(params.precision)
        self.lp = abi.lp_dtype(self.precision)
        h = C.c_void_p()
        st = self._lib.hidem_create(C.byref(params), int(device), C.byref(h))
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_create_error().decode())
        self._ctx = h
        self.n = 0
        self.L = 0
        self.end_timestep = end_timestep

    # ------------------------------------------------------------ plumbing
    def _check(self, st: int) -> None:
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_last_error(self._ctx).decode())

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.hidem_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self._lib.hidem_get_stream(self._ctx) or 0)

    # ------------------------------------------------------------ data
    def set_particles(self, arrays: dict) -> None:
        n = int(arrays["xCord"].shape[0])
        soa = abi.particle_soa(arrays, self.precision, n)
        self._check(self._lib.hidem_set_particles(self._ctx, C.byref(soa), n))
        self.n = n

    def set_links(self, arrays: dict) -> None:
        L = int(arrays["globalKeyEndA"].shape[0])
        soa = abi.link_soa(arrays, self.precision, L)
        self._check(self._lib.hidem_set_links(self._ctx, C.byref(soa), L))
        self.L = L

    def set_timestep(self, step: int) -> None:
        self._check(self._lib.hidem_set_timestep(self._ctx, int(step)))

    def set_params(self, params: abi.HidemParams) -> None:
        self._check(self._lib.hidem_set_params(self._ctx, C.byref(params)))
        self.params = params

    # ------------------------------------------------------------ timestep surface
    def gridService(self) -> None:
        self._check(self._lib.hidem_grid_service(self._ctx))

    def regenerate(self) -> None:
        self._check(self._lib.hidem_regenerate(self._ctx))

    def computePartForce(self) -> None:
        self._check(self._lib.hidem_compute_forces(self._ctx))

    def applyForce(self) -> None:
        self._check(self._lib.hidem_integrate(self._ctx))

    def linkUpdate(self) -> None:
        self._check(self._lib.hidem_link_update(self._ctx))

    def finalizeTs(self) -> None:
        self._check(self._lib.hidem_finalize_ts(self._ctx))

    def getCurrentTimestep(self) -> int:
        return int(self.stats()["step"])

    def run(self) -> bool:
        return self.end_timestep is None or self.getCurrentTimestep() < self.end_timestep

    def breakActive(self, step: int | None = None) -> bool:
        """The sample main's gate ``getCurrentTimestep() * dt > breakTime`` in lp (at
        ``step`` when given, which saves reading the context's statistics)."""
        lp = self.lp
        t = lp(self.getCurrentTimestep() if step is None else step)
        return bool(lp(t * lp(self.params.dt)) > lp(self.params.breakTime))

    def timestep_split(self) -> None:
        """One sample-main timestep through the separate operator calls."""
        self.gridService()
        self.computePartForce()
        self.applyForce()
        if self.breakActive():
            self.linkUpdate()
        self.finalizeTs()

    def step(self, nsteps: int = 1) -> None:
        self._check(self._lib.hidem_step(self._ctx, int(nsteps)))

    # ------------------------------------------------------------ slab decomposition hooks
    def grid_service_local(self) -> tuple[np.ndarray, bool]:
        """This rank's maxima of max(0, x/y/zDiff) and whether gridService reads them now."""
        mx = np.zeros(3)
        wants = C.c_int32()
        self._check(self._lib.hidem_grid_service_local(self._ctx, mx.ctypes.data, C.byref(wants)))
        return mx, bool(wants.value)

    def grid_service_decide(self, diff_max) -> bool:
        """gridService's decision from the maxima over all ranks; True: rebuild now."""
        mx = np.ascontiguousarray(diff_max, np.float64)
        regen = C.c_int32()
        self._check(self._lib.hidem_grid_service_decide(self._ctx, mx.ctypes.data, C.byref(regen)))
        return bool(regen.value)

    def local_bounds(self) -> tuple[np.ndarray, np.ndarray]:
        lo, hi = np.zeros(3), np.zeros(3)
        self._check(self._lib.hidem_local_bounds(self._ctx, lo.ctypes.data, hi.ctypes.data))
        return lo, hi

    def regenerate_frame(self, lower, upper) -> None:
        """Rebuild with the grid spanning [lower, upper] (every rank's particles)."""
        lo = np.ascontiguousarray(lower, np.float64)
        hi = np.ascontiguousarray(upper, np.float64)
        self._check(self._lib.hidem_regenerate_frame(self._ctx, lo.ctypes.data, hi.ctypes.data))

    def set_halo_exchange(self, send_index, recv_index) -> None:
        """Particle indices (input order) whose forces are sent / received each step."""
        snd = np.ascontiguousarray(send_index, np.int32)
        rcv = np.ascontiguousarray(recv_index, np.int32)
        self._check(self._lib.hidem_set_halo_exchange(self._ctx, snd.ctypes.data, snd.shape[0],
                                                      rcv.ctypes.data, rcv.shape[0]))

    def compute_forces_packed(self, device_ptr: int) -> None:
        """computePartForce with the halo send records written by the force pass itself
        (hidem_compute_forces_packed)."""
        self._check(self._lib.hidem_compute_forces_packed(self._ctx, C.c_void_p(device_ptr)))

    def pack_halo_forces(self, device_ptr: int) -> None:
        self._check(self._lib.hidem_pack_halo_forces(self._ctx, C.c_void_p(device_ptr)))

    def unpack_halo_forces(self, device_ptr: int) -> None:
        self._check(self._lib.hidem_unpack_halo_forces(self._ctx, C.c_void_p(device_ptr)))

    def set_bed_maps(self, bed=None, friction=None) -> None:
        """GlacierDem bed height / friction maps (abi.map2d structs, or None)."""
        self._check(self._lib.hidem_set_bed_maps(self._ctx, C.byref(bed) if bed is not None else None,
                                                 C.byref(friction) if friction is not None else None))

    def set_external_force_maps(self, maps=None) -> None:
        """Six external force maps (x, y, z, u, v, w; abi.map2d structs), or None."""
        arr = (abi.HidemMap2d * 6)(*maps) if maps is not None else None
        self._check(self._lib.hidem_set_external_force_maps(self._ctx, arr))

    def set_collision_mesh(self, mesh=None) -> None:
        """Collision mesh (an abi.mesh struct; the data is copied), or None to remove it."""
        self._check(self._lib.hidem_set_collision_mesh(self._ctx, C.byref(mesh) if mesh is not None else None))
        self._mesh_tris = int(mesh.triangles) if mesh is not None else 0

    def mesh_face_forces(self) -> np.ndarray:
        """[triangles][3] face forces accumulated since the mesh was set or zeroed."""
        lp = abi.lp_dtype(int(self.params.precision))
        out = [np.zeros(self._mesh_tris, lp) for _ in range(3)]
        self._check(self._lib.hidem_get_mesh_face_forces(self._ctx, *[a.ctypes.data for a in out]))
        return np.stack(out, axis=1)

    def zero_mesh_face_forces(self) -> None:
        self._check(self._lib.hidem_zero_mesh_face_forces(self._ctx))

    def mesh_accel(self) -> dict:
        """The MeshAccel grid: counts, lower, upper, sizes, starts, values."""
        return _mesh_accel(lambda *a: self._check(self._lib.hidem_get_mesh_accel(self._ctx, *a)))

    def functor_params(self) -> abi.HidemFunctorParams:
        """The default functors' parameters in use (derived from the run config unless set)."""
        f = abi.HidemFunctorParams()
        self._check(self._lib.hidem_get_functor_params(self._ctx, C.byref(f)))
        return f

    def set_functor_params(self, f: abi.HidemFunctorParams) -> None:
        """Replaces the default functors' parameters (as a caller's main constructs them)."""
        self._check(self._lib.hidem_set_functor_params(self._ctx, C.byref(f)))

    def momentum(self) -> tuple[np.ndarray, np.ndarray]:
        """(linear [3], angular about the origin [3]) momentum of the current state."""
        lin, ang = np.zeros(3), np.zeros(3)
        self._check(self._lib.hidem_momentum(self._ctx, lin.ctypes.data, ang.ctypes.data))
        return lin, ang

    def kinetic_energy(self) -> tuple[float, float, float]:
        """(translational, rotational, max speed) of the current state."""
        t, r, v = C.c_double(), C.c_double(), C.c_double()
        self._check(self._lib.hidem_kinetic_energy(self._ctx, C.byref(t), C.byref(r), C.byref(v)))
        return t.value, r.value, v.value

    def set_step_kernel(self, kernel: int) -> None:
        """abi.STEP_KERNEL_* (AUTO: timed on the first fused steps)."""
        self._check(self._lib.hidem_set_step_kernel(self._ctx, int(kernel)))

    def device_view(self) -> abi.HidemDeviceView:
        """The context's device arrays (hidem_get_device_view), valid until the next call
        that rebuilds or steps."""
        v = abi.HidemDeviceView()
        self._check(self._lib.hidem_get_device_view(self._ctx, C.byref(v)))
        return v

    def set_checks(self, flags: int) -> None:
        """abi.CHECK_* bits (hidem_set_checks): CHECK_GRID_GROWTH refuses a rebuild whose
        grid has more than 10x the previous one's cells."""
        self._check(self._lib.hidem_set_checks(self._ctx, int(flags)))

    def step_kernel(self) -> int:
        return int(self._lib.hidem_get_step_kernel(self._ctx))

    def profile(self, enable: bool = True) -> None:
        """CUDA-event timing of each step's kernels on the context's stream."""
        self._check(self._lib.hidem_profile(self._ctx, 1 if enable else 0))

    def profile_read(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        self._check(self._lib.hidem_profile_read(self._ctx, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def synchronize(self) -> None:
        self._check(self._lib.hidem_synchronize(self._ctx))

    # ------------------------------------------------------------ checkpoint
    def write_checkpoint(self, path: str) -> None:
        """HiDEMH5Checkpoint::writeCheckpoint layout (one rank)."""
        self._check(self._lib.hidem_checkpoint_write(self._ctx, str(path).encode()))

    def read_checkpoint(self, path: str) -> None:
        """HiDEMLib::setFromRestart + fromCheckpoint: timestep, particles, links, CT."""
        self._check(self._lib.hidem_checkpoint_read(self._ctx, str(path).encode()))
        s = self.stats()
        self.n = int(s["num_particles"])
        self.L = int(s["num_links"])

    # ------------------------------------------------------------ readback
    def get_particles(self, out: dict | None = None) -> dict:
        """Particle state in input order, into `out` (e.g. pinned arrays) when given."""
        if out is None:
            out = abi.empty_particles(self.n, self.precision)
        soa = abi.particle_soa(out, self.precision, self.n)
        self._check(self._lib.hidem_get_particles(self._ctx, C.byref(soa)))
        return out

    def get_links(self, out: dict | None = None) -> dict:
        if out is None:
            out = abi.empty_links(self.L, self.precision)
        soa = abi.link_soa(out, self.precision, self.L)
        self._check(self._lib.hidem_get_links(self._ctx, C.byref(soa)))
        return out

    def get_particles_device(self, fields=None) -> dict:
        """Particle state in input order as torch tensors on the context's GPU (copied on
        the device); only `fields` when given."""
        import torch
        out = abi.empty_particles_torch(self.n, self.precision, torch.device("cuda", self.device))
        if fields is not None:
            out = {k: out[k] for k in fields}
        return self.get_particles(out)

    def get_links_device(self) -> dict:
        """Link state in input order as torch tensors on the context's GPU."""
        import torch
        return self.get_links(abi.empty_links_torch(self.L, self.precision, torch.device("cuda", self.device)))

    def get_forces(self) -> np.ndarray:
        f = np.zeros((6, self.n), self.lp)
        ptrs = (C.c_void_p * 6)(*[f[k].ctypes.data for k in range(6)])
        self._check(self._lib.hidem_get_forces(self._ctx, ptrs))
        return f

    def get_cells(self):
        ix = np.zeros(self.n, np.int32)
        iy = np.zeros(self.n, np.int32)
        iz = np.zeros(self.n, np.int32)
        dims = (C.c_int64 * 3)()
        mins = (C.c_double * 3)()
        self._check(self._lib.hidem_get_cells(self._ctx, ix.ctypes.data, iy.ctypes.data,
                                              iz.ctypes.data, dims, mins))
        return ix, iy, iz, tuple(dims), tuple(mins)

    def get_neighbours(self):
        counts = np.zeros(self.n, np.int32)
        total = C.c_int64()
        self._check(self._lib.hidem_get_neighbours(self._ctx, counts.ctypes.data, None, 0,
                                                   C.byref(total)))
        lst = np.zeros(max(total.value, 1), np.int32)
        self._check(self._lib.hidem_get_neighbours(self._ctx, counts.ctypes.data, lst.ctypes.data,
                                                   lst.shape[0], C.byref(total)))
        return counts, lst[: total.value]

    def get_break_events(self, cap: int | None = None):
        cap = self.L if cap is None else cap
        li = np.zeros(max(cap, 1), np.int64)
        st = np.zeros(max(cap, 1), np.int64)
        cnt = C.c_int64()
        self._check(self._lib.hidem_get_break_events(self._ctx, li.ctypes.data, st.ctypes.data,
                                                     cap, C.byref(cnt)))
        return li[: cnt.value], st[: cnt.value]

    def stats(self) -> dict:
        s = abi.HidemStats()
        self._check(self._lib.hidem_get_stats(self._ctx, C.byref(s)))
        return s.as_dict()


class HiDEMBatch:
    """Independent contexts advanced together, one kernel launch per timestep over all of
    them (``hidem_batch_*``; no counterpart in the reference). Each context's results are
    those of ``HiDEMLib.step`` on it alone. The contexts must stay open while the batch
    exists; ``close`` the batch first."""

    def __init__(self, libs: list[HiDEMLib], graphs: bool = True, per_context: bool = False):
        self._lib = abi.load()
        self.libs = list(libs)
        arr = (C.c_void_p * len(self.libs))(*[l._ctx for l in self.libs])
        flags = (abi.BATCH_GRAPHS if graphs else 0) | (abi.BATCH_PER_CONTEXT if per_context else 0)
        h = C.c_void_p()
        st = self._lib.hidem_batch_create(arr, len(self.libs), flags, C.byref(h))
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_create_error().decode())
        self._b = h

    def _check(self, st: int) -> None:
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_batch_last_error(self._b).decode())

    def step(self, nsteps: int = 1) -> None:
        self._check(self._lib.hidem_batch_step(self._b, int(nsteps)))

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t the batch's work runs on."""
        return int(self._lib.hidem_batch_get_stream(self._b) or 0)

    def counts(self) -> dict:
        v = [C.c_int64() for _ in range(3)]
        self._check(self._lib.hidem_batch_counts(self._b, *[C.byref(x) for x in v]))
        return dict(launches=v[0].value, graph_launches=v[1].value, uploads=v[2].value)

    def close(self) -> None:
        if getattr(self, "_b", None):
            self._lib.hidem_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _mesh_accel(call) -> dict:
    """Reads a MeshAccel grid through `call(counts, lower, upper, sizes, starts, values, cap,
    count)` (the contract of hidem_get_mesh_accel), sizing the arrays from a first call."""
    counts = np.zeros(3, np.int32)
    lower, upper = np.zeros(3), np.zeros(3)
    nv = C.c_int64()
    call(counts.ctypes.data, lower.ctypes.data, upper.ctypes.data, None, None, None, 0, C.byref(nv))
    cells = int(np.prod(counts.astype(np.int64)))
    sizes, starts = np.zeros(cells, np.int32), np.zeros(cells, np.int32)
    values = np.zeros(max(nv.value, 1), np.int32)
    call(counts.ctypes.data, lower.ctypes.data, upper.ctypes.data, sizes.ctypes.data, starts.ctypes.data,
         values.ctypes.data, values.shape[0], C.byref(nv))
    return {"counts": counts, "lower": lower, "upper": upper, "sizes": sizes, "starts": starts,
            "values": values[:nv.value]}

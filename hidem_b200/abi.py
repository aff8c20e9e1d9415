"""ctypes mirror of ``include/hidem_b200.h`` and loader of ``libhidem_b200.so``.

The library is the product: there is no Python or CPU fallback. ``load()`` raises when
the in-tree shared object is missing (build it with ``python -m hidem_b200.build``).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libhidem_b200.so"

HIDEM_OK = 0
HIDEM_ERR_ARG, HIDEM_ERR_CUDA, HIDEM_ERR_STATE, HIDEM_ERR_CAPACITY = 1, 2, 3, 4
HIDEM_ERR_IO, HIDEM_ERR_DEVICE, HIDEM_ERR_NOT_FOUND = 5, 6, 7
STATUS_NAMES = {0: "HIDEM_OK", 1: "HIDEM_ERR_ARG", 2: "HIDEM_ERR_CUDA", 3: "HIDEM_ERR_STATE",
                4: "HIDEM_ERR_CAPACITY", 5: "HIDEM_ERR_IO", 6: "HIDEM_ERR_DEVICE",
                7: "HIDEM_ERR_NOT_FOUND"}
PREC_FP64 = 0
PREC_MIXED = 1
TYPE_FIXED = 0x40
TYPE_FRONT = 0x80
BATCH_GRAPHS = 1
BATCH_PER_CONTEXT = 2
CHECK_GRID_GROWTH = 1

STEP_KERNEL_AUTO = 0
STEP_KERNEL_ITEMS = 1
STEP_KERNEL_THREAD = 2
STEP_KERNEL_THREAD_CAPPED = 3
STEP_KERNEL_THREAD_ASYNC = 4
STEP_KERNEL_TWO_PASS = 5
SURROGATE_FORWARD_AUTO = 0
SURROGATE_FORWARD_BLOCK = 1
SURROGATE_FORWARD_PINGPONG = 2

_d = C.c_double
_i32 = C.c_int32
_i64 = C.c_int64
_p = C.c_void_p


class HidemParams(C.Structure):
    _fields_ = [
        ("dt", _d), ("scale", _d), ("E", _d), ("beamWidth", _d), ("damping", _d),
        ("dampingRotation", _d), ("attractDistance", _d), ("attractScaleForce", _d),
        ("maxLoad", _d), ("bendBreak", _d), ("breakTime", _d),
        ("g", _d), ("rhoIce", _d), ("rhoWater", _d), ("waterLevel", _d),
        ("airDrag", _d), ("waterDrag", _d), ("bedDrag", _d), ("bedStiffness", _d),
        ("bedInteract", _d), ("maxVel", _d), ("maxRot", _d),
        ("lowerLimit", _d * 3), ("upperLimit", _d * 3),
        ("boundaryMin", _i32 * 3), ("boundaryMax", _i32 * 3),
        ("searchDistanceScale", _d), ("gridRegenInterval", _i32), ("firstBalanceTimestep", _i32),
        ("maxRadius", _d),
        ("useBed", _i32), ("bedHeight", _d), ("bedFriction", _d),
        ("useVelocityLimit", _i32), ("useBoundary", _i32), ("useFixed", _i32),
        ("useFrontPressure", _i32), ("precision", _i32),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class HidemParticleSoA(C.Structure):
    _fields_ = [("xCord", _p), ("yCord", _p), ("zCord", _p),
                ("xTheta", _p), ("yTheta", _p), ("zTheta", _p),
                ("xDiff", _p), ("yDiff", _p), ("zDiff", _p),
                ("uDiff", _p), ("vDiff", _p), ("wDiff", _p),
                ("radius", _p), ("owners", _p), ("type", _p), ("globalKeys", _p)]


class HidemLinkSoA(C.Structure):
    _fields_ = [("owners", _p), ("state", _p), ("globalKeys", _p), ("globalKeyEndA", _p),
                ("globalKeyEndB", _p), ("initialLen", _p), ("particleLinkNum", _p),
                ("CT", _p * 6)]


class HidemDeviceView(C.Structure):
    """hidem_device_view: the context's device arrays (include/hidem_b200_iterate.cuh)."""
    _fields_ = [("precision", _i32), ("record_bytes", _i32), ("n", _i64), ("L", _i64), ("step", _i64),
                ("records", _p), ("force", _p), ("type", _p), ("input_index", _p), ("slot_of", _p),
                ("counts", _p), ("contact_offsets", _p), ("contacts", _p), ("end_offsets", _p),
                ("end_partner", _p), ("end_ct", _p * 6), ("end_state", _p), ("end_initial_length", _p),
                ("end_link", _p), ("link_state", _p), ("link_slot_a", _p), ("link_slot_b", _p),
                ("link_initial_length", _p), ("link_end_index", _p), ("events", _p),
                ("event_count", _p), ("event_capacity", _i64), ("stream", _p)]


class HidemStats(C.Structure):
    _fields_ = [("step", _i64), ("num_particles", _i64), ("num_links", _i64),
                ("num_neighbour_pairs", _i64), ("max_neighbours", _i64),
                ("max_links_per_particle", _i64), ("grid_dims", _i64 * 3), ("grid_min", _d * 3),
                ("regen_count", _i64), ("last_regen_step", _i64), ("accumulated_dist", _d),
                ("search_distance", _d), ("interact_distance", _d), ("broken_links", _i64),
                ("kernel_launches", _i64), ("grid_growth_events", _i64)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


# field order of the reference (HiDEMLib/HiDEMParticleData.h:45-51, HiDEMLinkData.h:39-50)
PARTICLE_FIELDS = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff",
                   "zDiff", "uDiff", "vDiff", "wDiff", "radius", "owners", "type", "globalKeys"]
LP_PARTICLE_FIELDS = ["xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff", "uDiff", "vDiff",
                      "wDiff", "radius"]
LINK_FIELDS = ["owners", "state", "globalKeys", "globalKeyEndA", "globalKeyEndB", "initialLen",
               "particleLinkNum"]
SIDE_FIELDS = ["CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]


def lp_dtype(precision: int):
    return np.float32 if precision == PREC_MIXED else np.float64


def particle_dtypes(precision: int) -> dict:
    lp = lp_dtype(precision)
    d = {k: lp for k in LP_PARTICLE_FIELDS}
    d.update(xCord=np.float64, yCord=np.float64, zCord=np.float64, owners=np.int32,
             type=np.uint8, globalKeys=np.int64)
    return d


def link_dtypes(precision: int) -> dict:
    lp = lp_dtype(precision)
    d = dict(owners=np.int32, state=np.uint8, globalKeys=np.int64, globalKeyEndA=np.int64,
             globalKeyEndB=np.int64, initialLen=lp, particleLinkNum=np.int32)
    d.update({k: lp for k in SIDE_FIELDS})
    return d


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _field_ptr(kind: str, k: str, a, dt, count: int | None):
    """The address of a field array — a numpy array, or a torch tensor in host or device
    memory (the library copies from / to either) — checked for dtype, layout and size."""
    if hasattr(a, "data_ptr"):  # torch tensor
        import torch
        want = getattr(torch, np.dtype(dt).name)
        if a.dtype != want or not a.is_contiguous() or a.dim() != 1:
            raise TypeError(f"{kind} field {k}: need a contiguous 1-D {want} tensor, got {a.dtype}")
        if count is not None and a.shape[0] != count:
            raise ValueError(f"{kind} field {k}: {a.shape[0]} elements, expected {count}")
        return C.c_void_p(a.data_ptr()) if a.numel() else None
    if a.dtype != dt or not a.flags.c_contiguous:
        raise TypeError(f"{kind} field {k}: need contiguous {np.dtype(dt)}, got {a.dtype}")
    if count is not None and a.shape[0] != count:
        raise ValueError(f"{kind} field {k}: {a.shape[0]} elements, expected {count}")
    return _ptr(a)


def particle_soa(arrays: dict, precision: int, n: int | None = None) -> HidemParticleSoA:
    """A particle SoA struct pointing into `arrays` (numpy arrays or torch tensors, host or
    device memory; checked for dtype / size)."""
    s = HidemParticleSoA()
    dts = particle_dtypes(precision)
    for k in PARTICLE_FIELDS:
        a = arrays.get(k)
        if a is None:
            continue
        setattr(s, k, _field_ptr("particle", k, a, dts[k], n))
    return s


def link_soa(arrays: dict, precision: int, L: int | None = None) -> HidemLinkSoA:
    s = HidemLinkSoA()
    dts = link_dtypes(precision)
    for k in LINK_FIELDS:
        a = arrays.get(k)
        if a is None:
            continue
        setattr(s, k, _field_ptr("link", k, a, dts[k], L))
    for i, k in enumerate(SIDE_FIELDS):
        a = arrays.get(k)
        if a is None:
            continue
        s.CT[i] = _field_ptr("side", k, a, dts[k], None if L is None else 2 * L)
    return s


def empty_particles(n: int, precision: int) -> dict:
    return {k: np.zeros(n, dt) for k, dt in particle_dtypes(precision).items()}


def empty_links(L: int, precision: int) -> dict:
    out = {}
    for k, dt in link_dtypes(precision).items():
        out[k] = np.zeros(2 * L if k in SIDE_FIELDS else L, dt)
    return out


def empty_particles_torch(n: int, precision: int, device) -> dict:
    """Particle fields as torch tensors on `device` (readback targets that stay there)."""
    import torch
    return {k: torch.empty(n, dtype=getattr(torch, np.dtype(dt).name), device=device)
            for k, dt in particle_dtypes(precision).items()}


def empty_links_torch(L: int, precision: int, device) -> dict:
    import torch
    return {k: torch.empty(2 * L if k in SIDE_FIELDS else L, dtype=getattr(torch, np.dtype(dt).name),
                           device=device)
            for k, dt in link_dtypes(precision).items()}


_lib = None

class HidemMap2d(C.Structure):
    _fields_ = [("data", C.c_void_p), ("x_points", C.c_int32), ("y_points", C.c_int32),
                ("x_min", C.c_float), ("y_min", C.c_float), ("x_max", C.c_float), ("y_max", C.c_float)]


def map2d(values, x_min: float, y_min: float, x_max: float, y_max: float, precision: int):
    """A hidem_map2d over `values` [y_points][x_points] (x fastest) in the lp type of
    `precision`; returns (struct, array) — keep the array alive while the struct is used."""
    arr = np.ascontiguousarray(values, dtype=lp_dtype(precision))
    m = HidemMap2d(arr.ctypes.data, arr.shape[1], arr.shape[0], x_min, y_min, x_max, y_max)
    return m, arr


class HidemMesh(C.Structure):
    _fields_ = [("x_vertex", C.c_void_p), ("y_vertex", C.c_void_p), ("z_vertex", C.c_void_p),
                ("x_normal", C.c_void_p), ("y_normal", C.c_void_p), ("z_normal", C.c_void_p),
                ("triangles", C.c_int32), ("cell_size", C.c_double), ("mesh_force", C.c_double),
                ("mesh_drag", C.c_double)]


def mesh(vertices, normals, cell_size: float, precision: int, mesh_force: float = 1e7,
         mesh_drag: float = 1000.0):
    """A hidem_mesh over `vertices` [triangles][3][3] (triangle, vertex, xyz) and `normals`
    [triangles][3] in the lp type of `precision`; returns (struct, arrays) — keep the
    arrays alive while the struct is used."""
    lp = lp_dtype(precision)
    v = np.asarray(vertices, np.float64).reshape(-1, 3, 3)
    nrm = np.asarray(normals, np.float64).reshape(-1, 3)
    arrs = [np.ascontiguousarray(v[:, :, k].ravel(), dtype=lp) for k in range(3)]
    arrs += [np.ascontiguousarray(nrm[:, k], dtype=lp) for k in range(3)]
    m = HidemMesh(*[a.ctypes.data for a in arrs], v.shape[0], cell_size, mesh_force, mesh_drag)
    return m, arrs


class HidemFunctorParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "neigh_invDt", "neigh_attractDistance", "neigh_attractScaleForce", "neigh_damping",
        "neigh_dampingRotation", "neigh_scaleE", "link_invDt", "link_damping", "link_dampingRotation",
        "link_E", "link_W2", "link_W4", "link_G", "break_bendBreak", "break_maxLoad")]


class HidemSurrogateConfig(C.Structure):
    _fields_ = [("hidden_layers", C.c_int32), ("width", C.c_int32), ("fourier_bands", C.c_int32),
                ("batch", C.c_int32), ("learning_rate", C.c_double), ("seed", C.c_uint64),
                ("inputs", C.c_int32), ("cosine_decay", C.c_int32)]


# (name, restype, argtypes)
_PROTOS = [
    ("hidem_abi_version", C.c_int, []),
    ("hidem_create_error", C.c_char_p, []),
    ("hidem_params_default", None, [C.POINTER(HidemParams)]),
    ("hidem_create", C.c_int, [C.POINTER(HidemParams), C.c_int, C.POINTER(C.c_void_p)]),
    ("hidem_destroy", None, [C.c_void_p]),
    ("hidem_last_error", C.c_char_p, [C.c_void_p]),
    ("hidem_set_particles", C.c_int, [C.c_void_p, C.POINTER(HidemParticleSoA), _i64]),
    ("hidem_set_links", C.c_int, [C.c_void_p, C.POINTER(HidemLinkSoA), _i64]),
    ("hidem_set_timestep", C.c_int, [C.c_void_p, _i64]),
    ("hidem_set_params", C.c_int, [C.c_void_p, C.POINTER(HidemParams)]),
    ("hidem_grid_service", C.c_int, [C.c_void_p]),
    ("hidem_regenerate", C.c_int, [C.c_void_p]),
    ("hidem_compute_forces", C.c_int, [C.c_void_p]),
    ("hidem_integrate", C.c_int, [C.c_void_p]),
    ("hidem_link_update", C.c_int, [C.c_void_p]),
    ("hidem_finalize_ts", C.c_int, [C.c_void_p]),
    ("hidem_step", C.c_int, [C.c_void_p, C.c_int32]),
    ("hidem_grid_service_local", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_i32)]),
    ("hidem_grid_service_decide", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_i32)]),
    ("hidem_local_bounds", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hidem_regenerate_frame", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hidem_set_halo_exchange", C.c_int, [C.c_void_p, C.c_void_p, _i64, C.c_void_p, _i64]),
    ("hidem_pack_halo_forces", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_unpack_halo_forces", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_synchronize", C.c_int, [C.c_void_p]),
    ("hidem_get_stream", C.c_void_p, [C.c_void_p]),
    ("hidem_profile", C.c_int, [C.c_void_p, C.c_int32]),
    ("hidem_profile_read", C.c_int, [C.c_void_p, C.POINTER(_d), C.POINTER(_i64)]),
    ("hidem_get_particles", C.c_int, [C.c_void_p, C.POINTER(HidemParticleSoA)]),
    ("hidem_get_links", C.c_int, [C.c_void_p, C.POINTER(HidemLinkSoA)]),
    ("hidem_get_forces", C.c_int, [C.c_void_p, C.c_void_p * 6]),
    ("hidem_get_cells", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(_i64), C.POINTER(_d)]),
    ("hidem_get_neighbours", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _i64,
                                       C.POINTER(_i64)]),
    ("hidem_get_break_events", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _i64,
                                         C.POINTER(_i64)]),
    ("hidem_get_stats", C.c_int, [C.c_void_p, C.POINTER(HidemStats)]),
    ("hidem_set_bed_maps", C.c_int, [C.c_void_p, C.POINTER(HidemMap2d), C.POINTER(HidemMap2d)]),
    ("hidem_set_external_force_maps", C.c_int, [C.c_void_p, C.POINTER(HidemMap2d)]),
    ("hidem_kinetic_energy", C.c_int, [C.c_void_p, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d)]),
    ("hidem_momentum", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hidem_set_functor_params", C.c_int, [C.c_void_p, C.POINTER(HidemFunctorParams)]),
    ("hidem_get_functor_params", C.c_int, [C.c_void_p, C.POINTER(HidemFunctorParams)]),
    ("hidem_set_collision_mesh", C.c_int, [C.c_void_p, C.POINTER(HidemMesh)]),
    ("hidem_get_mesh_face_forces", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hidem_zero_mesh_face_forces", C.c_int, [C.c_void_p]),
    ("hidem_get_mesh_accel", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, _i64, C.POINTER(_i64)]),
    ("hidem_set_step_kernel", C.c_int, [C.c_void_p, _i32]),
    ("hidem_set_checks", C.c_int, [C.c_void_p, _i32]),
    ("hidem_get_step_kernel", _i32, [C.c_void_p]),
    ("hidem_batch_create", C.c_int, [C.POINTER(C.c_void_p), _i32, _i32, C.POINTER(C.c_void_p)]),
    ("hidem_batch_destroy", None, [C.c_void_p]),
    ("hidem_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("hidem_batch_step", C.c_int, [C.c_void_p, _i32]),
    ("hidem_batch_get_stream", C.c_void_p, [C.c_void_p]),
    ("hidem_batch_counts", C.c_int, [C.c_void_p, C.POINTER(_i64), C.POINTER(_i64),
                                     C.POINTER(_i64)]),
    ("hidem_surrogate_config_default", None, [C.POINTER(HidemSurrogateConfig)]),
    ("hidem_surrogate_predict_device", C.c_int, [C.c_void_p, C.c_void_p, _i64, C.c_void_p]),
    ("hidem_surrogate_get_stream", C.c_void_p, [C.c_void_p]),
    ("hidem_surrogate_set_forward", C.c_int, [C.c_void_p, _i32]),
    ("hidem_surrogate_create", C.c_int, [C.POINTER(HidemSurrogateConfig), C.c_int,
                                         C.POINTER(C.c_void_p)]),
    ("hidem_surrogate_destroy", None, [C.c_void_p]),
    ("hidem_surrogate_last_error", C.c_char_p, [C.c_void_p]),
    ("hidem_surrogate_num_params", _i64, [C.c_void_p]),
    ("hidem_surrogate_get_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_surrogate_set_params", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_surrogate_set_data", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _i64]),
    ("hidem_surrogate_train", C.c_int, [C.c_void_p, _i32, C.POINTER(_d)]),
    ("hidem_surrogate_predict", C.c_int, [C.c_void_p, C.c_void_p, _i64, C.c_void_p]),
    ("hidem_surrogate_gradients", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _i64, C.c_void_p,
                                            C.POINTER(_d)]),
    ("hidem_bin_cells_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _i64, _d,
                                          C.c_void_p, C.c_void_p, C.POINTER(_i64), C.POINTER(_d),
                                          C.c_void_p]),
    ("hidem_params_from_toml", C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p),
                                         C.POINTER(HidemParams), C.POINTER(_i64)]),
    ("hidem_checkpoint_write", C.c_int, [C.c_void_p, C.c_char_p]),
    ("hidem_checkpoint_read", C.c_int, [C.c_void_p, C.c_char_p]),
    ("hidem_lattice_fcc", C.c_int, [_i32, _i32, _i32, _d, _d, C.POINTER(_d), _d, C.c_uint64,
                                    _i32, C.POINTER(HidemParticleSoA)]),
    ("hidem_links_by_distance", C.c_int, [C.POINTER(HidemParticleSoA), _i64, _i32, _d,
                                          C.POINTER(HidemLinkSoA), _i64, C.POINTER(_i64)]),
    ("hidem_get_device_view", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_compute_forces_packed", C.c_int, [C.c_void_p, C.c_void_p]),
    ("hidem_read_particle_file", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                           C.c_char_p, _i32, C.POINTER(HidemParticleSoA), _i64,
                                           C.POINTER(_i64)]),
]

EXPORTED = [name for name, _, _ in _PROTOS]


def load():
    """Load the in-tree library (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: the CUDA path has no fallback; build it with "
            "`python -m hidem_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in _PROTOS:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class HidemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def default_params(**overrides) -> HidemParams:
    p = HidemParams()
    load().hidem_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        cur = getattr(p, k)
        if hasattr(cur, "__len__"):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(p, k, v)
    return p

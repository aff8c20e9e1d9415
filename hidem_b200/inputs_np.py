"""The synthetic workloads' inputs generated in numpy / scipy, without loading
``libhidem_b200.so``: the reference arm of the benchmark times the reference's own CPU path,
and its process must map none of this library's native code. Each function gives the same
arrays, bit for bit, as the library's generators (``hidem_lattice_fcc``,
``hidem_links_by_distance``, ``hidem_params_default``); a CPU test holds them equal.

* ``default_params``: the MeshBlock sample's defaults (HiDEM/MeshBlock/MainMeshBlock.cpp:
  69-102, HiDEMLib/HiDEMLib.h:714-750), as ``hidem_params_default`` sets them.
* ``fcc_particles``: FCC sites in z, y, x, site order; jitter U(-j, +j) per coordinate from
  the 64-bit Mersenne Twister (std::mt19937_64's published parameters), 53-bit uniforms.
* ``distance_links``: LinkGenerator's rule (PLiB/Generators/LinkGenerator.h:60-110): pairs
  with globalKey[p] < globalKey[q] and |x_q - x_p| <= (r_p + r_q) * scale (distance in double,
  radius sum and scale in lp), ordered by (end A index, end B index), initialLen the distance.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

SQRT2 = math.sqrt(2.0)

_DEFAULTS = dict(dt=0.0001, scale=1.0, E=1e9, beamWidth=0.6, damping=1000.0, dampingRotation=1000.0,
                 attractDistance=0.0, attractScaleForce=0.0, maxLoad=0.35, bendBreak=0.35,
                 breakTime=10.0, g=9.81, rhoIce=910.0, rhoWater=1030.0, waterLevel=0.0, airDrag=1.0,
                 waterDrag=10.0, bedDrag=1000.0, bedStiffness=2e8, bedInteract=2.0, maxVel=20.0,
                 maxRot=5.0, searchDistanceScale=1.4, gridRegenInterval=-1,
                 firstBalanceTimestep=2000, maxRadius=0.5, bedHeight=0.0, bedFriction=1.0,
                 precision=abi.PREC_MIXED)


def default_params(**overrides) -> abi.HidemParams:
    """hidem_params_default plus overrides, without the library (every other field zero)."""
    p = abi.HidemParams()
    for k, v in {**_DEFAULTS, **overrides}.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        cur = getattr(p, k)
        if hasattr(cur, "__len__"):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(p, k, v)
    return p


class Mt64:
    """std::mt19937_64 (the published MT19937-64 parameters), whole state blocks at a time."""

    N, M = 312, 156
    MAG = np.uint64(0xB5026F5AA96619E9)
    UPPER, LOWER = np.uint64(0xFFFFFFFF80000000), np.uint64(0x7FFFFFFF)

    def __init__(self, seed: int):
        mt = [0] * self.N
        mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, self.N):
            mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.mt = np.array(mt, dtype=np.uint64)

    def _twist(self):
        mt, N, M = self.mt, self.N, self.M
        one = np.uint64(1)

        def mix(cur, nxt):
            x = (cur & self.UPPER) | (nxt & self.LOWER)
            return (x >> one) ^ np.where((x & one) != 0, self.MAG, np.uint64(0))

        # i < N - M reads mt[i + M] before it is rewritten; later i read the rewritten front
        mt[: N - M] = mt[M:] ^ mix(mt[: N - M], mt[1: N - M + 1])
        mt[N - M: N - 1] = mt[: M - 1] ^ mix(mt[N - M: N - 1], mt[N - M + 1:])
        mt[N - 1] = mt[M - 1] ^ mix(mt[N - 1: N], mt[0:1])[0]

    def draws(self, count: int) -> np.ndarray:
        out = np.empty(((count + self.N - 1) // self.N) * self.N, np.uint64)
        for b in range(out.shape[0] // self.N):
            self._twist()
            out[b * self.N:(b + 1) * self.N] = self.mt
        x = out[:count]
        x ^= (x >> np.uint64(29)) & np.uint64(0x5555555555555555)
        x ^= (x << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000)
        x ^= (x << np.uint64(37)) & np.uint64(0xFFF7EEE000000000)
        x ^= x >> np.uint64(43)
        return x

    def uniforms(self, count: int) -> np.ndarray:
        return (self.draws(count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def fcc_particles(nx: int, ny: int, nz: int, precision: int, a: float = SQRT2, radius: float = 0.5,
                  origin=(0.0, 0.0, 0.0), jitter: float = 0.01, seed: int = 1) -> dict:
    n = 4 * nx * ny * nz
    p = abi.empty_particles(n, precision)
    site = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    k, j, c, s = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), np.arange(4), indexing="ij")
    idx = (c.ravel(), j.ravel(), k.ravel())
    s = s.ravel()
    xyz = [origin[q] + (idx[q] + site[s, q]) * a for q in range(3)]
    if jitter > 0:
        u = Mt64(seed).uniforms(3 * n).reshape(n, 3)
        for q in range(3):
            xyz[q] = xyz[q] + (-jitter + 2.0 * jitter * u[:, q])
    p["xCord"][:], p["yCord"][:], p["zCord"][:] = xyz
    p["radius"][:] = radius
    p["globalKeys"][:] = np.arange(n)
    return p


def distance_links(p: dict, precision: int, scale: float = 1.01) -> dict:
    from scipy.spatial import cKDTree
    mixed = precision == abi.PREC_MIXED
    lp = np.float32 if mixed else np.float64
    x, y, z = p["xCord"], p["yCord"], p["zCord"]
    r = p["radius"].astype(lp)
    keys = p["globalKeys"]
    dist_scale = float(np.float32(scale)) if mixed else float(scale)
    reach = 2.0 * float(r.max()) * dist_scale
    tree = cKDTree(np.stack([x, y, z], axis=1))
    pairs = tree.query_pairs(reach * (1.0 + 1e-9) + 1e-12, output_type="ndarray")
    a, b = pairs[:, 0], pairs[:, 1]
    swap = keys[a] > keys[b]
    i = np.where(swap, b, a)
    q = np.where(swap, a, b)
    xd = x[q] - x[i]
    yd = y[q] - y[i]
    zd = z[q] - z[i]
    dist = np.sqrt((xd * xd) + (yd * yd) + (zd * zd))
    rsum = (r[q] + r[i]).astype(np.float64)
    keep = ~(dist > rsum * dist_scale)
    i, q, dist = i[keep], q[keep], dist[keep]
    order = np.lexsort((q, i))
    i, q, dist = i[order], q[order], dist[order]
    L = i.shape[0]
    links = abi.empty_links(L, precision)
    links["globalKeyEndA"][:] = keys[i]
    links["globalKeyEndB"][:] = keys[q]
    first = np.ones(L, bool)
    first[1:] = i[1:] != i[:-1]
    starts = np.flatnonzero(first)
    rank = np.arange(L) - np.repeat(starts, np.diff(np.append(starts, L)))
    links["particleLinkNum"][:] = rank
    links["globalKeys"][:] = keys[i] * 256 + rank
    links["state"][:] = 1
    links["initialLen"][:] = dist.astype(lp)
    return links


def calving_slab(size=(400.0, 100.0, 100.0), precision: int = abi.PREC_MIXED, seed: int = 7,
                 jitter: float = 0.01, broken_fraction: float = 0.01, water_level: float = 90.0):
    """The calving slab of ``workloads.calving_slab`` (FCC slab on a flat bed, calving front on
    the x-max face, a seeded fraction of links pre-broken), built without the library."""
    from .workloads import slab_params_overrides
    nx, ny, nz = (max(1, int(round(s / SQRT2))) for s in size)
    p = fcc_particles(nx, ny, nz, precision, jitter=jitter, seed=seed)
    xmax = p["xCord"].max()
    p["type"][p["xCord"] > xmax - 0.25 * SQRT2] |= abi.TYPE_FRONT
    links = distance_links(p, precision, 1.01)
    rng = np.random.default_rng(seed)
    L = links["state"].shape[0]
    k = int(round(broken_fraction * L))
    if k:
        links["state"][rng.choice(L, size=k, replace=False)] = 0
    params = default_params(**slab_params_overrides(precision, water_level, float(p["zCord"].min())))
    return params, p, links

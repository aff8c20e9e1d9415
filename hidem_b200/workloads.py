"""Synthetic workloads: FCC ice blocks and slabs with distance-rule links.

Seeded FCC lattices with the density, particle size and link rule of the reference's
MeshBlock benchmark inputs stand in for its HDF5 point files in the named configurations.
Generation runs in the library's host code (``hidem_lattice_fcc``,
``hidem_links_by_distance``); ``inputs_np`` restates it in numpy for processes that must not
load the library.

Parameter mapping of the named configurations (the reference keys they set):
  d = 1 m, a = sqrt(2) d            lattice.particleRadius = 0.5, fccSpacing = sqrt(2)
  bonds within 1.01 d               lattice.linkGenScale = 1.01 (PLiB/Generators/LinkGenerator.h:83-89)
  E 1e9, rho 910, g 9.81            general.E / rhoIce / g
  strain threshold 5e-4             general.maxLoad = 5e-4, bendBreak = 0.01, breakTime = 0
  repulsion below d                 general.attractDistance = 0, attractScaleForce = 0
  velocity damping 1e-3             general.damping = dampingRotation = 1e-3 * m / dt = 9100
  friction coefficient 0.3          bed friction 0.3 in the GlacierDem bed drag (slab only)
  cell size 1.2 d                   grid.searchDistanceScale = 1.2
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi

SQRT2 = math.sqrt(2.0)


def fcc_particles(nx: int, ny: int, nz: int, precision: int, a: float = SQRT2, radius: float = 0.5,
                  origin=(0.0, 0.0, 0.0), jitter: float = 0.01, seed: int = 1) -> dict:
    lib = abi.load()
    n = 4 * nx * ny * nz
    p = abi.empty_particles(n, precision)
    soa = abi.particle_soa(p, precision, n)
    org = (C.c_double * 3)(*origin)
    st = lib.hidem_lattice_fcc(nx, ny, nz, a, radius, org, jitter, seed, precision, C.byref(soa))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, "hidem_lattice_fcc failed")
    return p


def distance_links(p: dict, precision: int, scale: float = 1.01, lean: bool = False) -> dict:
    """Links of all pairs within scale * (r_i + r_j). lean: only the fields hidem_set_links
    needs (ends, state, initial length; the CT history starts at zero), for large sets."""
    lib = abi.load()
    n = p["xCord"].shape[0]
    soa = abi.particle_soa(p, precision, n)
    cnt = C.c_int64()
    st = lib.hidem_links_by_distance(C.byref(soa), n, precision, scale, None, 0, C.byref(cnt))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, "hidem_links_by_distance (count) failed")
    L = cnt.value
    if lean:
        dts = abi.link_dtypes(precision)
        links = {k: np.zeros(L, dts[k]) for k in ("globalKeyEndA", "globalKeyEndB", "state", "initialLen")}
    else:
        links = abi.empty_links(L, precision)
    lsoa = abi.link_soa(links, precision, L)
    st = lib.hidem_links_by_distance(C.byref(soa), n, precision, scale, C.byref(lsoa), L,
                                     C.byref(cnt))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, "hidem_links_by_distance failed")
    return links


def read_particle_file(path: str, precision: int, names=(None, None, None, None)) -> dict:
    """The reference's File lattice (hidem_read_particle_file; FileParticleGenerator,
    PLiB/Generators/FileParticleGenerator.h:23-105): particles from an HDF5 point file."""
    lib = abi.load()
    enc = [n.encode() if n else None for n in names]
    cnt = C.c_int64()
    st = lib.hidem_read_particle_file(str(path).encode(), *enc, precision, None, 0, C.byref(cnt))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, lib.hidem_create_error().decode())
    n = cnt.value
    p = abi.empty_particles(n, precision)
    soa = abi.particle_soa(p, precision, n)
    st = lib.hidem_read_particle_file(str(path).encode(), *enc, precision, C.byref(soa), n, C.byref(cnt))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, lib.hidem_create_error().decode())
    return p


def meshblock(config_path: str, particle_file: str | None = None, precision: int | None = None):
    """The reference's MeshBlock benchmark input (HiDEM/Benchmark/<size>/config_mesh_<size>.toml
    with its particles.h5, the run every published number is quoted on): run parameters from
    the TOML file (the library's front-end), particles from the File lattice, links by the
    distance rule with lattice.linkGenScale (LinkGenerator, PLiB/Generators/LinkGenerator.h:
    60-110; every particle is of ice type 0, linkWith [0], probability 1). `particle_file`
    overrides lattice.path (which the reference resolves against its working directory).
    Returns (params, particles, links, run info)."""
    import tomllib
    from pathlib import Path
    from .config import params_from_toml
    over = [] if precision is None else [f"--general.precision={'mixed' if precision == abi.PREC_MIXED else 'fp64'}"]
    P, time_steps = params_from_toml(str(config_path), over)
    prec = int(P.precision)
    cfg = tomllib.loads(Path(config_path).read_text())
    lat = cfg.get("lattice", {})
    if lat.get("type") != "File":
        raise ValueError(f"{config_path}: lattice.type is {lat.get('type')!r}, not 'File'")
    path = particle_file or lat["path"]
    names = (lat.get("xCords"), lat.get("yCords"), lat.get("zCords"), lat.get("radius"))
    p = read_particle_file(path, prec, names)
    links = distance_links(p, prec, float(lat["linkGenScale"]))
    info = {"time_steps": time_steps, "linkGenScale": float(lat["linkGenScale"]),
            "statIntervals": cfg.get("output", {}).get("statIntervals"),
            "particle_file": str(path)}
    return P, p, links, info


def block_overrides(precision: int, **over) -> dict:
    """Material and contact parameters of the ice-block configurations, as overrides of
    the MeshBlock defaults."""
    dt = 1e-4
    mass = 910.0 * 1.0 ** 3
    base = dict(dt=dt, scale=1.0, E=1e9, rhoIce=910.0, g=9.81, maxLoad=5e-4, bendBreak=0.01,
                breakTime=0.0, attractDistance=0.0, attractScaleForce=0.0,
                damping=1e-3 * mass / dt, dampingRotation=1e-3 * mass / dt,
                searchDistanceScale=1.2, maxRadius=0.5, waterLevel=-1.0e3, precision=precision)
    base.update(over)
    return base


def block_params(precision: int, **over) -> abi.HidemParams:
    """Material and contact parameters of the ice-block configurations."""
    return abi.default_params(**block_overrides(precision, **over))


def slab_params_overrides(precision: int, water_level: float, zmin: float, **over) -> dict:
    """The calving slab's parameters: the block's, on a flat bed half a diameter below the
    lowest centres (bed friction 0.3), water line, front pressure."""
    return block_overrides(precision, waterLevel=water_level, useBed=1, bedHeight=zmin + 0.5,
                           bedFriction=0.3, useFrontPressure=1, **over)


def ice_block(cells=(20, 20, 20), precision: int = abi.PREC_MIXED, seed: int = 1,
              jitter: float = 0.01, fixed_bottom: bool = True, **param_over):
    """FCC block of cells^3 unit cells (config: 20x20x20 = 32,000 spheres), bonded within
    1.01 d, bottom layer fixed, in air. Returns (params, particles, links)."""
    nx, ny, nz = cells
    p = fcc_particles(nx, ny, nz, precision, jitter=jitter, seed=seed)
    if fixed_bottom:
        z0 = p["zCord"].min()
        p["type"][p["zCord"] < z0 + 0.25 * SQRT2] |= abi.TYPE_FIXED
    links = distance_links(p, precision, 1.01)
    params = block_params(precision, useFixed=1 if fixed_bottom else 0, **param_over)
    return params, p, links


def container_mesh(lo, hi, bed, nx: int = 8, ny: int = 8, walls=True):
    """A collision mesh shaped as an open container, the form the MeshConstrainedDem
    sample's mesh takes: the bed z = bed(x, y) over [lo[0], hi[0]] x [lo[1], hi[1]] as a
    triangulated grid of nx x ny quads (two triangles each), and with `walls` four vertical
    walls up to hi[2]. Normals point out of the container (down through the bed, out
    through the walls), so the mesh force, along minus the normal, pushes the particles
    inside back in. `walls`: True (all four), False, or the sides to build out of
    "x-", "x+", "y-", "y+". Returns (vertices [T][3][3], normals [T][3])."""
    xs = np.linspace(lo[0], hi[0], nx + 1)
    ys = np.linspace(lo[1], hi[1], ny + 1)
    tris = []
    for i in range(nx):
        for j in range(ny):
            p00 = (xs[i], ys[j], bed(xs[i], ys[j]))
            p10 = (xs[i + 1], ys[j], bed(xs[i + 1], ys[j]))
            p11 = (xs[i + 1], ys[j + 1], bed(xs[i + 1], ys[j + 1]))
            p01 = (xs[i], ys[j + 1], bed(xs[i], ys[j + 1]))
            tris += [(p00, p10, p11), (p00, p11, p01)]
    v = np.array(tris, np.float64)
    nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])  # upward for these windings
    nrm = -nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    if walls:
        zb = min(bed(x, y) for x in (lo[0], hi[0]) for y in (lo[1], hi[1])) - 1.0
        zt = hi[2]
        sides = {"x-", "x+", "y-", "y+"} if walls is True else set(walls)
        wall = []
        for x, nx_, side in ((lo[0], -1.0, "x-"), (hi[0], 1.0, "x+")):
            if side not in sides:
                continue
            a, b, c, d = (x, lo[1], zb), (x, hi[1], zb), (x, hi[1], zt), (x, lo[1], zt)
            wall += [((a, b, c), (nx_, 0.0, 0.0)), ((a, c, d), (nx_, 0.0, 0.0))]
        for y, ny_, side in ((lo[1], -1.0, "y-"), (hi[1], 1.0, "y+")):
            if side not in sides:
                continue
            a, b, c, d = (lo[0], y, zb), (hi[0], y, zb), (hi[0], y, zt), (lo[0], y, zt)
            wall += [((a, b, c), (0.0, ny_, 0.0)), ((a, c, d), (0.0, ny_, 0.0))]
        v = np.concatenate([v, np.array([w[0] for w in wall])])
        nrm = np.concatenate([nrm, np.array([w[1] for w in wall])])
    return v, nrm


def calving_slab(size=(400.0, 100.0, 100.0), precision: int = abi.PREC_MIXED, seed: int = 7,
                 jitter: float = 0.01, broken_fraction: float = 0.01, water_level: float = 90.0,
                 **param_over):
    """FCC slab on a flat bed with a calving front on the x-max face, water line at
    `water_level`, a seeded fraction of links pre-broken (config: 400 x 100 x 100 m,
    ~5.7M particles, ~34M links)."""
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
    zmin = float(p["zCord"].min())
    params = abi.default_params(**slab_params_overrides(precision, water_level, zmin, **param_over))
    return params, p, links


def slab_in_fjord(size=(400.0, 100.0, 100.0), precision: int = abi.PREC_MIXED, quad: float = 4.0,
                  mesh_force: float = 1e5, mesh_drag: float = 1000.0, **param_over):
    """The calving slab in a fjord-shaped collision mesh, the MeshConstrainedDem setting: a
    bed surface (gently sloping, quads of `quad` m, two triangles each) 0.55 m below the
    bottom layer's centres and side walls 0.55 m from the x-min, y-min and y-max faces,
    open at the calving front (x-max); bed interaction distance 0.25 m, MeshAccel cells of
    16 maxRadius (the sample's choice). Returns (params, particles, links, mesh dict with
    vertices, normals, cell_size, mesh_force, mesh_drag)."""
    P, p, l = calving_slab(size=size, precision=precision, bedInteract=0.25, **param_over)
    x, y, z = p["xCord"], p["yCord"], p["zCord"]
    lo = (float(x.min()) - 0.55, float(y.min()) - 0.55)
    hi = (float(x.max()) + 0.55, float(y.max()) + 0.55, float(z.max()) + 5.0)
    z0 = float(z.min()) - 0.55

    def bed(xx, yy):
        return z0 - 0.002 * (xx - lo[0])

    nx = max(1, int(round((hi[0] - lo[0]) / quad)))
    ny = max(1, int(round((hi[1] - lo[1]) / quad)))
    v, nrm = container_mesh(lo, hi, bed, nx, ny, walls=("x-", "y-", "y+"))
    return P, p, l, {"vertices": v, "normals": nrm, "cell_size": 16.0 * float(P.maxRadius),
                     "mesh_force": mesh_force, "mesh_drag": mesh_drag}


def algorithmic_bytes(n: int, L: int, pairs: int, precision: int) -> dict:
    """Bytes per timestep of the byte model of the hot path: each particle's own fields
    once, partner reads as cache hits (sp = 8, lp = ct = 4 mixed / 8 fp64):
        N*(3sp+6lp+lp+6lp) force + N*(3sp+3lp+6lp+6lp+lp + 3sp+3lp+6lp) integrate
        + S*(12ct+8) link ends + L*(2+lp+8) link break + C*4 contact list."""
    sp = 8
    lp = 4 if precision == abi.PREC_MIXED else 8
    S = 2 * L
    force = n * (3 * sp + 6 * lp + lp + 6 * lp)
    integ = n * (3 * sp + 3 * lp + 6 * lp + 6 * lp + lp + 3 * sp + 3 * lp + 6 * lp)
    sides = S * (12 * lp + 8)
    brk = L * (2 + lp + 8)
    pair = pairs * 4
    total = force + integ + sides + brk + pair
    return dict(force=force, integrate=integ, sides=sides, link_break=brk, pairs=pair, total=total)


def ensemble_sizes(count: int = 256, n_min: int = 5000, n_max: int = 80000, seed: int = 11):
    """Cube edges (unit cells) and per-block maxLoad of the batched ensemble: particle
    counts drawn log-uniform from [n_min, n_max] and rounded to whole FCC unit cells
    (4 particles each), fracture strain threshold lognormal with median 5e-4, sigma 0.3."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=count))
    edges = np.maximum(1, np.rint(np.cbrt(n / 4.0))).astype(int)
    max_load = 5e-4 * np.exp(0.3 * rng.standard_normal(count))
    return edges, max_load


def ensemble(count: int = 256, precision: int = abi.PREC_MIXED, seed: int = 11,
             n_min: int = 5000, n_max: int = 80000):
    """Independent FCC ice blocks of uneven sizes (config: 256 blocks, 5k-80k particles
    log-uniform, per-block maxLoad lognormal(5e-4, 0.3), per-block jitter seed, other
    parameters as the 20^3 ice block). Returns a list of (params, particles, links)."""
    edges, max_load = ensemble_sizes(count, n_min, n_max, seed)
    out = []
    for i, (e, ml) in enumerate(zip(edges, max_load)):
        out.append(ice_block((int(e),) * 3, precision, seed=seed * 100003 + i, maxLoad=float(ml)))
    return out


def ensemble_shard(sizes, world: int, rank: int) -> list[int]:
    """Blocks of rank `rank` out of `world` (no data exchange between ranks): largest block
    first, each to the rank with the fewest particles so far (ties to the lower rank)."""
    load = [0] * world
    mine = []
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += int(sizes[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def bed_modes(seed: int, size, amplitude: float, count: int = 8):
    """Bed heightfield of `count` seeded Fourier modes over a plan of `size` (x, y), total
    amplitude at most `amplitude`: a function of (x, y)."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 1.0, count)
    amp *= amplitude / max(amp.sum(), 1e-12)
    kx = rng.integers(0, 5, count)
    ky = rng.integers(0, 3, count)
    kx[(kx == 0) & (ky == 0)] = 1
    ph = rng.uniform(0, 2 * math.pi, count)

    def height(x, y):
        out = np.zeros(np.broadcast(x, y).shape)
        for a, i, j, p in zip(amp, kx, ky, ph):
            out += a * np.cos(2 * math.pi * (i * x / size[0] + j * y / size[1]) + p)
        return out
    return height


def slab_on_bed(size=(1200.0, 200.0, 150.0), precision: int = abi.PREC_MIXED, seed: int = 13,
                amplitude: float = 15.0, water_level: float = 135.0, broken_fraction: float = 0.01,
                map_resolution: float = 5.0):
    """FCC slab of `size` whose base follows a bed of 8 seeded Fourier modes (config: 1200 x
    200 x 150 m, ~50M particles, bed amplitude <= 15 m, water line 135 m), calving front
    on the x-max face, a seeded fraction of links pre-broken; the bed enters the integrate
    step as a GlacierDem bed map. Returns (params, particles, links, bed map values
    [ny][nx], map extents (x_min, y_min, x_max, y_max))."""
    bed = bed_modes(seed, size[:2], amplitude)
    nx, ny = (max(1, int(round(s / SQRT2))) for s in size[:2])
    nz = max(1, int(math.ceil((size[2] + 2 * amplitude) / SQRT2)))
    p = fcc_particles(nx, ny, nz, precision, origin=(0.0, 0.0, -amplitude), jitter=0.0, seed=seed)
    b = bed(p["xCord"], p["yCord"])
    keep = (p["zCord"] >= b + 0.5) & (p["zCord"] <= b + size[2])
    p = {k: np.ascontiguousarray(v[keep]) for k, v in p.items()}
    p["globalKeys"][:] = np.arange(p["xCord"].shape[0])
    xmax = p["xCord"].max()
    p["type"][p["xCord"] > xmax - 0.25 * SQRT2] |= abi.TYPE_FRONT
    links = distance_links(p, precision, 1.01, lean=True)
    rng = np.random.default_rng(seed)
    L = links["state"].shape[0]
    k = int(round(broken_fraction * L))
    if k:
        links["state"][rng.choice(L, size=k, replace=False)] = 0
    ext = (-5.0, -5.0, size[0] + 5.0, size[1] + 5.0)
    mx = int(round((ext[2] - ext[0]) / map_resolution)) + 1
    my = int(round((ext[3] - ext[1]) / map_resolution)) + 1
    X, Y = np.meshgrid(np.linspace(ext[0], ext[2], mx), np.linspace(ext[1], ext[3], my))
    params = block_params(precision, waterLevel=water_level, useBed=1, bedHeight=0.0,
                          bedFriction=0.3, useFrontPressure=1)
    return params, p, links, bed(X, Y), ext

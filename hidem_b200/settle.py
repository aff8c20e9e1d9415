"""Settling runs and the learned warm start.

Glacier tongues (config: 64 tongues of 200 m x 60 m in plan, bed and surface heightfields
each a sum of 8 seeded Fourier modes of amplitude at most 10 m in total, filled with an
FCC lattice at d = 1 m) settle under gravity and buoyancy with the plain method until the
kinetic energy per particle stays below a tolerance. The cold start begins from the
undeformed lattice at rest; the warm start applies the surrogate's predicted settled
displacement first (to the positions and, as one increment, to the link ends' CT state:
see warm_state). The plain method judges both: the same step loop,
the same convergence test, and the displacement error of the warm-settled state against
the cold-settled one.

Choices the configuration leaves open, fixed here: the bottom lattice layer (within 1 m of
the bed) is held fixed (the ice frozen to its bed), the water line is half the base
thickness above the mean bed (6 m for the configuration's tongues), link
breaking is off during settling (the surrogate learns the elastic settled state), and
convergence means the kinetic energy per particle stayed below the tolerance at every
check (every `check` steps) of the last `window` steps.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import abi, workloads
from .hidemlib import HiDEMLib

Z_SCALE = 20.0
THICK_SCALE = 15.0
BED_SCALE = 10.0
DISP_SCALE = 1e-4   # metres per unit of the surrogate's output


@dataclass
class Tongue:
    params: abi.HidemParams
    particles: dict
    links: dict
    size: tuple[float, float]
    bed: np.ndarray        # bed height under each particle
    thick: np.ndarray      # ice thickness under each particle
    seed: int
    bed_modes: tuple = ()   # the heightfields as Fourier modes (amplitude, kx, ky, phase)
    surf_modes: tuple = ()
    base_thickness: float = 0.0

    def bed_at(self, x, y):
        return _field(np.asarray(x, np.float64), np.asarray(y, np.float64), self.size, self.bed_modes)

    def thickness_at(self, x, y):
        """ice thickness of the heightfields at (x, y); 0 outside the tongue's plan"""
        x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
        th = np.maximum(3.0, self.base_thickness + 0.5 * _field(x, y, self.size, self.surf_modes))
        inside = (x >= 0) & (x <= self.size[0]) & (y >= 0) & (y <= self.size[1])
        return np.where(inside, th, 0.0)


def _modes(rng, count: int, total_amp: float):
    amp = rng.uniform(0.0, 1.0, count)
    amp *= total_amp / max(amp.sum(), 1e-12)
    kx = rng.integers(0, 4, count)
    ky = rng.integers(0, 3, count)
    kx[(kx == 0) & (ky == 0)] = 1
    ph = rng.uniform(0, 2 * math.pi, count)
    return amp, kx, ky, ph


def _field(x, y, size, modes):
    amp, kx, ky, ph = modes
    out = np.zeros_like(x, dtype=np.float64)
    for a, i, j, p in zip(amp, kx, ky, ph):
        out += a * np.cos(2 * math.pi * (i * x / size[0] + j * y / size[1]) + p)
    return out


def glacier_tongue(seed: int, size=(200.0, 60.0), base_thickness: float = 12.0,
                   precision: int = abi.PREC_MIXED, amplitude: float = 10.0,
                   water_level: float | None = None) -> Tongue:
    """FCC tongue between a bed and a surface heightfield (8 Fourier modes each); the
    water line defaults to half the base thickness above the mean bed (z = 0)."""
    rng = np.random.default_rng(seed)
    bed_m = _modes(rng, 8, amplitude)
    surf_m = _modes(rng, 8, amplitude)
    zlo = -amplitude - 1.0
    zhi = amplitude + base_thickness + amplitude + 1.0
    nx = max(1, int(math.ceil(size[0] / workloads.SQRT2)))
    ny = max(1, int(math.ceil(size[1] / workloads.SQRT2)))
    nz = max(1, int(math.ceil((zhi - zlo) / workloads.SQRT2)))
    p = workloads.fcc_particles(nx, ny, nz, precision, origin=(0.0, 0.0, zlo), jitter=0.0, seed=seed)
    x, y, z = p["xCord"], p["yCord"], p["zCord"]
    bed = _field(x, y, size, bed_m)
    thick = np.maximum(3.0, base_thickness + 0.5 * _field(x, y, size, surf_m))
    keep = (x <= size[0]) & (y <= size[1]) & (z >= bed) & (z <= bed + thick)
    p = {k: np.ascontiguousarray(v[keep]) for k, v in p.items()}
    p["globalKeys"][:] = np.arange(p["xCord"].shape[0])
    bed, thick = bed[keep], thick[keep]
    p["type"][p["zCord"] < bed + 1.0] |= abi.TYPE_FIXED
    links = workloads.distance_links(p, precision, 1.01)
    wl = 0.5 * base_thickness if water_level is None else water_level
    params = workloads.block_params(precision, useFixed=1, waterLevel=wl, breakTime=1e30)
    return Tongue(params, p, links, size, bed, thick, seed, bed_m, surf_m, base_thickness)


def surrogate_inputs(t: Tongue) -> np.ndarray:
    """The 5 normalised inputs of every particle of a tongue: x and y across the plan,
    the height z expressed in its ice column (0 at the bed, 1 at the surface, mapped to
    [-1, 1]), the local thickness and the bed height."""
    p = t.particles
    zrel = (p["zCord"] - t.bed) / t.thick
    return np.stack([2 * p["xCord"] / t.size[0] - 1, 2 * p["yCord"] / t.size[1] - 1,
                     2 * zrel - 1, t.thick / THICK_SCALE - 1, t.bed / BED_SCALE],
                    axis=1).astype(np.float32)


# geometry sampled around each particle: thickness and bed at x +- d, y +- d
LATTICE_OFFSETS = (1.5, 3.0, 6.0)
# surrounding lattice columns (column spacing: half the FCC cell), rings 1 and 2
LATTICE_COLUMNS = tuple((i, j) for i in range(-2, 3) for j in range(-2, 3) if (i, j) != (0, 0))
N_LATTICE_INPUTS = 5 + 8 * len(LATTICE_OFFSETS) + 5 + 2 * len(LATTICE_COLUMNS)


def n_lattice_inputs(offsets=LATTICE_OFFSETS) -> int:
    return 5 + 8 * len(offsets) + 5 + 2 * len(LATTICE_COLUMNS)


def lattice_inputs(t: Tongue, mirror: tuple[int, int] = (1, 1), offsets=LATTICE_OFFSETS) -> np.ndarray:
    """The surrogate's lattice-neighbourhood inputs of every particle (N_LATTICE_INPUTS
    columns), optionally of the tongue's mirror image (x -> Lx - x for mirror[0] = -1,
    y -> Ly - y for mirror[1] = -1, the particles keeping their order):

    * the 5 coordinate inputs of surrogate_inputs;
    * ice thickness (0 outside the plan) and bed height at x +- d and y +- d for each d of
      `offsets` (LATTICE_OFFSETS by default; d-major, then the axis, then +d before -d);
    * the particle's lattice column (particles sharing x and y): its bond count, the
      particles above it, the free particles below it, and its height below the column's
      top and above the column's lowest free particle;
    * for each surrounding column of LATTICE_COLUMNS: the height of that column's top and
      of its lowest free particle relative to the particle (-2 where there is no column).

    The settled displacement of these coarse lattices depends on the discrete layering
    of the ice around a particle, which the smooth heightfields alone do not describe."""
    p = t.particles
    n = p["xCord"].shape[0]
    sx, sy = mirror
    x = p["xCord"] if sx > 0 else t.size[0] - p["xCord"]
    y = p["yCord"] if sy > 0 else t.size[1] - p["yCord"]
    z = p["zCord"]

    def geo(xx, yy):  # heightfields at mirror-frame points
        ox = xx if sx > 0 else t.size[0] - xx
        oy = yy if sy > 0 else t.size[1] - yy
        return t.thickness_at(ox, oy), t.bed_at(ox, oy)

    cols = [2 * x / t.size[0] - 1, 2 * y / t.size[1] - 1, 2 * (z - t.bed) / t.thick - 1,
            t.thick / THICK_SCALE - 1, t.bed / BED_SCALE]
    for d in offsets:
        for ax in (0, 1):
            for sgn in (1, -1):
                th, bd = geo(x + sgn * d, y) if ax == 0 else geo(x, y + sgn * d)
                cols += [th / THICK_SCALE - 1, bd / BED_SCALE]
    # bonds per particle
    keys = np.asarray(p["globalKeys"])
    korder = np.argsort(keys, kind="stable")
    ends = [korder[np.searchsorted(keys, np.asarray(t.links[k]), sorter=korder)]
            for k in ("globalKeyEndA", "globalKeyEndB")]
    deg = np.bincount(ends[0], minlength=n) + np.bincount(ends[1], minlength=n)
    # lattice columns
    h = workloads.SQRT2 / 2
    ci = np.rint(x / h).astype(np.int64) + 16
    cj = np.rint(y / h).astype(np.int64) + 16
    key = ci * 4096 + cj
    free = (p["type"] & abi.TYPE_FIXED) == 0
    order = np.lexsort((z, key))
    ks, zs, fs = key[order], z[order], free[order].astype(np.int64)
    start = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    size = np.diff(np.r_[start, n])
    g = np.repeat(np.arange(start.shape[0]), size)
    rank = np.arange(n) - start[g]
    above, below, gid = np.empty(n), np.empty(n), np.empty(n, np.int64)
    above[order] = size[g] - 1 - rank
    cum = np.cumsum(fs) - fs
    below[order] = cum - cum[start[g]]
    gid[order] = g
    top = zs[start + size - 1]
    zf = np.where(fs > 0, zs, np.inf)
    low_free = np.minimum.reduceat(zf, start)
    has_free = np.isfinite(low_free)
    lowest = np.where(has_free, low_free, zs[start])
    cols += [deg / 6.0 - 1, above / 5.0 - 1, below / 5.0 - 1, (top[gid] - z) / 5.0 - 1,
             (z - lowest[gid]) / 5.0 - 1]
    ukeys = ks[start]
    low_or_top = np.where(has_free, low_free, top)
    for di, dj in LATTICE_COLUMNS:
        nk = key + di * 4096 + dj
        q = np.minimum(np.searchsorted(ukeys, nk), ukeys.shape[0] - 1)
        ex = ukeys[q] == nk
        cols.append(np.where(ex, (top[q] - z) / 5.0, -2.0))
        cols.append(np.where(ex, (low_or_top[q] - z) / 5.0, -2.0))
    out = np.stack(cols, axis=1).astype(np.float32)
    assert out.shape[1] == n_lattice_inputs(offsets)
    return out


def rotation_from_displacement(t: Tongue, disp: np.ndarray) -> np.ndarray:
    """Small-strain rotation of each particle from a least-squares displacement gradient
    over the particle's bonded neighbours: minus half the curl of the displacement field,
    the sign convention of the particles' xTheta..zTheta in this model (a test compares
    it with settled states)."""
    p, l = t.particles, t.links
    idx = {int(k): i for i, k in enumerate(p["globalKeys"])}
    a = np.array([idx[int(k)] for k in l["globalKeyEndA"]])
    b = np.array([idx[int(k)] for k in l["globalKeyEndB"]])
    x = np.stack([p["xCord"], p["yCord"], p["zCord"]], axis=1)
    n = x.shape[0]
    dx = x[b] - x[a]
    du = disp[b] - disp[a]
    M = np.zeros((n, 3, 3))
    R = np.zeros((n, 3, 3))
    outer_xx = dx[:, :, None] * dx[:, None, :]
    outer_ux = du[:, :, None] * dx[:, None, :]
    for e in (a, b):
        np.add.at(M, e, outer_xx)
        np.add.at(R, e, outer_ux)
    ev = np.linalg.eigvalsh(M)
    good = ev[:, 0] > 0.05 * ev[:, 2]  # bonded neighbours span all three directions
    M[~good] += np.eye(3)
    G = np.einsum("nij,njk->nik", R, np.linalg.inv(M))  # G[i][j] = d u_i / d x_j
    rot = -0.5 * np.stack([G[:, 2, 1] - G[:, 1, 2], G[:, 0, 2] - G[:, 2, 0], G[:, 1, 0] - G[:, 0, 1]], axis=1)
    # particles whose bonds are (nearly) planar or linear take the mean of their bonded
    # neighbours with a full estimate
    acc = np.zeros((n, 3))
    cnt = np.zeros(n)
    for e, o in ((a, b), (b, a)):
        w = good[o].astype(np.float64)
        np.add.at(acc, e, rot[o] * w[:, None])
        np.add.at(cnt, e, w)
    bad = ~good
    rot[bad] = np.where(cnt[bad, None] > 0, acc[bad] / np.maximum(cnt[bad, None], 1), 0.0)
    return rot


@dataclass
class SettleResult:
    steps: int             # steps until converged (or the cap)
    converged: bool
    final: dict            # particle state at the end
    ke_trace: list         # (step, kinetic energy per particle)
    final_links: dict      # link state (CT) at the end


def warm_state(t: Tongue, displacement: np.ndarray, rotation: np.ndarray | None = None):
    """Particle and link state of a warm start. The beam forces of the reference's model
    are incremental (CT accumulates K * B of each step's relative increments,
    HiDEMDefaultFunctions.h:170-204), so moving particles alone leaves the links
    unstressed. The predicted displacement (and rotation, when given) is therefore first
    applied as one increment — the particles' diffs set to it and one force evaluation
    (hidem_compute_forces) run, which adds K * B(displacement) to every link end's CT —
    and then to the positions, with the diffs back at zero (the particles at rest)."""
    free = (t.particles["type"] & abi.TYPE_FIXED) == 0
    d = np.where(free[:, None], displacement, 0.0)
    r = np.zeros_like(d) if rotation is None else np.where(free[:, None], rotation, 0.0)
    p = {k: v.copy() for k, v in t.particles.items()}
    lp = p["xDiff"].dtype
    for k, name in enumerate(["xDiff", "yDiff", "zDiff"]):
        p[name][:] = d[:, k].astype(lp)
    for k, name in enumerate(["uDiff", "vDiff", "wDiff"]):
        p[name][:] = r[:, k].astype(lp)
    lib = HiDEMLib(t.params)
    lib.set_particles(p)
    lib.set_links(t.links)
    lib.computePartForce()
    links = lib.get_links()
    lib.close()
    q = {k: v.copy() for k, v in t.particles.items()}
    for k, name in enumerate(["xCord", "yCord", "zCord"]):
        q[name] += d[:, k]
    for k, name in enumerate(["xTheta", "yTheta", "zTheta"]):
        q[name] += r[:, k].astype(q[name].dtype)
    return q, links


def settle(t: Tongue, state=None, tol: float = 1e-6, check: int = 20, window: int = 200,
           max_steps: int = 40000, kernel: int = abi.STEP_KERNEL_AUTO) -> SettleResult:
    """Plain-method settling of a tongue from rest (state None: the undeformed lattice; or
    the (particles, links) of warm_state)."""
    p, links = (t.particles, t.links) if state is None else state
    lib = HiDEMLib(t.params)
    lib.set_step_kernel(kernel)
    lib.set_particles(p)
    lib.set_links(links)
    n = p["xCord"].shape[0]
    trace, below = [], 0
    steps, converged = 0, False
    while steps < max_steps:
        lib.step(check)
        steps += check
        kt, kr, _ = lib.kinetic_energy()
        e = (kt + kr) / n
        trace.append((steps, e))
        below = below + check if e < tol else 0
        if below >= window:
            converged = True
            break
    final = lib.get_particles()
    final_links = lib.get_links()
    lib.close()
    return SettleResult(steps, converged, final, trace, final_links)


def displacement_of(t: Tongue, final: dict) -> np.ndarray:
    p = t.particles
    return np.stack([final["xCord"] - p["xCord"], final["yCord"] - p["yCord"],
                     final["zCord"] - p["zCord"]], axis=1)


def rotation_of(t: Tongue, final: dict) -> np.ndarray:
    p = t.particles
    return np.stack([final[k].astype(np.float64) - p[k] for k in ("xTheta", "yTheta", "zTheta")], axis=1)


def settle_many(tongues, states=None, tol: float = 1e-6, check: int = 20, window: int = 200,
                max_steps: int = 40000, kernel: int = abi.STEP_KERNEL_AUTO):
    """settle() for many tongues at once: one batched launch per timestep (hidem_batch),
    kinetic energy read per tongue every `check` steps. Each tongue's trajectory is that of
    settle() on it alone; a tongue that has converged keeps stepping with the others (its
    convergence step is recorded when it converges)."""
    from .hidemlib import HiDEMBatch
    libs = []
    for i, t in enumerate(tongues):
        p, links = (t.particles, t.links) if states is None or states[i] is None else states[i]
        lib = HiDEMLib(t.params)
        lib.set_step_kernel(kernel)
        lib.set_particles(p)
        lib.set_links(links)
        libs.append(lib)
    n = [t.particles["xCord"].shape[0] for t in tongues]
    done = [None] * len(tongues)
    below = [0] * len(tongues)
    traces = [[] for _ in tongues]
    steps = 0
    with HiDEMBatch(libs) as batch:
        while steps < max_steps and any(d is None for d in done):
            batch.step(check)
            steps += check
            for i, lib in enumerate(libs):
                kt, kr, _ = lib.kinetic_energy()
                e = (kt + kr) / n[i]
                traces[i].append((steps, e))
                if done[i] is None:
                    below[i] = below[i] + check if e < tol else 0
                    if below[i] >= window:
                        done[i] = steps
    results = []
    for i, lib in enumerate(libs):
        results.append(SettleResult(done[i] if done[i] is not None else steps, done[i] is not None,
                                    lib.get_particles(), traces[i], lib.get_links()))
        lib.close()
    return results


@dataclass
class WarmStartReport:
    train_tongues: int
    test_tongues: int
    particles_per_tongue: float
    train_samples: int
    train_steps: int
    final_loss: float
    cold_steps: list
    warm_steps: list
    step_ratio: float              # mean cold steps / mean warm steps
    prediction_rel_error: list     # |pred - settled| / |settled| (L2, per test tongue)
    settled_error_over_d: list     # max |x_warm - x_cold| / d after both settled
    cold_converged: bool
    warm_converged: bool
    seconds: dict


def warm_start_experiment(n_train: int = 256, n_test: int = 16, size=(40.0, 12.0),
                          base_thickness: float = 6.0, amplitude: float = 2.0,
                          train_steps: int = 20000, batch: int = 8192, seed: int = 1000,
                          tol: float = 1e-6, max_steps: int = 40000, surrogate_cfg: dict | None = None,
                          with_rotation: bool = True, mirror: bool = True, inputs: str = "lattice",
                          max_train_rows: int | None = None, check: int = 20,
                          offsets=LATTICE_OFFSETS):
    """Cold settles of the training tongues, surrogate training on their settled
    displacements, then cold and warm settles of held-out tongues, compared by the plain
    method's convergence test. inputs: "lattice" (lattice_inputs, 4 Fourier bands, the
    learning rate decayed along a half cosine) or "coords" (the 5 coordinate inputs of
    surrogate_inputs, 6 bands, constant rate). max_train_rows: a seeded uniform sample of
    at most that many training rows (large tongues); check: steps between the kinetic-energy
    reads of the settles; offsets: the distances at which lattice_inputs samples the
    heightfields (longer ones for larger tongues)."""
    import time
    from . import surrogate as sg
    sec = {}
    t0 = time.time()
    train = [glacier_tongue(seed + i, size, base_thickness, amplitude=amplitude) for i in range(n_train)]
    test = [glacier_tongue(seed + 100000 + i, size, base_thickness, amplitude=amplitude) for i in range(n_test)]
    sec["geometry"] = time.time() - t0
    t0 = time.time()
    cold_train = settle_many(train, tol=tol, max_steps=max_steps, check=check)
    sec["cold_train_settles"] = time.time() - t0
    if inputs not in ("lattice", "coords"):
        raise ValueError(f"inputs {inputs!r}: 'lattice' or 'coords'")

    def feats(t, m=(1, 1)):
        if inputs == "lattice":
            return lattice_inputs(t, m, offsets)
        return surrogate_inputs(t) * np.array([m[0], m[1], 1, 1, 1], np.float32)

    t0 = time.time()
    ys = np.concatenate([displacement_of(t, r.final) for t, r in zip(train, cold_train)]) / DISP_SCALE
    # the settling problem is symmetric under x -> Lx - x and y -> Ly - y (vertical
    # gravity and buoyancy, a fixed base): each mirror image is a valid sample, with the
    # mirrored displacement component negated
    mirrors = ((1, 1), (-1, 1), (1, -1), (-1, -1)) if mirror else ((1, 1),)
    xs = np.concatenate([feats(t, m) for m in mirrors for t in train])
    ys = np.concatenate([ys * np.array([m[0], m[1], 1]) for m in mirrors])
    if max_train_rows is not None and xs.shape[0] > max_train_rows:
        pick = np.sort(np.random.default_rng(seed).choice(xs.shape[0], size=max_train_rows, replace=False))
        xs, ys = xs[pick], ys[pick]
    sec["features"] = time.time() - t0
    t0 = time.time()
    base = {"fourier_bands": 4, "cosine_decay": 1} if inputs == "lattice" else {"fourier_bands": 6}
    cfg = sg.default_config(batch=batch, inputs=xs.shape[1], **(base | (surrogate_cfg or {})))
    with sg.Surrogate(cfg) as net:
        net.set_data(xs, ys.astype(np.float32))
        loss = net.train(train_steps)
        preds = [net.predict(feats(t)).astype(np.float64) * DISP_SCALE for t in test]
    sec["training"] = time.time() - t0
    t0 = time.time()
    cold = settle_many(test, tol=tol, max_steps=max_steps, check=check)
    sec["cold_test_settles"] = time.time() - t0
    t0 = time.time()
    warm = settle_many(test, [warm_state(t, d, rotation_from_displacement(t, d) if with_rotation else None)
                              for t, d in zip(test, preds)], tol=tol, max_steps=max_steps, check=check)
    sec["warm_test_settles"] = time.time() - t0
    rel, err = [], []
    for t, d, c, w in zip(test, preds, cold, warm):
        true = displacement_of(t, c.final)
        rel.append(float(np.linalg.norm(d - true) / (np.linalg.norm(true) + 1e-30)))
        dx = np.stack([w.final[k] - c.final[k] for k in ("xCord", "yCord", "zCord")], axis=1)
        err.append(float(np.abs(dx).max() / (2 * float(t.particles["radius"][0]))))
    cs, ws = [r.steps for r in cold], [r.steps for r in warm]
    return WarmStartReport(n_train, n_test, float(np.mean([t.particles["xCord"].shape[0] for t in test])),
                           int(xs.shape[0]), train_steps, float(loss), cs, ws,
                           float(np.mean(cs) / max(np.mean(ws), 1)), rel, err,
                           all(r.converged for r in cold), all(r.converged for r in warm), sec)

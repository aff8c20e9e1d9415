"""Settling runs and the learned warm start: the tongue generator and the rotation
estimate (CPU); the kinetic-energy diagnostic, batched settles, the warm state built from
a displacement and a small end-to-end warm-start experiment (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, settle


def small(seed):
    return settle.glacier_tongue(seed, size=(24.0, 8.0), base_thickness=5.0, amplitude=1.5)


def test_tongue_geometry():
    t = small(3)
    p = t.particles
    n = p["xCord"].shape[0]
    assert 1000 < n < 3000
    assert np.all(p["zCord"] >= t.bed - 1e-12) and np.all(p["zCord"] <= t.bed + t.thick + 1e-12)
    fixed = (p["type"] & abi.TYPE_FIXED) != 0
    assert np.array_equal(fixed, p["zCord"] < t.bed + 1.0)
    assert 0 < fixed.sum() < n // 2
    assert t.links["state"].shape[0] > 4 * n
    u = settle.surrogate_inputs(t)
    assert u.shape == (n, 5) and np.all(np.abs(u[:, :3]) <= 1.0 + 1e-6)
    # the configuration's tongue: 200 m x 60 m, 150k-250k particles
    big = settle.glacier_tongue(1)
    assert 150_000 <= big.particles["xCord"].shape[0] <= 250_000


def test_lattice_inputs_and_their_mirror_images():
    t = small(9)
    p = t.particles
    n = p["xCord"].shape[0]
    f = settle.lattice_inputs(t)
    assert f.shape == (n, settle.N_LATTICE_INPUTS) and np.all(np.isfinite(f))
    assert np.array_equal(f[:, :5], settle.surrogate_inputs(t))
    no = len(settle.LATTICE_OFFSETS)
    disc = 5 + 8 * no
    # bonds, particles above, free particles below, against a direct count per column
    x, y, z = p["xCord"], p["yCord"], p["zCord"]
    free = (p["type"] & abi.TYPE_FIXED) == 0
    deg = np.zeros(n, int)
    np.add.at(deg, t.links["globalKeyEndA"], 1)
    np.add.at(deg, t.links["globalKeyEndB"], 1)
    for i in np.random.default_rng(0).choice(n, 40, replace=False):
        col = (np.abs(x - x[i]) < 1e-6) & (np.abs(y - y[i]) < 1e-6)
        assert f[i, disc] == pytest.approx(deg[i] / 6.0 - 1)
        assert f[i, disc + 1] == pytest.approx((col & (z > z[i])).sum() / 5.0 - 1)
        assert f[i, disc + 2] == pytest.approx((col & free & (z < z[i])).sum() / 5.0 - 1)
        assert f[i, disc + 3] == pytest.approx((z[col].max() - z[i]) / 5.0 - 1, abs=1e-6)
    # the x mirror image: x and the x offsets flip, the columns swap with their mirror
    fm = settle.lattice_inputs(t, (-1, 1))
    assert np.allclose(fm[:, 0], -f[:, 0], atol=1e-6) and np.array_equal(fm[:, 1:5], f[:, 1:5])
    for k in range(no):
        o = 5 + 8 * k
        assert np.allclose(fm[:, o:o + 2], f[:, o + 2:o + 4], atol=1e-6)   # +d x <-> -d x
        assert np.allclose(fm[:, o + 4:o + 8], f[:, o + 4:o + 8], atol=1e-6)  # y unchanged
    assert np.array_equal(fm[:, disc:disc + 5], f[:, disc:disc + 5])
    cols = settle.LATTICE_COLUMNS
    for q, (di, dj) in enumerate(cols):
        r = cols.index((-di, dj))
        a, b = disc + 5 + 2 * q, disc + 5 + 2 * r
        assert np.allclose(fm[:, a:a + 2], f[:, b:b + 2], atol=1e-6)
    # outside the plan the thickness input is that of zero ice: column 7 is the thickness
    # at x - 1.5 m, outside for x < 1 m
    edge = x < 1.0
    assert edge.any() and np.all(f[edge, 7] == -1.0)


def test_rotation_estimate_of_a_rigid_rotation():
    """For u = w x x (a small rigid rotation) the estimate returns -w: the model's rotation
    sign convention."""
    t = small(4)
    x = np.stack([t.particles[k] for k in ("xCord", "yCord", "zCord")], axis=1)
    w = np.array([1e-5, -2e-5, 3e-5])
    r = settle.rotation_from_displacement(t, np.cross(w, x))
    exact = np.all(np.abs(r + w) < 1e-10, axis=1)
    assert exact.mean() > 0.995 and np.all(np.isfinite(r))


@pytest.mark.gpu
def test_kinetic_energy_matches_the_host_formula(gpu):
    from hidem_b200.hidemlib import HiDEMLib
    t = small(5)
    lib = HiDEMLib(t.params)
    lib.set_particles(t.particles)
    lib.set_links(t.links)
    lib.step(30)
    kt, kr, vmax = lib.kinetic_energy()
    p = lib.get_particles()
    lib.close()
    lp = abi.lp_dtype(int(t.params.precision))
    dt = float(lp(t.params.dt))  # the library's constants are in lp precision
    d = 2.0 * p["radius"].astype(np.float64)
    m = float(lp(t.params.rhoIce)) * d ** 3
    inertia = m * d * d / 6.0
    v2 = sum((p[k].astype(np.float64) / dt) ** 2 for k in ("xDiff", "yDiff", "zDiff"))
    w2 = sum((p[k].astype(np.float64) / dt) ** 2 for k in ("uDiff", "vDiff", "wDiff"))
    assert kt == pytest.approx(float(np.sum(0.5 * m * v2)), rel=1e-9)
    assert kr == pytest.approx(float(np.sum(0.5 * inertia * w2)), rel=1e-9)
    assert vmax == pytest.approx(float(np.sqrt(v2.max())), rel=1e-9)
    assert kt > 0
    # momentum: linear and angular about the origin, the same velocities and masses
    lib = HiDEMLib(t.params)
    lib.set_particles(t.particles)
    lib.set_links(t.links)
    lib.step(30)
    lin, ang = lib.momentum()
    q = lib.get_particles()
    lib.close()
    v = np.stack([q[k].astype(np.float64) / dt for k in ("xDiff", "yDiff", "zDiff")], axis=1)
    w = np.stack([q[k].astype(np.float64) / dt for k in ("uDiff", "vDiff", "wDiff")], axis=1)
    x = np.stack([q[k] for k in ("xCord", "yCord", "zCord")], axis=1)
    pm = m[:, None] * v
    scale = float(np.abs(pm).sum())
    assert np.allclose(lin, pm.sum(axis=0), rtol=1e-9, atol=1e-12 * scale)
    want = np.cross(x, pm).sum(axis=0) + (inertia[:, None] * w).sum(axis=0)
    assert np.allclose(ang, want, rtol=1e-9, atol=1e-12 * float(np.abs(np.cross(x, pm)).sum()))


@pytest.mark.gpu
def test_batched_settles_equal_single_settles(gpu):
    ts = [small(6), small(7)]
    many = settle.settle_many(ts, max_steps=3000)
    for t, r in zip(ts, many):
        one = settle.settle(t, max_steps=3000)
        assert one.steps == r.steps or not (one.converged and r.converged)
        k = min(len(one.ke_trace), len(r.ke_trace))
        assert one.ke_trace[:k] == r.ke_trace[:k]


@pytest.mark.gpu
def test_exact_warm_state_settles_at_once_and_to_the_same_state(gpu):
    t = small(8)
    cold = settle.settle(t)
    assert cold.converged and cold.steps > 2000
    d = settle.displacement_of(t, cold.final)
    rot = settle.rotation_of(t, cold.final)
    free = (t.particles["type"] & abi.TYPE_FIXED) == 0
    est = settle.rotation_from_displacement(t, d)
    for k in range(3):
        assert np.corrcoef(rot[free, k], est[free, k])[0, 1] > 0.8
    warm = settle.settle(t, state=settle.warm_state(t, d, rot))
    assert warm.converged and warm.steps <= cold.steps // 5
    dx = max(np.abs(warm.final[k] - cold.final[k]).max() for k in ("xCord", "yCord", "zCord"))
    assert dx < 1e-4


@pytest.mark.gpu
def test_small_warm_start_experiment(gpu):
    r = settle.warm_start_experiment(n_train=8, n_test=2, size=(24.0, 8.0), base_thickness=5.0,
                                     amplitude=1.5, train_steps=1500, batch=4096, seed=77)
    assert r.cold_converged and r.warm_converged
    assert max(r.prediction_rel_error) < 0.5
    assert all(w < c for w, c in zip(r.warm_steps, r.cold_steps))
    assert max(r.settled_error_over_d) < 1e-3

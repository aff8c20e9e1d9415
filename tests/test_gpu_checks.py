"""Run-time checks of the rebuild, with the failure made on the host (a NaN or an infinite
coordinate written into the input arrays, a particle moved far away between uploads, a
crowd of particles placed in one cell): each ends in a status code, never in a GPU fault.

* non-finite coordinates: the reference bins floor(NaN) into some cell and carries on; the
  library refuses the rebuild (HIDEM_ERR_DEVICE);
* the grid-growth warning of NeighbourGrid::generateNeighbourGrid (PLiB/NeighbourGrid.cpp:
  89-92): counted in the statistics, a refusal with HIDEM_CHECK_GRID_GROWTH;
* a crowded neighbour-grid cell: sorted by input index as the reference's
  generateIterationList orders it (NeighbourGrid.cpp:163-184) up to 4096 members, refused
  (HIDEM_ERR_CAPACITY) beyond."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMLib
from oracle import oracle

pytestmark = pytest.mark.gpu


def _status(fn):
    with pytest.raises(abi.HidemError) as e:
        fn()
    return e.value.status


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("axis", ["xCord", "zCord"])
def test_non_finite_coordinate_fails_the_rebuild(gpu, bad, axis):
    P, p, l = workloads.ice_block(cells=(5, 4, 3), precision=abi.PREC_MIXED, seed=3)
    p[axis][37] = bad
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    assert _status(lib.regenerate) == abi.HIDEM_ERR_DEVICE
    assert _status(lambda: lib.local_bounds()) == abi.HIDEM_ERR_DEVICE
    lib.close()


def test_nan_after_steps_fails_the_next_rebuild(gpu):
    """A particle that becomes NaN between uploads (the host writes it, as an exploded
    state read back and re-set would carry it) stops the run at the next rebuild."""
    P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=abi.PREC_FP64, seed=5)
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    lib.step(5)
    lib.synchronize()
    q = lib.get_particles()
    q["yCord"][11] = np.nan
    lib.set_particles(q)
    lib.set_links(l)
    assert _status(lambda: lib.step(1)) == abi.HIDEM_ERR_DEVICE
    lib.close()


def test_grid_growth_is_counted_and_refused_on_request(gpu):
    P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=abi.PREC_MIXED, seed=7)
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    lib.regenerate()
    assert lib.stats()["grid_growth_events"] == 0
    far = {k: v.copy() for k, v in p.items()}
    far["xCord"][3] += 500.0  # one particle thrown far away: the grid grows ~100x
    lib.set_particles(far)
    lib.set_links(l)
    lib.regenerate()  # the reference only warns
    assert lib.stats()["grid_growth_events"] == 1
    lib.set_particles(p)
    lib.set_links(l)
    lib.regenerate()  # back to the small grid: no growth
    lib.set_checks(abi.CHECK_GRID_GROWTH)
    lib.set_particles(far)
    lib.set_links(l)
    assert _status(lib.regenerate) == abi.HIDEM_ERR_DEVICE
    assert lib.stats()["grid_growth_events"] == 2
    with pytest.raises(abi.HidemError):
        lib.set_checks(8)
    lib.close()


def _crowd(n, seed, precision):
    """n particles of radius 0.5 inside one 1 m cube, [0.05, 1.05)^3: with a grid whose
    corner is at -1.2 (or at the crowd's own corner), one cell of the 1.2 m grid."""
    rng = np.random.default_rng(seed)
    p = abi.empty_particles(n, precision)
    for k in ("xCord", "yCord", "zCord"):
        p[k][:] = rng.uniform(0.05, 1.05, n)
    p["radius"][:] = 0.5
    p["globalKeys"][:] = np.arange(n)
    return p


@pytest.mark.parametrize("n", [33, 700, 4096])
def test_crowded_cell_is_ordered_like_the_oracle(gpu, n):
    precision = abi.PREC_MIXED
    p = _crowd(n, n, precision)
    # one particle in each of the 26 cells around the crowd (the grid's corner at -1.2), so
    # the crowd is one cell among several and its neighbours walk it too
    pts = np.array([(a, b, c) for a in (-1.2, 0.6, 1.8) for b in (-1.2, 0.6, 1.8)
                    for c in (-1.2, 0.6, 1.8) if (a, b, c) != (0.6, 0.6, 0.6)])
    rng = np.random.default_rng(0)
    order = rng.permutation(n + len(pts))  # the crowd's members spread over the input order
    q = abi.empty_particles(n + len(pts), precision)
    for j, k in enumerate(("xCord", "yCord", "zCord")):
        q[k][order] = np.concatenate([p[k], pts[:, j]])
    q["radius"][:] = 0.5
    q["globalKeys"][:] = np.arange(n + len(pts))
    P = abi.default_params(precision=precision, maxRadius=0.5, searchDistanceScale=1.2)
    lib = HiDEMLib(P)
    lib.set_particles(q)
    lib.set_links(abi.empty_links(0, precision))
    lib.regenerate()
    ix, iy, iz, dims, mins = lib.get_cells()
    counts, lst = lib.get_neighbours()
    lib.close()
    ox, oy, oz, odims, omins = oracle.port().cells(P, q)
    assert np.array_equal(ix, ox) and np.array_equal(iy, oy) and np.array_equal(iz, oz)
    assert tuple(dims) == (3, 3, 3)
    colour = ix.astype(np.int64) + dims[0] * (iy + dims[1] * iz.astype(np.int64))
    assert np.bincount(colour).max() == n
    oc, ol = oracle.port().neighbours(P, q)
    assert np.array_equal(counts, oc)
    assert np.array_equal(lst, ol)  # the crowd's members in input order


def test_overcrowded_cell_is_refused(gpu):
    p = _crowd(4097, 3, abi.PREC_MIXED)
    P = abi.default_params(precision=abi.PREC_MIXED, maxRadius=0.5, searchDistanceScale=1.2)
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(abi.empty_links(0, abi.PREC_MIXED))
    assert _status(lib.regenerate) == abi.HIDEM_ERR_CAPACITY
    lib.close()

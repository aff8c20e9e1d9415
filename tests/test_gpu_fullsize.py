"""Parity at the benchmark's own size: the 5.7M-particle calving slab (400 x 100 x 100 m FCC,
d = 1 m, flat bed, water line 90 m, front pressure, 1 % of the links pre-broken), both
precisions, against the reference's own CPU path (oracle/_ref, IEEE build; the C
restatement where that was not built). Bit-exact, as on the small fixtures:

* cells and the contact list (pairs and their per-particle order) of the first rebuild;
* three timesteps of the sample main loop with a rebuild every two steps
  (grid.gridRegenInterval = 2, so the rebuild of step 2 bins moved particles): positions,
  rotations, increments, link states, CT history, break events, rebuild steps;
* cells and contact list of a rebuild forced on the final state."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMLib
from oracle import oracle

pytestmark = pytest.mark.gpu

P_OUT = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
         "uDiff", "vDiff", "wDiff"]
L_OUT = ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]


def _checker(precision):
    if oracle.reference_available(precision):
        return oracle.reference(precision)
    return oracle.port()


def _same_grid(lib, cpu, P, particles):
    ix, iy, iz, dims, mins = lib.get_cells()
    ox, oy, oz, odims, omins = cpu.cells(P, particles)
    assert tuple(dims) == tuple(odims) and tuple(mins) == tuple(omins)
    assert np.array_equal(ix, ox) and np.array_equal(iy, oy) and np.array_equal(iz, oz)
    counts, lst = lib.get_neighbours()
    oc, ol = cpu.neighbours(P, particles)
    assert np.array_equal(counts, oc)
    assert np.array_equal(lst, ol)


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_full_slab_bit_exact_against_reference(gpu, precision):
    P, p, l = workloads.calving_slab(size=(400.0, 100.0, 100.0), precision=precision, jitter=0.0)
    P.gridRegenInterval = 2
    n = p["xCord"].shape[0]
    assert n == 5706412
    cpu = _checker(precision)
    steps = 3

    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    lib.regenerate()
    _same_grid(lib, cpu, P, p)

    lib.step(steps)
    lib.synchronize()
    out_p = lib.get_particles()
    out_l = lib.get_links()
    li, st = lib.get_break_events()
    stats = lib.stats()
    ref_p, ref_l, _, ref_events, ref_regen, _ = cpu.run(P, p, l, steps)
    for k in P_OUT:
        assert np.array_equal(out_p[k], ref_p[k]), (k, float(np.abs(out_p[k] - ref_p[k]).max()))
    for k in L_OUT:
        assert np.array_equal(out_l[k], ref_l[k]), k
    order = np.lexsort((li, st))
    events = np.stack([li[order], st[order]], axis=1) if len(li) else np.zeros((0, 2), np.int64)
    assert np.array_equal(events.reshape(-1, 2), np.asarray(ref_events).reshape(-1, 2))
    assert stats["regen_count"] - 1 == len(ref_regen)  # the explicit rebuild above, then the policy's

    lib.regenerate()
    _same_grid(lib, cpu, P, ref_p)
    lib.close()

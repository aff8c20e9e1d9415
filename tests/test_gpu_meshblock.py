"""Parity on the reference's own benchmark inputs: the MeshBlock runs of
HiDEM/Benchmark/<size> (config_mesh_<size>.toml with its particles.h5: File lattice, scale 12,
links by the distance rule with linkGenScale 1.2), read by the library's TOML front-end and
HDF5 reader, against the reference's CPU path (oracle/_ref, IEEE build; the C restatement
where that was not built). The inputs are read from data/meshblock_<size>/ (copies of the
reference's files); a size whose files are absent is skipped.

The run config is the reference's except for two settings that make three steps exercise
every part of the path: breakTime 0 (the benchmark breaks links only after t = 5 s, step
25,000) and a rebuild every two steps (grid.gridRegenInterval = 2). Bit-exact, as on the
small fixtures: cells and contact list of the first rebuild; positions, rotations,
increments, link states, CT history, break events and rebuild steps after three steps; cells
and contact list of a rebuild forced on the final state."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMLib
from oracle import oracle

pytestmark = pytest.mark.gpu

DATA = Path(__file__).resolve().parents[1] / "data"
P_OUT = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
         "uDiff", "vDiff", "wDiff"]
L_OUT = ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]
KNOWN = {"310k": 318777, "5700k": 5723826}


def _files(size):
    d = DATA / f"meshblock_{size}"
    cfg, pf = d / f"config_mesh_{size}.toml", d / "particles.h5"
    if not (cfg.exists() and pf.exists()):
        pytest.skip(f"{d} does not hold the reference's benchmark files")
    return cfg, pf


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


@pytest.mark.parametrize("size,precision", [("310k", abi.PREC_MIXED), ("310k", abi.PREC_FP64),
                                            ("5700k", abi.PREC_MIXED)])
def test_meshblock_input_bit_exact_against_reference(gpu, size, precision):
    cfg, pf = _files(size)
    P, p, l, info = workloads.meshblock(str(cfg), str(pf), precision)
    assert p["xCord"].shape[0] == KNOWN[size]
    P.breakTime = 0.0
    P.gridRegenInterval = 2
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
    assert stats["regen_count"] - 1 == len(ref_regen)
    # the particles moved: the comparison covers the force and integrate arithmetic
    assert np.abs(out_p["zDiff"]).max() > 0

    lib.regenerate()
    _same_grid(lib, cpu, P, ref_p)
    lib.close()

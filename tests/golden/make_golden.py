"""Generates the golden fixtures of tests/golden/ from the reference's own CPU hot path.

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores the inputs (a seeded FCC lattice and its distance-rule links) and the
outputs of oracle/_ref/libhidem_ref_{mixed,fp64}.so — the reference's NeighbourGrid,
NeighAccel, LinkAccelSide, CombinedAccel and HiDEMDefaultFunctions compiled from its
sources with IEEE flags — so the C restatement in oracle/ is pinned against the reference
even where the reference tree is absent.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from hidem_b200 import abi, workloads  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # 6x6x6 unit cells = 864 particles, bottom layer fixed, in air; links break
    "block6": dict(kind="block", cells=(6, 6, 6), steps=100, seed=3),
    # 5x3x3 cells with a bed, water line, calving front, velocity limit and boundaries
    "slab533": dict(kind="slab", cells=(5, 3, 3), steps=60, seed=5),
}


def make_case(name: str, spec: dict, precision: int):
    if spec["kind"] == "block":
        P, p, l = workloads.ice_block(cells=spec["cells"], precision=precision, seed=spec["seed"])
    else:
        nx, ny, nz = spec["cells"]
        size = (nx * workloads.SQRT2, ny * workloads.SQRT2, nz * workloads.SQRT2)
        P, p, l = workloads.calving_slab(size=size, precision=precision, seed=spec["seed"],
                                         jitter=0.01, broken_fraction=0.05, water_level=2.5,
                                         useVelocityLimit=1, useBoundary=1, maxVel=0.5,
                                         lowerLimit=(-0.6, -0.6, -100.0),
                                         upperLimit=(nx * 1.4142 + 0.2, ny * 1.4142 + 0.2, 100.0),
                                         boundaryMin=(1, 1, 0), boundaryMax=(1, 1, 0),
                                         gridRegenInterval=25)
    ref = oracle.reference(precision)
    ix, iy, iz, dims, mins = ref.cells(P, p)
    counts, nlist = ref.neighbours(P, p)
    p1, l1, F, events, regen, _ = ref.run(P, p, l, spec["steps"])
    tag = "mixed" if precision == abi.PREC_MIXED else "fp64"
    arrays = {}
    for k, v in p.items():
        arrays["in_p_" + k] = v
    for k, v in l.items():
        arrays["in_l_" + k] = v
    for k in ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
              "uDiff", "vDiff", "wDiff"]:
        arrays["out_p_" + k] = p1[k]
    for k in ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]:
        arrays["out_l_" + k] = l1[k]
    arrays.update(out_force=F, out_events=events, out_regen=regen, cells=np.stack([ix, iy, iz]),
                  dims=np.array(dims), mins=np.array(mins), nbr_counts=counts, nbr_list=nlist,
                  steps=np.array(spec["steps"]))
    params = P.as_dict()
    for k, v in params.items():
        arrays["param_" + k] = np.array(v)
    np.savez_compressed(OUT / f"{name}_{tag}.npz", **arrays)
    print(f"{name}_{tag}: n={p['xCord'].shape[0]} L={l['state'].shape[0]} "
          f"events={len(events)} regen={list(regen)}")


def main():
    for precision in (abi.PREC_MIXED, abi.PREC_FP64):
        if not oracle.reference_available(precision):
            raise SystemExit("oracle/_ref not built: run `make -C oracle` with the reference tree")
        for name, spec in CASES.items():
            make_case(name, spec, precision)


if __name__ == "__main__":
    main()

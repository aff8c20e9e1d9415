"""Batched contexts (hidem_batch_*): many independent blocks advanced by one launch per
timestep must give, per block, exactly the results of hidem_step on that block alone
(particles, CT history, break events, rebuild count), with and without CUDA graphs, for
each step kernel and in the per-context fallback; one block is also checked against the
oracle."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMBatch, HiDEMLib
from oracle import oracle

pytestmark = pytest.mark.gpu

P_OUT = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
         "uDiff", "vDiff", "wDiff"]
L_OUT = ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]
PRECS = [abi.PREC_MIXED, abi.PREC_FP64]


def mixed_blocks(precision):
    """Blocks of uneven sizes with different rebuild phases: a falling block that
    triggers the displacement rule, one with a fixed rebuild interval, one starting at
    step 3, one with a forced rebuild at step 17, one with a low break threshold, and one
    with other material constants (a second launch group)."""
    specs = [
        dict(cells=(4, 4, 4), seed=4, fixed_bottom=False, g=-9.81e4, waterLevel=-1e3),
        dict(cells=(5, 3, 4), seed=5, gridRegenInterval=7),
        dict(cells=(3, 3, 3), seed=6, start=3),
        dict(cells=(6, 5, 4), seed=7, firstBalanceTimestep=17),
        dict(cells=(5, 5, 5), seed=8, maxLoad=2e-5),
        dict(cells=(2, 2, 2), seed=9),
        dict(cells=(4, 3, 3), seed=10, E=5e8, maxLoad=1e-4),
    ]
    out = []
    for sp in specs:
        sp = dict(sp)
        start = sp.pop("start", 0)
        cells = sp.pop("cells")
        seed = sp.pop("seed")
        P, p, l = workloads.ice_block(cells=cells, precision=precision, seed=seed, **sp)
        out.append((P, p, l, start))
    return out


def open_lib(P, p, l, start):
    lib = HiDEMLib(P)
    if start:
        lib.set_timestep(start)
    lib.set_particles(p)
    lib.set_links(l)
    return lib


def snapshot(lib):
    lib.synchronize()
    out_p = lib.get_particles()
    out_l = lib.get_links()
    li, st = lib.get_break_events()
    order = np.lexsort((li, st))
    ev = np.stack([li[order], st[order]], axis=1) if len(li) else np.zeros((0, 2), np.int64)
    return out_p, out_l, ev, lib.stats()["regen_count"], lib.getCurrentTimestep()


def assert_same(a, b):
    for k in P_OUT:
        assert np.array_equal(a[0][k], b[0][k]), k
    for k in L_OUT:
        assert np.array_equal(a[1][k], b[1][k]), k
    assert np.array_equal(a[2], b[2])
    assert a[3] == b[3] and a[4] == b[4]


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("mode", ["graphs", "launches", "per_context", "items", "thread", "two_pass",
                                  "two_pass_launches"])
def test_batch_equals_individual_runs(gpu, precision, mode):
    blocks = mixed_blocks(precision)
    alone = []
    for P, p, l, start in blocks:
        lib = open_lib(P, p, l, start)
        lib.step(13)
        lib.step(24)
        alone.append(snapshot(lib))
        lib.close()
    libs = [open_lib(P, p, l, start) for P, p, l, start in blocks]
    kernels = {"items": abi.STEP_KERNEL_ITEMS, "thread": abi.STEP_KERNEL_THREAD,
               "two_pass": abi.STEP_KERNEL_TWO_PASS, "two_pass_launches": abi.STEP_KERNEL_TWO_PASS}
    if mode in kernels:  # the batch runs the first context's step kernel
        libs[0].set_step_kernel(kernels[mode])
    batch = HiDEMBatch(libs, graphs=(mode not in ("launches", "two_pass_launches")),
                       per_context=(mode == "per_context"))
    batch.step(13)
    batch.step(24)
    counts = batch.counts()
    batch.close()
    for lib, ref in zip(libs, alone):
        assert_same(snapshot(lib), ref)
        lib.close()
    if mode == "per_context":
        assert counts["launches"] == 37 * len(blocks)
    else:
        # three groups of shared constants: the falling block (g, no fixed layer), the
        # block with another E, and the rest; the two-pass step (the default) is three
        # launches, the fused kernels one
        assert counts["launches"] == 37 * 3 * (1 if mode in ("items", "thread") else 3)
    if mode in ("graphs", "items", "thread", "two_pass"):
        assert counts["graph_launches"] > 0
    assert sum(r[3] for r in alone) > len(blocks)  # rebuilds happened inside the runs


@pytest.mark.parametrize("precision", PRECS)
def test_batch_block_matches_oracle(gpu, precision):
    P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=precision, seed=4,
                                  fixed_bottom=False, g=-9.81e4, waterLevel=-1e3,
                                  firstBalanceTimestep=30)
    P2, p2, l2 = workloads.ice_block(cells=(5, 4, 3), precision=precision, seed=12)
    ref = oracle.port().run(P, p, l, 45)
    libs = [open_lib(P, p, l, 0), open_lib(P2, p2, l2, 0)]
    with HiDEMBatch(libs) as batch:
        batch.step(45)
    got = snapshot(libs[0])
    for k in P_OUT:
        assert np.array_equal(got[0][k], ref[0][k]), k
    for k in L_OUT:
        assert np.array_equal(got[1][k], ref[1][k]), k
    assert np.array_equal(got[2].reshape(-1, 2), np.asarray(ref[3]).reshape(-1, 2))
    assert got[3] == len(ref[4])
    for lib in libs:
        lib.close()


def test_batch_interleaves_with_single_context_calls(gpu):
    """A context may be stepped alone between batch calls; the batch picks up its state."""
    precision = abi.PREC_MIXED
    blocks = mixed_blocks(precision)[:3]
    alone = []
    for P, p, l, start in blocks:
        lib = open_lib(P, p, l, start)
        lib.step(21)
        alone.append(snapshot(lib))
        lib.close()
    libs = [open_lib(P, p, l, start) for P, p, l, start in blocks]
    with HiDEMBatch(libs) as batch:
        batch.step(6)
        libs[1].step(5)
        libs[0].step(5)
        libs[2].step(5)
        batch.step(10)
    for lib, ref in zip(libs, alone):
        assert_same(snapshot(lib), ref)
        lib.close()


def test_batch_argument_errors(gpu):
    P, p, l = workloads.ice_block(cells=(2, 2, 2), precision=abi.PREC_MIXED)
    P64, p64, l64 = workloads.ice_block(cells=(2, 2, 2), precision=abi.PREC_FP64)
    a = open_lib(P, p, l, 0)
    b = open_lib(P64, p64, l64, 0)
    with pytest.raises(abi.HidemError, match="precision"):
        HiDEMBatch([a, b])
    with pytest.raises(abi.HidemError, match="twice"):
        HiDEMBatch([a, a])
    with pytest.raises(abi.HidemError, match="no contexts"):
        HiDEMBatch([])
    c = HiDEMLib(P)
    with HiDEMBatch([a, c]) as batch:
        with pytest.raises(abi.HidemError, match="particles and links"):
            batch.step(1)
        with pytest.raises(abi.HidemError, match="negative"):
            batch.step(-1)
    for x in (a, b, c):
        x.close()


@pytest.mark.parametrize("with_links", [True, False])
def test_batch_with_contexts_without_links(gpu, with_links):
    """Blocks whose link set is empty beside one with links, and (with_links False) a batch
    in which no context has links (the break pass's own grid keeps one idle CTA): every block
    matches its run alone."""
    blocks = []
    for k, (cells, seed) in enumerate([((3, 3, 3), 21), ((4, 3, 3), 22), ((2, 3, 2), 23)]):
        P, p, l = workloads.ice_block(cells=cells, precision=abi.PREC_MIXED, seed=seed,
                                      fixed_bottom=False, g=-9.81e3, waterLevel=-1e3)
        if k > 0 or not with_links:
            l = {key: v[:0] for key, v in l.items()}
        blocks.append((P, p, l, 0))
    alone = []
    for P, p, l, start in blocks:
        lib = open_lib(P, p, l, start)
        lib.step(13)
        lib.step(12)
        alone.append(snapshot(lib))
        lib.close()
    libs = [open_lib(P, p, l, start) for P, p, l, start in blocks]
    batch = HiDEMBatch(libs, graphs=True)
    batch.step(13)
    batch.step(12)
    batch.close()
    for lib, ref in zip(libs, alone):
        assert_same(snapshot(lib), ref)
        lib.close()
    assert np.abs(alone[1][0]["zDiff"]).min() > 0  # the blocks moved


@pytest.mark.parametrize("kernel", [abi.STEP_KERNEL_TWO_PASS, abi.STEP_KERNEL_THREAD_CAPPED])
def test_batch_runs_without_grid_service_between_them(gpu, kernel):
    """Every context rebuilds on a fixed interval longer than the longest run (10 steps),
    so consecutive runs meet no gridService point: each run still starts from the host's
    step state (step, record buffer, owed link update)."""
    blocks = []
    for cells, seed in [((4, 3, 3), 31), ((3, 3, 4), 32)]:
        P, p, l = workloads.ice_block(cells=cells, precision=abi.PREC_MIXED, seed=seed,
                                      gridRegenInterval=50, maxLoad=2e-5)
        blocks.append((P, p, l, 0))
    alone = []
    for P, p, l, start in blocks:
        lib = open_lib(P, p, l, start)
        lib.set_step_kernel(kernel)
        lib.step(13)
        lib.step(24)
        alone.append(snapshot(lib))
        lib.close()
    libs = [open_lib(P, p, l, start) for P, p, l, start in blocks]
    libs[0].set_step_kernel(kernel)
    batch = HiDEMBatch(libs, graphs=True)
    batch.step(13)
    batch.step(24)
    batch.close()
    for lib, ref in zip(libs, alone):
        assert_same(snapshot(lib), ref)
        lib.close()
    assert sum(len(r[2]) for r in alone) > 0  # links broke inside the runs

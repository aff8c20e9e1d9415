"""Slab decomposition on the GPU: 2 and 3 ranks as contexts of one process (the halo force
exchange as device-to-device copies between them), against one context holding every
particle. The decomposed run must give the same bits: positions, rotations, differences,
link states and every link side's CT, through rebuilds (with the particles recut over the
ranks at each) and link breaks."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, slab, workloads
from hidem_b200.hidemlib import HiDEMLib

pytestmark = pytest.mark.gpu

PRECS = [abi.PREC_MIXED, abi.PREC_FP64]


def case(name, precision):
    if name == "falling_block":
        # falls through the displacement rule's rebuilds; a low break threshold
        P, p, l = workloads.ice_block(cells=(9, 4, 4), precision=precision, seed=4, fixed_bottom=False,
                                      g=-9.81e4, waterLevel=-1e3, maxLoad=2e-5, breakTime=0.0)
        return P, p, l, 60
    # bed, front pressure, pre-broken links, a fixed rebuild interval
    P, p, l = workloads.calving_slab(size=(14.0, 4.3, 4.3), precision=precision, seed=2,
                                     broken_fraction=0.1, water_level=3.0, gridRegenInterval=7,
                                     breakTime=0.0, maxLoad=1e-4)
    return P, p, l, 40


def one_context(P, p, l, steps):
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    lib.step(steps)
    lib.synchronize()
    out = lib.get_particles(), lib.get_links(), lib.stats()
    lib.close()
    return out


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("name", ["falling_block", "calving_slab"])
@pytest.mark.parametrize("nranks,slack", [(2, 0.5), (3, 0.5), (2, 0.0), (3, 0.0)])
def test_decomposed_run_matches_one_context(gpu, precision, name, nranks, slack):
    """slack 0.5: rebuilds keep the held sets (the particles move far less than the halo's
    room); slack 0: every rebuild after the first movement redistributes."""
    P, p, l, steps = case(name, precision)
    rp, rl, rs = one_context(P, p, l, steps)
    assert rs["regen_count"] >= 3
    libs = [HiDEMLib(P) for _ in range(nranks)]
    try:
        run = slab.SlabRun(slab.LocalComm(nranks), libs, p, l, slack=slack)
        assert run._on_device()  # redistributions keep the state on the GPU
        assert all(0 < lib.n < p["xCord"].shape[0] for lib in libs)
        run.step(steps)
        gp, gl = run.gather()
        assert run.redistributions + run.kept == 1 + rs["regen_count"]
        if slack > 0:
            assert run.kept == rs["regen_count"]
        else:
            assert run.redistributions >= rs["regen_count"]
        assert run.exchanged > 0
        assert all(lib.stats()["step"] == steps for lib in libs)
    finally:
        for lib in libs:
            lib.close()
    for k, v in rp.items():
        if k != "owners":
            assert np.array_equal(gp[k], v), f"particle field {k}"
    for k, v in rl.items():
        if k != "owners":
            assert np.array_equal(gl[k], v), f"link field {k}"
    broke = int((l["state"] != 0).sum() - (rl["state"] != 0).sum())
    if name == "falling_block":
        assert broke > 0


def test_halo_exchange_entry_points_check_their_arguments(gpu):
    P, p, l, _ = case("calving_slab", abi.PREC_MIXED)
    lib = HiDEMLib(P)
    try:
        lib.set_particles(p)
        lib.set_links(l)
        n = p["xCord"].shape[0]
        with pytest.raises(abi.HidemError) as e:
            lib.set_halo_exchange(np.array([0, n]), np.zeros(0))
        assert e.value.status == abi.HIDEM_ERR_ARG
        lo, hi = lib.local_bounds()
        assert np.allclose(lo, [p["xCord"].min(), p["yCord"].min(), p["zCord"].min()])
        with pytest.raises(abi.HidemError) as e:
            lib.regenerate_frame(lo + 1.0, hi)          # particles outside the box
        assert e.value.status == abi.HIDEM_ERR_ARG
        with pytest.raises(abi.HidemError) as e:
            lib.grid_service_decide([np.nan, 0.0, 0.0])
        assert e.value.status == abi.HIDEM_ERR_ARG
        # a larger box than the particles' own gives the same contact pairs
        lib.regenerate()
        c0, n0 = lib.get_neighbours()
        lib.regenerate_frame(lo - 3.0, hi + 5.0)
        c1, n1 = lib.get_neighbours()
        assert np.array_equal(c0, c1)
        assert np.allclose(lib.stats()["grid_min"], lo - 3.0)
    finally:
        lib.close()


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("kernel", [abi.STEP_KERNEL_THREAD_CAPPED, abi.STEP_KERNEL_ITEMS])
def test_pack_in_the_force_pass_equals_the_pack_kernel(gpu, precision, kernel):
    """hidem_compute_forces_packed: the send records written by the force pass's epilogue
    (the item kernel: by the pack kernel after it) equal hidem_compute_forces followed by
    hidem_pack_halo_forces, before and after a rebuild that moves the slots."""
    import torch
    P, p, l, _ = case("calving_slab", precision)
    n = p["xCord"].shape[0]
    rng = np.random.default_rng(3)
    send = np.sort(rng.choice(n, size=n // 7, replace=False)).astype(np.int32)
    recv = np.sort(rng.choice(n, size=n // 9, replace=False)).astype(np.int32)
    dt = torch.float32 if precision == abi.PREC_MIXED else torch.float64
    libs = []
    for _ in range(2):
        lib = HiDEMLib(P)
        lib.set_step_kernel(kernel)
        lib.set_particles(p)
        lib.set_links(l)
        lib.set_halo_exchange(send, recv)
        libs.append(lib)
    a, b = libs
    for rnd in range(3):
        ba = torch.zeros(6 * send.size, dtype=dt, device="cuda")
        bb = torch.full((6 * send.size,), -7.0, dtype=dt, device="cuda")
        a.computePartForce()
        a.pack_halo_forces(ba.data_ptr())
        b.compute_forces_packed(bb.data_ptr())
        a.synchronize()
        b.synchronize()
        assert torch.equal(ba, bb)
        assert np.array_equal(a.get_forces(), b.get_forces())
        for lib in libs:
            lib.applyForce()
            lib.finalizeTs()
            if rnd == 1:
                lib.regenerate()
    for lib in libs:
        lib.close()


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("keys", ["identity", "ascending", "shuffled"])
def test_state_from_and_to_device_arrays(gpu, precision, keys):
    """hidem_set_particles / hidem_set_links from arrays in device memory and the readbacks
    into device memory give the state the host arrays give, bit for bit; with global keys
    that are not 0..n-1 the link ends are resolved by a search of the key table (on the device
    when the keys ascend, on the host otherwise)."""
    import torch
    P, p, l = workloads.ice_block(cells=(5, 4, 4), precision=precision, seed=21, fixed_bottom=False,
                                  g=-9.81e4, waterLevel=-1e3, maxLoad=2e-5, breakTime=0.0)
    if keys != "identity":
        # keys in ascending order (ends found on the device) or shuffled (on the host)
        rng = np.random.default_rng(5)
        n = p["xCord"].shape[0]
        perm = (np.arange(n) if keys == "ascending" else rng.permutation(n)).astype(np.int64) * 3 + 7
        p = dict(p, globalKeys=perm)
        l = dict(l, globalKeyEndA=perm[l["globalKeyEndA"]], globalKeyEndB=perm[l["globalKeyEndB"]])
    dev = torch.device("cuda", 0)
    tp = {k: torch.from_numpy(v).to(dev) for k, v in p.items()}
    tl = {k: torch.from_numpy(v).to(dev) for k, v in l.items()}
    torch.cuda.synchronize()
    a, b = HiDEMLib(P), HiDEMLib(P)
    try:
        a.set_particles(p)
        a.set_links(l)
        b.set_particles(tp)
        b.set_links(tl)
        for lib in (a, b):
            lib.step(25)
        ha, hl = a.get_particles(), a.get_links()
        db, dl = b.get_particles_device(), b.get_links_device()
        for k, v in ha.items():
            assert np.array_equal(db[k].cpu().numpy(), v), k
        for k, v in hl.items():
            assert np.array_equal(dl[k].cpu().numpy(), v), k
        assert (hl["state"] == 0).any()  # links broke in the run
    finally:
        a.close()
        b.close()

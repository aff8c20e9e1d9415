"""Slab decomposition host logic (no GPU): the partition and its halos, the split / merge
of the whole state, and the driver's rank-spanning steps with a stand-in rank whose force
of a particle is a known function of its key and the step, in one process and as two gloo
ranks."""
from __future__ import annotations

import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hidem_b200 import abi, slab, workloads


def _block(cells=(12, 4, 4), precision=abi.PREC_MIXED, seed=3):
    P, p, l = workloads.ice_block(cells=cells, precision=precision, seed=seed, fixed_bottom=False)
    return P, p, l


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_layout_owns_every_particle_once_and_halos_hold_every_partner(nranks):
    from scipy.spatial import cKDTree
    P, p, l = _block()
    a, b = slab.link_ends(p, l)
    search = 1.2 * 1.0            # searchDistanceScale x diameter of the block's spheres
    halo = slab.halo_width(search, search - 1.0, 0.5)
    lay = slab.slab_layout(p["xCord"], a, b, nranks, halo)
    n = p["xCord"].shape[0]
    assert np.bincount(lay.owner, minlength=nranks).sum() == n
    counts = np.bincount(lay.owner, minlength=nranks)
    assert counts.max() - counts.min() <= max(1, n // 20)   # count-balanced cuts (lattice planes)
    pts = np.stack([p["xCord"], p["yCord"], p["zCord"]], 1)
    pairs = cKDTree(pts).query_pairs(search * 1.001, output_type="ndarray")
    for r in range(nranks):
        held = np.zeros(n, bool)
        held[lay.local[r]] = True
        own = lay.owner == r
        # every contact candidate and every link partner of an owned particle is held
        for i, j in ((pairs[:, 0], pairs[:, 1]), (pairs[:, 1], pairs[:, 0])):
            assert held[j[own[i]]].all()
        mine = lay.links[r]
        assert held[a[mine]].all() and held[b[mine]].all()
        assert np.array_equal(mine, np.flatnonzero(own[a] | own[b]))
        # the halo particles are exactly those whose forces arrive, once each
        recv = lay.local[r][lay.recv_list(r)]
        assert np.array_equal(np.sort(recv), np.flatnonzero(held & ~own))
        assert (lay.owner[lay.local[r][lay.send_list(r)]] == r).all()
    for r in range(nranks):
        for s in range(nranks):
            if r != s:
                assert lay.send_counts(r)[s] == lay.recv_counts(s)[r]


def test_split_then_merge_gives_back_the_state():
    P, p, l = _block(cells=(10, 3, 3))
    rng = np.random.default_rng(1)
    for k in abi.SIDE_FIELDS:
        l[k][:] = rng.standard_normal(l[k].shape[0]).astype(l[k].dtype)
    l["state"][rng.choice(l["state"].shape[0], 20, replace=False)] = 0
    a, b = slab.link_ends(p, l)
    lay = slab.slab_layout(p["xCord"], a, b, 3, 1.3)
    parts = [slab.split_state(p, l, lay, r) for r in range(3)]
    for r, (pr, lr) in enumerate(parts):
        assert np.array_equal(pr["globalKeys"], p["globalKeys"][lay.local[r]])
        assert lr["CT0"].shape[0] == 2 * lr["state"].shape[0]
    mp_, ml = slab.merge_state(parts, lay, p["xCord"].shape[0], l["state"].shape[0])
    for k, v in p.items():
        if k != "owners":
            assert np.array_equal(mp_[k], v), k
    assert np.array_equal(mp_["owners"], lay.owner)
    for k, v in l.items():
        assert np.array_equal(ml[k], v), k


def test_cuts_are_quantiles_and_owner_follows_them():
    x = np.array([5.0, 1.0, 3.0, 2.0, 4.0, 0.0])
    cuts = slab.slab_cuts(x, 3)
    assert cuts[0] == -np.inf and cuts[-1] == np.inf
    assert list(cuts[1:-1]) == [2.0, 4.0]
    assert list(slab.slab_owner(x, cuts)) == [2, 0, 1, 1, 2, 0]


# -------------------------------------------------------------------- driver, stand-in ranks

def _force(keys, step, q):
    return ((keys * 7 + step * 3 + q) % 101).astype(np.float32) * 0.5


class FakeRank:
    """Stand-in for HiDEMLib with the methods the slab driver calls: the force of a
    particle is _force(key, step, q), computed only for the particles this rank owns (halo
    forces are garbage until the exchange), and applyForce adds the x force to uDiff and
    moves every particle 0.4 in x, so that particles change owner across redistributions."""

    precision = abi.PREC_MIXED
    device = 0

    def __init__(self, rank, regen_every=4):
        self.rank, self.step_, self.regen_every = rank, 0, regen_every
        self.checked = 0

    def stats(self):
        return {"search_distance": 1.2, "interact_distance": 0.2}

    def set_particles(self, p):
        self.p = {k: v.copy() for k, v in p.items()}
        self.n = p["xCord"].shape[0]

    def set_links(self, l):
        self.l = {k: v.copy() for k, v in l.items()}

    def set_halo_exchange(self, snd, rcv):
        self.snd, self.rcv = np.asarray(snd), np.asarray(rcv)

    def get_particles(self):
        return {k: v.copy() for k, v in self.p.items()}

    def get_links(self):
        return {k: v.copy() for k, v in self.l.items()}

    def grid_service_local(self):
        return np.zeros(3), self.step_ % 10 == 0

    def grid_service_decide(self, mx):
        return self.step_ % self.regen_every == 0

    def local_bounds(self):
        xyz = np.stack([self.p["xCord"], self.p["yCord"], self.p["zCord"]])
        return xyz.min(1), xyz.max(1)

    def regenerate_frame(self, lo, hi):
        self.frame = (np.array(lo), np.array(hi))

    def computePartForce(self):
        own = self.p["owners"] == self.rank
        self.F = np.full((6, self.n), -1.0, np.float32)
        for q in range(6):
            self.F[q, own] = _force(self.p["globalKeys"][own], self.step_, q)

    def pack_halo_forces(self, ptr):
        m = self.snd.size
        buf = np.ctypeslib.as_array((C.c_float * (6 * m)).from_address(ptr)) if m else None
        if m:
            buf[:] = self.F[:, self.snd].T.reshape(-1)

    def unpack_halo_forces(self, ptr):
        m = self.rcv.size
        if m:
            buf = np.ctypeslib.as_array((C.c_float * (6 * m)).from_address(ptr))
            self.F[:, self.rcv] = buf.reshape(m, 6).T

    def synchronize(self):
        pass

    def getCurrentTimestep(self):
        return self.step_

    def breakActive(self, step=None):
        assert step is None or step == self.step_
        return False

    def applyForce(self):
        for q in range(6):
            want = _force(self.p["globalKeys"], self.step_, q)
            assert np.array_equal(self.F[q], want), "a halo force did not arrive"
        self.checked += self.n
        self.p["uDiff"] += self.F[0]
        self.p["xCord"] += 0.4

    def linkUpdate(self):
        pass

    def finalizeTs(self):
        self.step_ += 1


def _expected(p, steps):
    u = p["uDiff"].copy()
    for t in range(steps):
        u += _force(p["globalKeys"], t, 0)
    return u


@pytest.mark.parametrize("nranks", [2, 3])
def test_driver_in_one_process_moves_every_halo_force(nranks):
    P, p, l = _block()
    run = slab.SlabRun(slab.LocalComm(nranks), [FakeRank(r) for r in range(nranks)], p, l, halo=1.3)
    run.step(9)
    gp, gl = run.gather()
    assert np.array_equal(gp["uDiff"], _expected(p, 9))
    assert np.allclose(gp["xCord"], p["xCord"] + 0.4 * 9)
    # the first distribution, then rebuilds at steps 0 (nothing moved yet: held sets kept),
    # 4 and 8 (every particle moved 1.6 in x, more than the halo's room: redistributed)
    assert run.redistributions == 3 and run.kept == 1
    assert run.exchanged > 0
    for k, v in l.items():
        assert np.array_equal(gl[k], v), k


def _gloo_rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P, p, l = _block()
        comm = slab.DistComm()
        assert comm.allmax([np.array([float(rank), -float(rank)])]).tolist() == [world - 1.0, 0.0]
        fake = FakeRank(rank)
        run = slab.SlabRun(comm, [fake], p, l, halo=1.3)
        run.step(7)
        gp, gl = run.gather()
        ok = bool(np.array_equal(gp["uDiff"], _expected(p, 7)))
        ok &= all(np.array_equal(gl[k], v) for k, v in l.items())
        q.put((rank, ok, fake.checked, run.exchanged))
    except Exception as e:  # reported to the parent instead of a queue timeout
        q.put((rank, repr(e), 0, 0))
    finally:
        dist.destroy_process_group()


def test_driver_on_two_gloo_ranks_moves_every_halo_force():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] is True for r in res), res
    assert all(r[2] > 0 and r[3] > 0 for r in res)


def _gloo_exchange_rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch
        comm = slab.DistComm()
        # rank r sends (r + 1) * 10 + d bytes of value 16 r + d to every other rank d
        sends = {(rank, d): torch.full(((rank + 1) * 10 + d,), 16 * rank + d, dtype=torch.uint8)
                 for d in range(world) if d != rank}
        sizes = {(s_, rank): (s_ + 1) * 10 + rank for s_ in range(world) if s_ != rank}
        got = comm.exchange_tensors(sends, sizes, [torch.device("cpu")])
        ok = sorted(got) == sorted(sizes)
        ok &= all(int(t.numel()) == sizes[k] and bool((t == 16 * k[0] + k[1]).all()) for k, t in got.items())
        q.put((rank, ok))
    except Exception as e:  # reported to the parent instead of a queue timeout
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_tensor_exchange_on_gloo_ranks(world):
    """The redistribution's byte-buffer exchange between processes (point to point, every
    size known to both sides) delivers each buffer to its destination intact."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_exchange_rank, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
    assert [r[0] for r in res] == list(range(world))
    assert all(r[1] is True for r in res), res


@pytest.mark.parametrize("nranks", [2, 3, 4])
def test_incremental_redistribution_equals_the_whole_set_split(nranks):
    """After a redistribution (every particle moved past the halo's room) each rank holds
    exactly what splitting the gathered whole set by the new layout gives, array for array,
    although it received only the particles and links it did not hold before."""
    P, p, l = _block()
    fakes = [FakeRank(r) for r in range(nranks)]
    run = slab.SlabRun(slab.LocalComm(nranks), fakes, p, l, halo=1.3)
    run.step(5)  # redistributes at step 4
    assert run.redistributions == 2
    whole_p, whole_l = run.gather()
    for r, f in enumerate(fakes):
        ep, el = slab.split_state(whole_p, whole_l, run.layout, r)
        for k, v in ep.items():
            assert np.array_equal(f.p[k], v), (r, k)
        for k, v in el.items():
            assert np.array_equal(f.l[k], v), (r, k)
        assert np.array_equal(f.snd, run.layout.send_list(r))
        assert np.array_equal(f.rcv, run.layout.recv_list(r))


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_layout_with_torch_equals_numpy(nranks):
    """The recut computed with torch (on the device in a run; here on the host) gives the
    numpy layout's cuts, owners and index sets exactly."""
    import torch
    P, p, l = _block()
    a, b = slab.link_ends(p, l)
    a, b = a.astype(np.int64), b.astype(np.int64)
    x = p["xCord"] + np.random.default_rng(nranks).normal(0, 0.3, p["xCord"].shape[0])
    want = slab.slab_layout(x, a, b, nranks, 1.3)
    got = slab.slab_layout_torch(torch.from_numpy(x), torch.from_numpy(a), torch.from_numpy(b), nranks, 1.3)
    assert np.array_equal(got.cuts, want.cuts)
    assert np.array_equal(got.owner, want.owner)
    for r in range(nranks):
        assert np.array_equal(got.local[r], want.local[r])
        assert np.array_equal(got.links[r], want.links[r])
        for s_ in range(nranks):
            assert np.array_equal(got.send[r][s_], want.send[r][s_])


def test_local_tensor_exchange_checks_sizes():
    """Between ranks of one process the redistribution's buffers go to the destination's
    device as they are; a buffer whose size differs from the one both sides computed is an
    error, not a silent short copy."""
    import torch
    comm = slab.LocalComm(2)
    buf = torch.arange(7, dtype=torch.uint8)
    got = comm.exchange_tensors({(0, 1): buf}, {(0, 1): 7}, [torch.device("cpu")] * 2)
    assert torch.equal(got[(0, 1)], buf)
    with pytest.raises(RuntimeError):
        comm.exchange_tensors({(0, 1): buf}, {(0, 1): 8}, [torch.device("cpu")] * 2)

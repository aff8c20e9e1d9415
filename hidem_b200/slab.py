"""Slab decomposition of one particle set over ranks, one context per rank.

What the reference does with MPI (HiDEMLib/HiDEMDistribution.h:99-234): each rank owns
the particles inside its domain, holds halo copies of the other ranks' particles within a
halo distance of it (ParticleTransporter.h:114-130, ``Domain::withinHalo``) and of the
links that touch its own particles (LinkTransporter.h), computes the forces of its own
particles, receives the forces of its halo particles from their owners and integrates
both (``computePartForce``, HiDEMLib.h:316-382, the ``pForceComm`` exchange of 6 force
components), so that halo copies stay identical to their originals; gridService reduces
the displacement over ranks (``accumulateDist``, HiDEMLib.h:463-474) and, when the
domains are rebalanced, particles move to their new owners with their link-side state
(``syncLinkSideData`` + ``reDistribute``, HiDEMDistribution.h:59-98, 188-234).

Here the domains are slabs along x with count-balanced cuts (the reference's
``DomainBuilder::generateBalancedDomains`` in one dimension with unit weights), recut at
every rebuild of the neighbour structures. Two choices differ from the reference so that
a decomposed run is bit-identical to one context holding every particle:

* every rank bins its particles in the grid of the whole set (``hidem_regenerate_frame``
  with the box over all ranks), so cell colours, and with them the order of every contact
  list, are those of one rank; particles and links keep the relative order of the whole
  set, so the (colour, index) order and the link-id order of every link-end list are too;
* gridService reduces the three displacement maxima over ranks, not each rank's norm of
  its own.

The per-step exchange is one packed buffer per rank (``hidem_pack_halo_forces``), one
contiguous run per peer, moved by the ``comm`` object: ``LocalComm`` for several contexts
in one process (device-to-device copies), ``DistComm`` for one rank per process over
``torch.distributed`` (NCCL point-to-point on GPUs; gloo on the host for tests).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import abi

# ---------------------------------------------------------------------------------------
# partition (numpy only)


def slab_cuts(x: np.ndarray, nranks: int) -> np.ndarray:
    """nranks + 1 cut positions along x: -inf, the count quantiles, +inf. Particle i
    belongs to rank r when cuts[r] <= x_i < cuts[r + 1]."""
    if nranks < 1:
        raise ValueError("need at least one rank")
    xs = np.sort(np.asarray(x, np.float64))
    n = xs.shape[0]
    inner = [xs[min(n - 1, (k * n) // nranks)] for k in range(1, nranks)] if n else [0.0] * (nranks - 1)
    return np.array([-np.inf, *inner, np.inf])


def slab_owner(x: np.ndarray, cuts: np.ndarray) -> np.ndarray:
    return np.searchsorted(cuts[1:-1], np.asarray(x, np.float64), side="right").astype(np.int32)


@dataclass
class SlabLayout:
    """Which particles and links each rank holds (indices into the whole set, ascending)."""
    cuts: np.ndarray
    owner: np.ndarray            # int32[N] owning rank of every particle
    local: list                  # local[r]: particles rank r holds (own + halo)
    links: list                  # links[r]: links with an end rank r owns
    send: list                   # send[r][s]: particles r owns whose force s integrates

    @property
    def nranks(self) -> int:
        return len(self.local)

    def local_index(self, r: int, glob: np.ndarray) -> np.ndarray:
        """Positions of the whole-set particle indices `glob` in rank r's particle order."""
        idx = np.searchsorted(self.local[r], glob)
        if glob.size and not np.array_equal(self.local[r][np.minimum(idx, self.local[r].size - 1)], glob):
            raise ValueError(f"particles not held by rank {r}")
        return idx.astype(np.int32)

    def send_list(self, r: int) -> np.ndarray:
        """Rank r's send list in its own indices: the runs for peers 0, 1, ... in order."""
        runs = [self.send[r][s] for s in range(self.nranks) if s != r]
        glob = np.concatenate(runs) if runs else np.zeros(0, np.int64)
        return self.local_index(r, glob)

    def recv_list(self, r: int) -> np.ndarray:
        runs = [self.send[s][r] for s in range(self.nranks) if s != r]
        glob = np.concatenate(runs) if runs else np.zeros(0, np.int64)
        return self.local_index(r, glob)

    def send_counts(self, r: int) -> list:
        return [0 if s == r else int(self.send[r][s].size) for s in range(self.nranks)]

    def recv_counts(self, r: int) -> list:
        return [0 if s == r else int(self.send[s][r].size) for s in range(self.nranks)]


def slab_layout(x: np.ndarray, link_a: np.ndarray, link_b: np.ndarray, nranks: int,
                halo: float, cuts: np.ndarray | None = None) -> SlabLayout:
    """Owners by x slab, halos of width `halo` on either side of each slab plus the far
    ends of every link that touches a rank's own particles (so that every link of an owned
    particle is complete), and the force lists between ranks."""
    x = np.asarray(x, np.float64)
    link_a = np.asarray(link_a, np.int64)
    link_b = np.asarray(link_b, np.int64)
    if cuts is None:
        cuts = slab_cuts(x, nranks)
    owner = slab_owner(x, cuts)
    oa, ob = owner[link_a], owner[link_b]
    local, links = [], []
    for r in range(nranks):
        near = (x >= cuts[r] - halo) & (x < cuts[r + 1] + halo)
        mine = (oa == r) | (ob == r)
        held = near | (owner == r)
        held[link_a[mine]] = True
        held[link_b[mine]] = True
        local.append(np.flatnonzero(held).astype(np.int64))
        links.append(np.flatnonzero(mine).astype(np.int64))
    send = [[np.zeros(0, np.int64) for _ in range(nranks)] for _ in range(nranks)]
    for s in range(nranks):
        held = local[s]
        for r in range(nranks):
            if r != s:
                send[r][s] = held[owner[held] == r]
    return SlabLayout(cuts=cuts, owner=owner, local=local, links=links, send=send)


def slab_layout_torch(x, link_a, link_b, nranks: int, halo: float) -> SlabLayout:
    """slab_layout computed with torch on the device the tensors live on (x float64[N],
    link_a / link_b int64[L]); the same cuts, owners and index sets, returned as numpy."""
    import torch
    n = x.shape[0]
    if nranks < 1:
        raise ValueError("need at least one rank")
    xs = torch.sort(x).values
    inner = [float(xs[min(n - 1, (k * n) // nranks)]) for k in range(1, nranks)] if n else [0.0] * (nranks - 1)
    cuts = np.array([-np.inf, *inner, np.inf])
    cuts_t = torch.tensor(cuts, dtype=torch.float64, device=x.device)
    owner = torch.searchsorted(cuts_t[1:-1].contiguous(), x, right=True).to(torch.int32)
    oa, ob = owner[link_a], owner[link_b]
    local, links, held_sets = [], [], []
    for r in range(nranks):
        near = (x >= cuts[r] - halo) & (x < cuts[r + 1] + halo)
        mine = (oa == r) | (ob == r)
        held = near | (owner == r)
        held[link_a[mine]] = True
        held[link_b[mine]] = True
        loc = torch.nonzero(held).flatten()
        held_sets.append(loc)
        local.append(loc.cpu().numpy())
        links.append(torch.nonzero(mine).flatten().cpu().numpy())
    send = [[np.zeros(0, np.int64) for _ in range(nranks)] for _ in range(nranks)]
    for s_ in range(nranks):
        held = held_sets[s_]
        ow = owner[held]
        for r in range(nranks):
            if r != s_:
                send[r][s_] = held[ow == r].cpu().numpy()
    return SlabLayout(cuts=cuts, owner=owner.cpu().numpy(), local=local, links=links, send=send)


def key_index(keys: np.ndarray, wanted: np.ndarray) -> np.ndarray:
    """Positions of the particle keys `wanted` in `keys` (globalKey -> index)."""
    keys = np.asarray(keys, np.int64)
    order = np.argsort(keys, kind="stable")
    pos = np.searchsorted(keys[order], wanted)
    pos = np.minimum(pos, keys.size - 1)
    if not np.array_equal(keys[order][pos], wanted):
        raise ValueError("link end key without a particle")
    return order[pos]


def link_ends(particles: dict, links: dict) -> tuple[np.ndarray, np.ndarray]:
    keys = particles["globalKeys"]
    return key_index(keys, links["globalKeyEndA"]), key_index(keys, links["globalKeyEndB"])


def split_state(particles: dict, links: dict, layout: SlabLayout, r: int) -> tuple[dict, dict]:
    """Rank r's particle and link arrays (whole-set order kept; owners = owning rank)."""
    sel = layout.local[r]
    p = {k: np.ascontiguousarray(v[sel]) for k, v in particles.items()}
    p["owners"] = np.ascontiguousarray(layout.owner[sel].astype(np.int32))
    ls = layout.links[r]
    side = np.stack([2 * ls, 2 * ls + 1], axis=1).reshape(-1)
    l = {}
    for k, v in links.items():
        l[k] = np.ascontiguousarray(v[side] if k in abi.SIDE_FIELDS else v[ls])
    return p, l


def merge_state(parts: list, layout: SlabLayout, n: int, L: int) -> tuple[dict, dict]:
    """The whole set from every rank's arrays (as split_state laid them out): each
    particle from its owner, each link side's state (CT0..5) from the owner of that side's
    particle, the rest of a link from the owner of its end A."""
    p0, l0 = parts[0]
    particles = {k: np.zeros(n, v.dtype) for k, v in p0.items()}
    links = {k: np.zeros(2 * L if k in abi.SIDE_FIELDS else L, v.dtype) for k, v in l0.items()}
    have = np.zeros(n, bool)
    for r, (p, l) in enumerate(parts):
        sel = layout.local[r]
        own = layout.owner[sel] == r
        for k, v in p.items():
            particles[k][sel[own]] = v[own]
        have[sel[own]] = True
    if not have.all():
        raise ValueError("a particle has no owner")
    a, b = link_ends(particles, links_keys(parts, layout, L))
    for r, (p, l) in enumerate(parts):
        ls = layout.links[r]
        ownA = layout.owner[a[ls]] == r
        ownB = layout.owner[b[ls]] == r
        for k, v in l.items():
            if k in abi.SIDE_FIELDS:
                v2 = v.reshape(-1, 2)
                links[k][2 * ls[ownA]] = v2[ownA, 0]
                links[k][2 * ls[ownB] + 1] = v2[ownB, 1]
            else:
                links[k][ls[ownA]] = v[ownA]
    return particles, links


def links_keys(parts: list, layout: SlabLayout, L: int) -> dict:
    """The link end keys of the whole set (every link is held by the owner of an end)."""
    ka = np.zeros(L, np.int64)
    kb = np.zeros(L, np.int64)
    for r, (_, l) in enumerate(parts):
        ls = layout.links[r]
        ka[ls] = l["globalKeyEndA"]
        kb[ls] = l["globalKeyEndB"]
    return {"globalKeyEndA": ka, "globalKeyEndB": kb}


def contact_reach(search_distance: float, interact_distance: float, max_radius: float) -> float:
    """Reach of a contact-list pair at a rebuild (NeighAccel.h:104-114:
    d - (r_i + r_j) < interactDist), with 1 % to spare for the rounding of d."""
    return 1.01 * max(search_distance, 2.0 * max_radius + interact_distance)


def halo_width(search_distance: float, interact_distance: float, max_radius: float,
               slack: float = 0.5) -> float:
    """The contact reach plus `slack` of it, the room particles may move in x between two
    distributions (rebuilds in between keep the held sets while no particle has moved
    more than half the room)."""
    return (1.0 + slack) * contact_reach(search_distance, interact_distance, max_radius)


# ---------------------------------------------------------------------------------------
# transports


class LocalComm:
    """Every rank in this process (several contexts, on one GPU or several)."""

    def __init__(self, nranks: int):
        self.size = nranks
        self.ranks = list(range(nranks))

    def allmax(self, vals: list) -> np.ndarray:
        return np.max(np.stack([np.asarray(v, np.float64) for v in vals]), axis=0)

    def allgather(self, objs: list) -> list:
        return list(objs)

    def exchange_tensors(self, sends: dict, recv_sizes: dict, devices: list) -> dict:
        """Byte buffers keyed (source, destination) between ranks of this process."""
        return _local_exchange_tensors(sends, recv_sizes, devices, self.ranks)

    def exchange(self, layout: SlabLayout, send_bufs: list, recv_bufs: list) -> None:
        """recv_bufs[s]'s run from r <- send_bufs[r]'s run for s (torch tensors). Device
        buffers are copied on the devices' current streams, which the caller orders between
        its contexts' packs and unpacks; host buffers are copied when this returns."""
        R = self.size
        soff = [np.concatenate([[0], np.cumsum(layout.send_counts(r))]) for r in range(R)]
        roff = [np.concatenate([[0], np.cumsum(layout.recv_counts(s))]) for s in range(R)]
        for r in range(R):
            for s in range(R):
                cnt = 0 if r == s else int(layout.send[r][s].size)
                if cnt:
                    src = send_bufs[r][6 * soff[r][s]: 6 * (soff[r][s] + cnt)]
                    dst = recv_bufs[s][6 * roff[s][r]: 6 * (roff[s][r] + cnt)]
                    dst.copy_(src, non_blocking=False)


def _local_exchange_tensors(sends: dict, recv_sizes: dict, devices: list, ranks: list) -> dict:
    """Every send is to a rank of this process: the destination's device gets the buffer."""
    dev_of = dict(zip(ranks, devices))
    out = {}
    for (s, r), n in recv_sizes.items():
        buf = sends[(s, r)]
        if buf.numel() != n:
            raise RuntimeError(f"redistribution buffer {s} -> {r}: {buf.numel()} bytes, expected {n}")
        out[(s, r)] = buf.to(dev_of[r])
    return out


class DistComm:
    """One rank per process over torch.distributed (NCCL with CUDA buffers, gloo with host
    buffers); the process group is initialised by the caller."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.size = dist.get_world_size()
        self.ranks = [dist.get_rank()]
        self.backend = dist.get_backend()

    def _dev(self):
        import torch
        return torch.device("cuda", torch.cuda.current_device()) if self.backend == "nccl" else torch.device("cpu")

    def allmax(self, vals: list) -> np.ndarray:
        import torch
        t = torch.tensor(np.asarray(vals[0], np.float64), device=self._dev())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def allgather(self, objs: list) -> list:
        out = [None] * self.size
        self.dist.all_gather_object(out, objs[0])
        return out

    def exchange_tensors(self, sends: dict, recv_sizes: dict, devices: list) -> dict:
        """Byte buffers keyed (source, destination): this rank's sends to the other ranks,
        its receives from them, point to point (NCCL moves device tensors between GPUs;
        gloo host tensors). Both sides know every size, so no size travels first."""
        import torch
        dev = self._dev()
        r = self.ranks[0]
        ops, out = [], {}
        for (s, d), buf in sorted(sends.items()):
            ops.append(self.dist.P2POp(self.dist.isend, buf.to(dev), d))
        for (s, d), n in sorted(recv_sizes.items()):
            t = torch.empty(n, dtype=torch.uint8, device=dev)
            out[(s, d)] = t
            ops.append(self.dist.P2POp(self.dist.irecv, t, s))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        if dev.type == "cuda":
            torch.cuda.current_stream(dev).synchronize()
        target = devices[0] if devices else dev
        return {k: v.to(target) for k, v in out.items()}

    def exchange(self, layout: SlabLayout, send_bufs: list, recv_bufs: list) -> None:
        r = self.ranks[0]
        sc, rc = layout.send_counts(r), layout.recv_counts(r)
        soff, roff = np.concatenate([[0], np.cumsum(sc)]), np.concatenate([[0], np.cumsum(rc)])
        ops = []
        for s in range(self.size):
            if sc[s]:
                ops.append(self.dist.P2POp(self.dist.isend, send_bufs[0][6 * soff[s]: 6 * soff[s + 1]], s))
            if rc[s]:
                ops.append(self.dist.P2POp(self.dist.irecv, recv_bufs[0][6 * roff[s]: 6 * roff[s + 1]], s))
        if ops:
            # with NCCL, wait() orders the current stream after the transfers (no host wait);
            # the caller orders its contexts' streams after the current stream
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()


# ---------------------------------------------------------------------------------------
# driver


class SlabRun:
    """The ranks of one particle set that live in this process, stepped together.

    ``libs`` are this process's contexts (``HiDEMLib``, or any object with the same
    methods), one per rank in ``comm.ranks``; ``particles`` / ``links`` the whole set
    (numpy arrays as ``HiDEMLib.set_particles`` / ``set_links`` take them), the same on
    every process. Steps follow the sample main: gridService, computePartForce (with the
    halo force exchange), applyForce, linkUpdate when t*dt > breakTime, finalizeTs."""

    def __init__(self, comm, libs: list, particles: dict, links: dict, halo: float | None = None,
                 slack: float = 0.5, device_redistribution: bool = True):
        import torch
        if len(libs) != len(comm.ranks):
            raise ValueError("one context per rank of this process")
        self.comm, self.libs = comm, list(libs)
        self.n = int(particles["xCord"].shape[0])
        self.L = int(links["globalKeyEndA"].shape[0])
        self.precision = int(self.libs[0].precision)
        self.lp = abi.lp_dtype(self.precision)
        self._tdtype = torch.float32 if self.lp == np.float32 else torch.float64
        self._halo, self._slack = halo, float(slack)
        # redistribute with the state in device memory where the contexts and the transport
        # allow it (else, or when False, through host arrays)
        self.device_redistribution = bool(device_redistribution)
        self._a_dev = self._b_dev = None  # link ends on the device, for the device recut
        self.redistributions = 0
        self.kept = 0           # rebuilds that kept the held sets (no redistribution)
        self.exchanged = 0      # halo force records moved so far (all ranks of this process)
        self._distribute(particles, links)

    # -- state movement
    def _widths(self, particles: dict) -> tuple[float, float]:
        """(contact reach, halo width)."""
        s = self.libs[0].stats()
        rmax = float(np.max(particles["radius"])) if self.n else 0.0
        rmax = float(self.comm.allmax([np.array([rmax])])[0])
        reach = contact_reach(s["search_distance"], s["interact_distance"], rmax)
        width = float(self._halo) if self._halo is not None else (1.0 + self._slack) * reach
        return reach, width

    def _distribute(self, particles: dict, links: dict) -> None:
        """The first distribution, from the whole set (every process has it)."""
        a, b = link_ends(particles, links)
        self._a, self._b = a.astype(np.int64), b.astype(np.int64)  # link ends never change
        self._reach, self._width = self._widths(particles)
        self.layout = slab_layout(particles["xCord"], a, b, self.comm.size, self._width)
        self._install([split_state(particles, links, self.layout, r) for r in self.comm.ranks])

    def _install(self, states: list) -> None:
        """Sets this process's contexts to their held sets of self.layout."""
        import torch
        self.send_bufs, self.recv_bufs = [], []
        self._x0 = []
        if any(hasattr(p["xCord"], "is_cuda") and p["xCord"].is_cuda for p, _ in states):
            torch.cuda.synchronize()  # device arrays are complete before the library reads them
        for lib, r, (p, l) in zip(self.libs, self.comm.ranks, states):
            dev = _lib_device(lib)
            x = p["xCord"]
            if dev.type == "cuda" and hasattr(lib, "get_particles_device"):
                # the x at distribution, where the moved-distance check reads it back
                self._x0.append(torch.as_tensor(x).to(dev).clone())
            else:
                self._x0.append(x.clone() if hasattr(x, "clone") else x.copy())
            lib.set_particles(p)
            lib.set_links(l)
            snd, rcv = self.layout.send_list(r), self.layout.recv_list(r)
            lib.set_halo_exchange(snd, rcv)
            self.send_bufs.append(torch.zeros(6 * max(1, snd.size), dtype=self._tdtype, device=dev))
            self.recv_bufs.append(torch.zeros(6 * max(1, rcv.size), dtype=self._tdtype, device=dev))
        self.redistributions += 1

    def _redistribute(self) -> None:
        """A new distribution from the ranks' current state, moving only what changes hands
        (the reference's ParticleTransporter / LinkTransporter, HiDEMDistribution.h:188-234):
        every rank publishes the x of the particles it owns, every process recomputes the
        same layout from them (slab_layout is deterministic), and each rank receives only
        the particles and links it did not hold before — each from a rank that held it:
        particles from their old owner, links from the old owner of their end A. Halo
        copies and every held link's two sides are bit-equal to their originals (forces
        are exchanged; a side's history depends only on the two end records), so what a
        rank already holds stays as it is. The result equals splitting the gathered whole
        set by the new layout, array for array."""
        if self._on_device():
            return self._redistribute_device()
        old = self.layout
        R = self.comm.size
        states, mine = [], []
        for lib, r in zip(self.libs, self.comm.ranks):
            p, l = lib.get_particles(), lib.get_links()
            states.append((p, l))
            own = old.owner[old.local[r]] == r
            mine.append((old.local[r][own], p["xCord"][own]))
        x_all = np.empty(self.n, np.float64)
        seen = np.zeros(self.n, bool)
        for idx, x in self.comm.allgather(mine):
            x_all[idx] = x
            seen[idx] = True
        if not seen.all():
            raise RuntimeError("a particle has no owner")
        new = slab_layout(x_all, self._a, self._b, R, self._width)
        # what each destination lacks, from the ranks of this process that can supply it
        payloads = []
        for (p, l), r in zip(states, self.comm.ranks):
            pay = {}
            for d in range(R):
                if d == r:
                    continue
                need_p = np.setdiff1d(new.local[d], old.local[d], assume_unique=True)
                need_p = need_p[old.owner[need_p] == r]
                need_l = np.setdiff1d(new.links[d], old.links[d], assume_unique=True)
                need_l = need_l[old.owner[self._a[need_l]] == r]
                if need_p.size == 0 and need_l.size == 0:
                    continue
                pi = old.local_index(r, need_p)
                li = np.searchsorted(old.links[r], need_l)
                side = np.stack([2 * li, 2 * li + 1], axis=1).reshape(-1)
                pay[d] = (need_p, {k: v[pi] for k, v in p.items()}, need_l,
                          {k: (v[side] if k in abi.SIDE_FIELDS else v[li]) for k, v in l.items()})
            payloads.append(pay)
        received = self.comm.allgather(payloads)
        out = []
        for (p, l), r in zip(states, self.comm.ranks):
            gp, gl = new.local[r], new.links[r]
            np_ = {k: np.zeros(gp.size, v.dtype) for k, v in p.items()}
            nl = {k: np.zeros(2 * gl.size if k in abi.SIDE_FIELDS else gl.size, v.dtype) for k, v in l.items()}
            # kept: what this rank held before
            pos = np.minimum(np.searchsorted(old.local[r], gp), max(old.local[r].size - 1, 0))
            kept = old.local[r][pos] == gp if old.local[r].size else np.zeros(gp.size, bool)
            for k, v in p.items():
                np_[k][kept] = v[pos[kept]]
            lpos = np.minimum(np.searchsorted(old.links[r], gl), max(old.links[r].size - 1, 0))
            lkept = old.links[r][lpos] == gl if old.links[r].size else np.zeros(gl.size, bool)
            for k, v in l.items():
                if k in abi.SIDE_FIELDS:
                    nl[k].reshape(-1, 2)[lkept] = v.reshape(-1, 2)[lpos[lkept]]
                else:
                    nl[k][lkept] = v[lpos[lkept]]
            got_p, got_l = kept.copy(), lkept.copy()
            for pays in received:
                if r not in pays:
                    continue
                idx, vals, lidx, lvals = pays[r]
                if idx.size:
                    at = np.searchsorted(gp, idx)
                    for k, v in vals.items():
                        np_[k][at] = v
                    got_p[at] = True
                if lidx.size:
                    at = np.searchsorted(gl, lidx)
                    for k, v in lvals.items():
                        if k in abi.SIDE_FIELDS:
                            nl[k].reshape(-1, 2)[at] = v.reshape(-1, 2)
                        else:
                            nl[k][at] = v
                    got_l[at] = True
            if not (got_p.all() and got_l.all()):
                raise RuntimeError(f"rank {r}: particles or links missing after the redistribution")
            np_["owners"] = np.ascontiguousarray(new.owner[gp].astype(np.int32))
            out.append((np_, nl))
        self.layout = new
        self._install(out)

    def _on_device(self) -> bool:
        """Whether the redistribution can keep the state on the GPUs: contexts that read back
        to device memory, halo buffers there, and a transport that moves device tensors."""
        return (self.device_redistribution and bool(self.send_bufs) and self.send_bufs[0].is_cuda
                and all(hasattr(lib, "get_particles_device") for lib in self.libs)
                and hasattr(self.comm, "exchange_tensors"))

    def _redistribute_device(self) -> None:
        """_redistribute with the particle and link state kept in device memory: each
        context reads its held set back into device arrays; the moves are gathered, packed
        into one byte buffer per destination and sent by the transport's device exchange
        (device copies between contexts of this process, NCCL point-to-point between
        processes); the new held sets are assembled on the device and handed to the contexts
        from there. Only the owned particles' x (for the new cut) and index arrays travel
        through host memory."""
        import torch
        old = self.layout
        R = self.comm.size
        states, mine = [], []
        for lib, r in zip(self.libs, self.comm.ranks):
            p, l = lib.get_particles_device(), lib.get_links_device()
            states.append((p, l))
            own = old.owner[old.local[r]] == r
            dev = p["xCord"].device
            mine.append((old.local[r][own], p["xCord"][torch.from_numpy(np.flatnonzero(own)).to(dev)].cpu().numpy()))
        x_all = np.empty(self.n, np.float64)
        seen = np.zeros(self.n, bool)
        for idx, x in self.comm.allgather(mine):
            x_all[idx] = x
            seen[idx] = True
        if not seen.all():
            raise RuntimeError("a particle has no owner")
        dev0 = states[0][0]["xCord"].device
        if self._a_dev is None or self._a_dev.device != dev0:
            self._a_dev = torch.from_numpy(self._a).to(dev0)
            self._b_dev = torch.from_numpy(self._b).to(dev0)
        new = slab_layout_torch(torch.from_numpy(x_all).to(dev0), self._a_dev, self._b_dev, R, self._width)
        # what each rank held before (masks over the whole set) and, for this process's
        # ranks, where each held particle / link sat in their arrays (inverse maps): every
        # set difference and position below is one gather
        held_p = [_mask(old.local[q], self.n) for q in range(R)]
        held_l = [_mask(old.links[q], self.L) for q in range(R)]
        inv_p = {r: _inverse(old.local[r], self.n) for r in self.comm.ranks}
        inv_l = {r: _inverse(old.links[r], self.L) for r in self.comm.ranks}
        owner_a = old.owner[self._a]
        moves = {}

        def move(r, d):
            """What rank r sends rank d — the particles d did not hold and r owned, the
            links d did not hold whose end A r owned — as whole-set indices; every process
            computes the same."""
            if (r, d) not in moves:
                gp_, gl_ = new.local[d], new.links[d]
                need_p = gp_[~held_p[d][gp_]]
                need_l = gl_[~held_l[d][gl_]]
                moves[(r, d)] = (need_p[old.owner[need_p] == r], need_l[owner_a[need_l] == r])
            return moves[(r, d)]

        pkeys = sorted(states[0][0].keys())
        lkeys = sorted(states[0][1].keys())
        p_dt = {k: states[0][0][k].dtype for k in pkeys}
        l_dt = {k: states[0][1][k].dtype for k in lkeys}

        def nbytes(np_count, nl_count):
            tot = 0
            for k in pkeys:
                tot += np_count * p_dt[k].itemsize
            for k in lkeys:
                tot += (2 if k in abi.SIDE_FIELDS else 1) * nl_count * l_dt[k].itemsize
            return tot

        # pack: one byte buffer per (source rank of this process, destination)
        sends = {}
        for (p, l), r in zip(states, self.comm.ranks):
            dev = p["xCord"].device
            for d in range(R):
                if d == r:
                    continue
                need_p, need_l = move(r, d)
                if need_p.size == 0 and need_l.size == 0:
                    continue
                pi, li = inv_p[r][need_p], inv_l[r][need_l]
                pit = torch.from_numpy(pi.astype(np.int64)).to(dev)
                lit = torch.from_numpy(li.astype(np.int64)).to(dev)
                side = torch.stack([2 * lit, 2 * lit + 1], dim=1).reshape(-1)
                parts = [p[k].index_select(0, pit).view(torch.uint8) for k in pkeys]
                parts += [l[k].index_select(0, side if k in abi.SIDE_FIELDS else lit).view(torch.uint8)
                          for k in lkeys]
                sends[(r, d)] = torch.cat(parts)
        # what each rank of this process receives, and its size
        recv_sizes = {}
        for r in self.comm.ranks:
            for s_ in range(R):
                if s_ == r:
                    continue
                need_p, need_l = move(s_, r)
                if need_p.size or need_l.size:
                    recv_sizes[(s_, r)] = (need_p, need_l, nbytes(need_p.size, need_l.size))
        got = self.comm.exchange_tensors(sends, {k: v[2] for k, v in recv_sizes.items()},
                                         [st[0]["xCord"].device for st in states])
        # assemble each rank's new held set on its device
        out = []
        for (p, l), r in zip(states, self.comm.ranks):
            dev = p["xCord"].device
            gp, gl = new.local[r], new.links[r]
            # every position is filled below, from what was kept or what was received
            np_ = {k: torch.empty(gp.size, dtype=p_dt[k], device=dev) for k in pkeys}
            nl = {k: torch.empty((2 if k in abi.SIDE_FIELDS else 1) * gl.size, dtype=l_dt[k], device=dev)
                  for k in lkeys}
            pos = inv_p[r][gp]
            kept = pos >= 0
            at_t = torch.from_numpy(np.flatnonzero(kept)).to(dev)
            from_t = torch.from_numpy(pos[kept].astype(np.int64)).to(dev)
            for k in pkeys:
                np_[k][at_t] = p[k].index_select(0, from_t)
            lpos = inv_l[r][gl]
            lkept = lpos >= 0
            lat = torch.from_numpy(np.flatnonzero(lkept)).to(dev)
            lfrom = torch.from_numpy(lpos[lkept].astype(np.int64)).to(dev)
            lat2 = torch.stack([2 * lat, 2 * lat + 1], dim=1).reshape(-1)
            lfrom2 = torch.stack([2 * lfrom, 2 * lfrom + 1], dim=1).reshape(-1)
            for k in lkeys:
                if k in abi.SIDE_FIELDS:
                    nl[k][lat2] = l[k].index_select(0, lfrom2)
                else:
                    nl[k][lat] = l[k].index_select(0, lfrom)
            got_p, got_l = kept.copy(), lkept.copy()
            for s_ in range(R):
                if (s_, r) not in recv_sizes:
                    continue
                need_p, need_l, _ = recv_sizes[(s_, r)]
                buf = got[(s_, r)]
                off = 0
                at = torch.from_numpy(np.searchsorted(gp, need_p)).to(dev)
                for k in pkeys:
                    nb = need_p.size * p_dt[k].itemsize
                    np_[k][at] = buf[off: off + nb].view(p_dt[k])
                    off += nb
                lat = torch.from_numpy(np.searchsorted(gl, need_l)).to(dev)
                lat2 = torch.stack([2 * lat, 2 * lat + 1], dim=1).reshape(-1)
                for k in lkeys:
                    m = (2 if k in abi.SIDE_FIELDS else 1) * need_l.size
                    nb = m * l_dt[k].itemsize
                    vals = buf[off: off + nb].view(l_dt[k])
                    if k in abi.SIDE_FIELDS:
                        nl[k][lat2] = vals
                    else:
                        nl[k][lat] = vals
                    off += nb
                got_p[np.searchsorted(gp, need_p)] = True
                got_l[np.searchsorted(gl, need_l)] = True
            if not (got_p.all() and got_l.all()):
                raise RuntimeError(f"rank {r}: particles or links missing after the redistribution")
            np_["owners"] = torch.from_numpy(new.owner[gp].astype(np.int32)).to(dev)
            out.append((np_, nl))
        self.layout = new
        self._install(out)

    def gather(self) -> tuple[dict, dict]:
        """The whole set's particles and links (every process gets them)."""
        mine = [(lib.get_particles(), lib.get_links()) for lib in self.libs]
        parts = self.comm.allgather(mine)
        return merge_state(parts, self.layout, self.n, self.L)

    # -- one timestep
    def _grid_service(self) -> None:
        loc = [lib.grid_service_local() for lib in self.libs]
        if any(w for _, w in loc):
            # a step where gridService reads the displacement maxima (every 10th): their
            # maximum over all ranks, and the rebuild if any rank's policy asks for it
            mx = self.comm.allmax([m for m, _ in loc])
            regen = [np.array([1.0 if lib.grid_service_decide(mx) else 0.0]) for lib in self.libs]
            if not self.comm.allmax(regen)[0]:
                return
        else:
            # no maxima are read at this step, on any rank (every rank is at the same step
            # with the same policy): the decision depends only on the step and on whether
            # the context is built, which all ranks share, so it takes no collective
            if not any([lib.grid_service_decide(np.zeros(3)) for lib in self.libs]):
                return
        # Each rank's held set contains every contact partner of its own particles while
        # no particle has moved more than half the halo's room in x since the last
        # distribution (partners lie within the reach; each end moved at most that much):
        # then the rebuild keeps the held sets, else every particle goes to the owner of
        # its slab, the slabs are recut and the halos rebuilt.
        moved = [np.array([_max_moved(lib, x0)]) for lib, x0 in zip(self.libs, self._x0)]
        delta = float(self.comm.allmax(moved)[0])
        if 2.0 * delta > self._width - self._reach:
            self._redistribute()
        else:
            self.kept += 1
        bounds = [lib.local_bounds() for lib in self.libs]
        lo = -self.comm.allmax([-b[0] for b in bounds])
        hi = self.comm.allmax([b[1] for b in bounds])
        for lib in self.libs:
            lib.regenerate_frame(lo, hi)

    def _streams(self):
        """(context stream, the device's current stream) per context, when the halo buffers
        live in device memory and the contexts expose their streams; else None."""
        import torch
        if not (self.send_bufs and self.send_bufs[0].is_cuda):
            return None
        if not all(hasattr(lib, "stream_handle") for lib in self.libs):
            return None
        out = []
        for lib, buf in zip(self.libs, self.send_bufs):
            dev = buf.device
            out.append((torch.cuda.ExternalStream(lib.stream_handle, device=dev), torch.cuda.current_stream(dev)))
        return out

    def _forces(self) -> None:
        for lib, buf in zip(self.libs, self.send_bufs):
            if hasattr(lib, "compute_forces_packed"):
                lib.compute_forces_packed(buf.data_ptr())  # the pack in the force pass
            else:
                lib.computePartForce()
                lib.pack_halo_forces(buf.data_ptr())
        streams = self._streams()
        if streams is None:
            for lib in self.libs:
                lib.synchronize()
        else:
            # ordered on the devices instead of the host: the exchange (on the current
            # streams) after each context's pack, each context's unpack after the exchange
            for ctx_stream, cur in streams:
                cur.wait_stream(ctx_stream)
        self.comm.exchange(self.layout, self.send_bufs, self.recv_bufs)
        if streams is not None:
            for ctx_stream, cur in streams:
                ctx_stream.wait_stream(cur)
        for lib, r, buf in zip(self.libs, self.comm.ranks, self.recv_bufs):
            lib.unpack_halo_forces(buf.data_ptr())
            self.exchanged += sum(self.layout.recv_counts(r))

    def step(self, nsteps: int = 1) -> None:
        # the sample main's break gate (getCurrentTimestep() * dt > breakTime) from a step
        # count kept here, so that a timestep makes no host round trip for it
        t0 = self.libs[0].getCurrentTimestep()
        for k in range(nsteps):
            self._grid_service()
            self._forces()
            brk = self.libs[0].breakActive(t0 + k)
            for lib in self.libs:
                lib.applyForce()
                if brk:
                    lib.linkUpdate()
                lib.finalizeTs()
        for lib in self.libs:
            lib.synchronize()



def _mask(idx: np.ndarray, size: int) -> np.ndarray:
    m = np.zeros(size, bool)
    m[idx] = True
    return m


def _inverse(idx: np.ndarray, size: int) -> np.ndarray:
    """inv[idx[k]] = k, -1 elsewhere."""
    inv = np.full(size, -1, np.int32)
    inv[idx] = np.arange(idx.size, dtype=np.int32)
    return inv


def _max_moved(lib, x0) -> float:
    """The largest |x - x0| over a context's held particles, on the device when x0 is there."""
    if x0.shape[0] == 0:
        return 0.0
    if hasattr(x0, "is_cuda") and x0.is_cuda:
        x = lib.get_particles_device(fields=["xCord"])["xCord"]
        return float((x - x0).abs().max().item())
    return float(np.max(np.abs(lib.get_particles()["xCord"] - x0)))


def _lib_device(lib):
    import torch
    dev = getattr(lib, "device", 0)
    return torch.device("cuda", int(dev)) if torch.cuda.is_available() else torch.device("cpu")

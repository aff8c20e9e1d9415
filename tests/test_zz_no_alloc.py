"""hidem_bin_cells_noalloc: the binning of the rebuild for callers that cannot let the
library allocate device memory (applications that place every device buffer in their
own pool, loops that cannot take cudaMalloc's device-wide synchronisation). The caller
allocates the inputs and outputs (here with torch); the entry point itself allocates
nothing and keeps its scratch in one fixed device array. Two calls in a row, on inputs
of different sizes, must each reproduce the cells of the existing entry point
(hidem_regenerate + hidem_get_cells) exactly — cells are integers, so the tolerance is
zero — and the (cell, index) order those cells imply. This file is collected last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMLib

pytestmark = pytest.mark.gpu


def existing_cells(P, p):
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(abi.empty_links(0, int(P.precision)))
    lib.regenerate()
    ix, iy, iz, dims, mins = lib.get_cells()
    h = lib.stats()["search_distance"]
    lib.close()
    colour = ix.astype(np.int64) + dims[0] * (iy.astype(np.int64) + dims[1] * iz.astype(np.int64))
    return colour, dims, mins, h


def noalloc_cells(p, h):
    import torch
    lib = abi.load()
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(p["xCord"]).to(dev)
    y = torch.from_numpy(p["yCord"]).to(dev)
    z = torch.from_numpy(p["zCord"]).to(dev)
    n = x.numel()
    cell_of = torch.full((n,), -1, dtype=torch.int32, device=dev)
    order = torch.full((n,), -1, dtype=torch.int32, device=dev)
    dims = (C.c_int64 * 3)()
    mins = (C.c_double * 3)()
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.hidem_bin_cells_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), n, h,
                                     cell_of.data_ptr(), order.data_ptr(), dims, mins, stream)
    assert st == abi.HIDEM_OK, lib.hidem_create_error()
    torch.cuda.synchronize(dev)
    return cell_of.cpu().numpy(), order.cpu().numpy(), tuple(dims), tuple(mins)


def cloud(n, seed):
    rng = np.random.default_rng(seed)
    p = abi.empty_particles(n, abi.PREC_MIXED)
    p["xCord"][:] = rng.uniform(-3, 30, n)
    p["yCord"][:] = rng.uniform(0, 9, n)
    p["zCord"][:] = rng.uniform(-2, 5, n)
    p["radius"][:] = 0.5
    p["globalKeys"][:] = np.arange(n)
    return p


def test_noalloc_binning_matches_existing_entry_point_twice(gpu):
    _, block, _ = workloads.ice_block(cells=(12, 9, 7), precision=abi.PREC_MIXED, seed=4)
    inputs = [block, cloud(5000, 2)]  # two calls in a row, different sizes and grids
    P = abi.default_params(precision=abi.PREC_MIXED, searchDistanceScale=1.2)
    for p in inputs:
        colour, dims, mins, h = existing_cells(P, p)
        cell_of, order, ndims, nmins = noalloc_cells(p, h)
        assert ndims == tuple(dims) and nmins == tuple(mins)
        assert np.array_equal(cell_of.astype(np.int64), colour)
        n = colour.shape[0]
        assert np.array_equal(order, np.lexsort((np.arange(n), colour)).astype(np.int32))


def test_noalloc_refuses_grids_beyond_the_fixed_scratch(gpu):
    import torch
    lib = abi.load()
    dev = torch.device("cuda", 0)
    x = torch.tensor([0.0, 100.0], dtype=torch.float64, device=dev)
    y = torch.tensor([0.0, 100.0], dtype=torch.float64, device=dev)
    z = torch.tensor([0.0, 100.0], dtype=torch.float64, device=dev)
    out = torch.zeros(2, dtype=torch.int32, device=dev)
    dims = (C.c_int64 * 3)()
    mins = (C.c_double * 3)()
    st = lib.hidem_bin_cells_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), 2, 1.0,
                                     out.data_ptr(), out.data_ptr(), dims, mins, 0)
    assert st == 4  # HIDEM_ERR_CAPACITY: 101^3 cells > HIDEM_NOALLOC_MAX_CELLS
    assert b"HIDEM_NOALLOC_MAX_CELLS" in lib.hidem_create_error()


def _device_xyz(p):
    import torch
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(np.ascontiguousarray(p[k])).to(dev) for k in ("xCord", "yCord", "zCord")]


def _call(xyz, h):
    import torch
    lib = abi.load()
    n = xyz[0].numel()
    cell_of = torch.full((n,), -1, dtype=torch.int32, device=xyz[0].device)
    order = torch.full((n,), -1, dtype=torch.int32, device=xyz[0].device)
    dims = (C.c_int64 * 3)()
    mins = (C.c_double * 3)()
    st = lib.hidem_bin_cells_noalloc(xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr(), n, h,
                                     cell_of.data_ptr(), order.data_ptr(), dims, mins, 0)
    return st, lib.hidem_create_error(), cell_of.cpu().numpy(), order.cpu().numpy()


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_noalloc_refuses_non_finite_coordinates(gpu, bad):
    """One NaN (or infinite) coordinate written into the host input before upload."""
    p = cloud(3000, 5)
    p["yCord"][1234] = bad
    st, msg, _, _ = _call(_device_xyz(p), 1.2)
    assert st == abi.HIDEM_ERR_ARG and b"non-finite" in msg


def test_noalloc_orders_a_crowded_cell_and_refuses_an_overcrowded_one(gpu):
    """A cell_size that puts the whole cloud into one cell: up to 4096 members the order is
    still ascending input index; beyond, the call is refused instead of sorting for long."""
    p = cloud(4000, 6)
    st, msg, cell_of, order = _call(_device_xyz(p), 100.0)
    assert st == abi.HIDEM_OK, msg
    assert np.all(cell_of == 0) and np.array_equal(order, np.arange(4000, dtype=np.int32))
    p = cloud(4097, 6)
    st, msg, _, _ = _call(_device_xyz(p), 100.0)
    assert st == abi.HIDEM_ERR_CAPACITY and b"4096" in msg

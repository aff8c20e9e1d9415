"""The HDF5 reader on files in the layout libhdf5 writes (superblock 0, version-1 object
headers, symbol-table groups, chunked deflate / shuffle datasets): the reference's own
benchmark inputs where its tree is present, and files of every supported storage form made
by an independent encoder (tests/h5_legacy.py). Host code only: no GPU."""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np
import pytest

import h5_legacy as h5
from hidem_b200 import abi, workloads

REF = Path(os.environ.get("HIDEM_REFERENCE_TREE", "/root/reference"))
BENCH = REF / "HiDEM" / "Benchmark"
# particle counts of the benchmark inputs (the 5700k and 310k counts are the ones the
# reference's scaling plot quotes, HiDEM/Docs/Images/GPU_scaling.png)
KNOWN = {"5700k": 5723826, "310k": 318777}


def _benchmark_files():
    if not BENCH.is_dir():
        return []
    return sorted(p for p in BENCH.glob("*/particles.h5"))


@pytest.mark.parametrize("path", _benchmark_files(), ids=lambda p: p.parent.name)
def test_reads_the_reference_benchmark_inputs(path):
    p = workloads.read_particle_file(str(path), abi.PREC_MIXED)
    n = p["xCord"].shape[0]
    if path.parent.name in KNOWN:
        assert n == KNOWN[path.parent.name]
    assert n > 100000
    for k in ("xCord", "yCord", "zCord"):
        assert np.all(np.isfinite(p[k]))
    assert np.all(p["radius"] == 6.0)  # lattice.particleRadius 0.5 x general.scale 12
    # the File lattice is an FCC lattice of spacing 12 * 1.41421 (the values stored in double,
    # read as float): every coordinate is a whole number of half cells from the minimum
    half = 12 * 1.41421 / 2
    for k in ("xCord", "yCord", "zCord"):
        q = (p[k] - p[k].min()) / half
        assert np.abs(q - np.round(q)).max() < 2e-3
    assert np.array_equal(p["globalKeys"], np.arange(n))
    assert p["zCord"].min() >= 29.9 and p["zCord"].max() <= 330.0


def test_meshblock_input_builds_the_reference_run():
    cfg = BENCH / "5700k" / "config_mesh_5700k.toml"
    if not cfg.exists():
        pytest.skip("the reference tree is not present")
    P, p, l, info = workloads.meshblock(str(cfg), str(cfg.parent / "particles.h5"))
    assert p["xCord"].shape[0] == 5723826
    assert P.scale == 12.0 and P.maxRadius == 6.0 and P.dt == 0.0002 and P.breakTime == 5.0
    assert info["linkGenScale"] == 1.2
    deg = np.bincount(np.concatenate([l["globalKeyEndA"], l["globalKeyEndB"]]))
    assert deg.max() == 12  # FCC nearest neighbours at 12 m, the next shell at 17 m > 1.2 x 12


def _points(n, seed):
    rng = np.random.default_rng(seed)
    return {"xCord": rng.uniform(-50, 50, n), "yCord": rng.uniform(0, 9, n),
            "zCord": rng.uniform(30, 40, n), "radius": rng.uniform(0.4, 0.6, n).astype(np.float32)}


@pytest.mark.parametrize("form", ["contiguous", "compact", "chunked", "chunked_shuffle_deflate",
                                  "deflate_many_chunks", "continuation"])
def test_reads_each_storage_form(tmp_path, form):
    n = 777 if form == "compact" else 5000
    pts = _points(n, 3)
    kw = {}
    if form == "chunked":
        kw = dict(layout="chunked", chunk=(1024,))
    elif form == "chunked_shuffle_deflate":
        kw = dict(layout="chunked", chunk=(1500,), shuffle=True, deflate=6)
    elif form == "deflate_many_chunks":  # two B-tree levels, a partial last chunk
        kw = dict(layout="chunked", chunk=(256,), deflate=1)
    elif form == "continuation":
        kw = dict(layout="chunked", chunk=(700,), deflate=4, continuation=True)
    elif form == "compact":
        kw = dict(layout="compact")
    tree = {k: h5.Data(v, **kw) for k, v in pts.items()}
    # more entries than one symbol node holds, so the root group's B-tree has two levels
    for i in range(20):
        tree[f"extra_{i:02d}"] = h5.Data(np.arange(i + 1, dtype=np.int32), attrs={"idx": np.int32(i)})
    tree["sub"] = {"attrs": {"timeStep": np.int32(123)}, "inner": np.zeros(3)}
    path = tmp_path / "p.h5"
    h5.write(path, tree)
    for prec in (abi.PREC_MIXED, abi.PREC_FP64):
        p = workloads.read_particle_file(str(path), prec)
        for k in ("xCord", "yCord", "zCord"):
            assert np.array_equal(p[k], pts[k].astype(np.float32).astype(np.float64)), k
        assert np.array_equal(p["radius"], pts["radius"].astype(abi.lp_dtype(prec)))


def test_named_datasets_and_errors(tmp_path):
    pts = _points(100, 4)
    path = tmp_path / "named.h5"
    h5.write(path, {"X": pts["xCord"], "Y": pts["yCord"], "Z": pts["zCord"], "R": pts["radius"],
                    "short": np.zeros(5)})
    p = workloads.read_particle_file(str(path), abi.PREC_MIXED, ("X", "Y", "Z", "R"))
    assert np.array_equal(p["yCord"], pts["yCord"].astype(np.float32).astype(np.float64))
    with pytest.raises(abi.HidemError) as e:
        workloads.read_particle_file(str(path), abi.PREC_MIXED)  # no xCord
    assert e.value.status == abi.HIDEM_ERR_IO and "xCord" in str(e.value)
    with pytest.raises(abi.HidemError) as e:
        workloads.read_particle_file(str(path), abi.PREC_MIXED, ("X", "Y", "short", "R"))
    assert e.value.status == abi.HIDEM_ERR_IO
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(abi.HidemError) as e:
        workloads.read_particle_file(str(bad), abi.PREC_MIXED)
    assert e.value.status == abi.HIDEM_ERR_IO

"""The templated operator surface (include/hidem_b200_iterate.cuh): a sample main's own
functors, compiled by nvcc against the header (tests/iterate_harness.cu), run on the
library's device data. With functors that restate the default ones the results are the
library's own bit for bit; with the IceBlock sample's link functor
(HiDEM/IceBlock/MainIceBlock.cpp:173-262) they match the oracle's restatement of it."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import golden_inputs, load_golden
from hidem_b200 import abi, workloads
from hidem_b200.hidemlib import HiDEMLib
from oracle import oracle

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
P_OUT = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
         "uDiff", "vDiff", "wDiff"]
L_OUT = ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = tmp_path_factory.mktemp("harness") / "libiterate_harness.so"
    lib = ROOT / "hidem_b200"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3", "-fmad=false",
           "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC", "-shared", f"-I{ROOT / 'include'}",
           "-o", str(out), str(Path(__file__).with_name("iterate_harness.cu")), f"-L{lib}", "-lhidem_b200",
           f"-Xlinker=-rpath={lib}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    abi.load()  # the library first, so the harness binds to the same copy
    h = C.CDLL(str(out))
    h.harness_steps.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
    h.harness_forces.argtypes = [C.c_void_p, C.c_int]
    h.harness_apply.argtypes = [C.c_void_p, C.c_double]
    h.harness_iterate_count.argtypes = [C.c_void_p]
    h.harness_iterate_count.restype = C.c_longlong
    return h


def _lib(P, p, l):
    lib = HiDEMLib(P)
    lib.set_particles(p)
    lib.set_links(l)
    return lib


@pytest.mark.parametrize("name", ["block6_mixed", "block6_fp64"])
def test_default_functors_through_the_header_equal_the_library(gpu, harness, name):
    g = load_golden(name)
    P, p, l = golden_inputs(g)
    a = _lib(P, p, l)
    a.regenerate()
    a.computePartForce()
    a.synchronize()
    fa, la = a.get_forces(), a.get_links()
    b = _lib(P, p, l)
    b.regenerate()
    assert harness.harness_forces(b._ctx, 0) == 0
    fb, lb = b.get_forces(), b.get_links()
    assert np.array_equal(fa, fb)
    for k in L_OUT:
        assert np.array_equal(la[k], lb[k]), k
    n_contacts = int(b.stats()["num_neighbour_pairs"])
    assert harness.harness_iterate_count(b._ctx) == n_contacts  # Iterator::iterate over the slots
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
@pytest.mark.parametrize("user_break", [0, 1])
def test_sample_loop_with_caller_functors_matches_the_oracle(gpu, harness, precision, user_break):
    """gridService, computePartForce(caller's default-restating functors), the library's
    integrate, linkUpdate (the caller's break functor or the library's), finalizeTs — 40
    steps of a breaking block, bit-exact against the oracle."""
    P, p, l = workloads.ice_block(cells=(5, 4, 5), precision=precision, seed=12)
    lib = _lib(P, p, l)
    assert harness.harness_steps(lib._ctx, 0, user_break, 40, P.dt, P.breakTime) == 0
    out_p, out_l = lib.get_particles(), lib.get_links()
    li, st = lib.get_break_events()
    lib.close()
    ref = oracle.port().run(P, p, l, 40)
    for k in P_OUT:
        assert np.array_equal(out_p[k], ref[0][k]), k
    for k in L_OUT:
        assert np.array_equal(out_l[k], ref[1][k]), k
    order = np.lexsort((li, st))
    ev = np.stack([li[order], st[order]], axis=1) if len(li) else np.zeros((0, 2), np.int64)
    assert np.array_equal(ev.reshape(-1, 2), np.asarray(ref[3]).reshape(-1, 2))
    assert len(ref[3]) > 0  # the block fractures in these steps


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_iceblock_link_functor_matches_the_oracle(gpu, harness, precision):
    P, p, l = workloads.ice_block(cells=(5, 4, 4), precision=precision, seed=13)
    lib = _lib(P, p, l)
    assert harness.harness_steps(lib._ctx, 1, 1, 30, P.dt, P.breakTime) == 0
    out_p, out_l = lib.get_particles(), lib.get_links()
    lib.close()
    port = oracle.port()
    port.lib.hidem_oracle_set_link_variant(1)
    try:
        ref = port.run(P, p, l, 30)
    finally:
        port.lib.hidem_oracle_set_link_variant(0)
    for k in P_OUT:
        assert np.array_equal(out_p[k], ref[0][k]), k
    for k in L_OUT:
        assert np.array_equal(out_l[k], ref[1][k]), k
    # the variant is a different functor: its history differs from the default one's
    dflt = oracle.port().run(P, p, l, 30)
    assert not np.array_equal(ref[1]["CT1"], dflt[1]["CT1"])


def test_apply_force_with_a_caller_integrate(gpu, harness):
    P, p, l = workloads.ice_block(cells=(4, 4, 3), precision=abi.PREC_MIXED, seed=14)
    lib = _lib(P, p, l)
    lib.regenerate()
    lib.computePartForce()
    F = lib.get_forces()
    before = lib.get_particles()
    assert harness.harness_apply(lib._ctx, 1e-9) == 0
    after = lib.get_particles()
    lib.close()
    s = np.float32(1e-9)
    for c, (d, f) in enumerate([("xDiff", 0), ("yDiff", 1), ("zDiff", 2)]):
        nd = before[d] + s * F[f]
        assert np.array_equal(after[d], nd), d
        xc = "xyz"[c] + "Cord"
        assert np.array_equal(after[xc], before[xc] + nd.astype(np.float64)), xc
    assert np.array_equal(after["zTheta"], before["zTheta"] + s * F[5])
    assert np.array_equal(after["uDiff"], before["uDiff"])

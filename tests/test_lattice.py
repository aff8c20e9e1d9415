"""Setup-side generators (host code of the library) against the reference's
LinkGenerator and the known answer that an interior FCC site has 12 bonds
(CatchTests/LinkGeneratorTester.cpp:129,197,256)."""
from __future__ import annotations

import numpy as np
import pytest

from hidem_b200 import abi, workloads
from oracle import oracle


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_fcc_interior_site_has_twelve_links(precision):
    p = workloads.fcc_particles(5, 5, 5, precision, jitter=0.0)
    l = workloads.distance_links(p, precision, 1.01)
    deg = np.bincount(np.concatenate([l["globalKeyEndA"], l["globalKeyEndB"]]), minlength=500)
    x, y, z = p["xCord"], p["yCord"], p["zCord"]
    a = workloads.SQRT2
    interior = (x > a) & (x < 4 * a - 0.1) & (y > a) & (y < 4 * a - 0.1) & (z > a) & (z < 4 * a - 0.1)
    assert interior.sum() > 0 and np.all(deg[interior] == 12)
    assert deg.max() == 12


def test_lattice_is_deterministic_and_seeded():
    a = workloads.fcc_particles(3, 3, 3, abi.PREC_MIXED, seed=5)
    b = workloads.fcc_particles(3, 3, 3, abi.PREC_MIXED, seed=5)
    c = workloads.fcc_particles(3, 3, 3, abi.PREC_MIXED, seed=6)
    assert np.array_equal(a["xCord"], b["xCord"]) and not np.array_equal(a["xCord"], c["xCord"])
    assert np.all(np.abs(a["xCord"] - workloads.fcc_particles(3, 3, 3, abi.PREC_MIXED, jitter=0)["xCord"]) <= 0.01)


@pytest.mark.skipif(not oracle.reference_available(abi.PREC_MIXED), reason="oracle/_ref not built")
@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_link_set_matches_reference_link_generator(precision):
    import ctypes as C
    if not oracle.reference_available(precision):
        pytest.skip("oracle/_ref not built")
    p = workloads.fcc_particles(6, 5, 4, precision, jitter=0.01, seed=2)
    ours = workloads.distance_links(p, precision, 1.01)
    ref = oracle.reference(precision)
    lib = ref.lib
    lib.hidem_ref_links.argtypes = [C.POINTER(abi.HidemParticleSoA), C.c_int64, C.c_double,
                                    C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                    C.POINTER(C.c_int64)]
    n = p["xCord"].shape[0]
    cap = 20 * n
    ka, kb = np.zeros(cap, np.int64), np.zeros(cap, np.int64)
    L0 = np.zeros(cap, abi.lp_dtype(precision))
    cnt = C.c_int64()
    soa = abi.particle_soa(p, precision, n)
    assert lib.hidem_ref_links(C.byref(soa), n, 0.5, 1.01, ka.ctypes.data, kb.ctypes.data,
                               L0.ctypes.data, cap, C.byref(cnt)) == 0
    k = cnt.value
    ref_set = {(int(a), int(b)): float(x) for a, b, x in zip(ka[:k], kb[:k], L0[:k])}
    our_set = {(int(a), int(b)): float(x) for a, b, x in
               zip(ours["globalKeyEndA"], ours["globalKeyEndB"], ours["initialLen"])}
    assert our_set == ref_set


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
@pytest.mark.parametrize("jitter", [0.0, 0.01])
def test_numpy_inputs_equal_the_library_generators(precision, jitter):
    """hidem_b200.inputs_np (the reference arm's inputs, built without the library) gives the
    library generators' arrays and parameters bit for bit."""
    from hidem_b200 import inputs_np
    P, p, l = workloads.calving_slab(size=(30.0, 12.0, 9.0), precision=precision, jitter=jitter, seed=3)
    Q, q, m = inputs_np.calving_slab(size=(30.0, 12.0, 9.0), precision=precision, jitter=jitter, seed=3)
    for k in p:
        assert np.array_equal(p[k], q[k]), k
    for k in l:
        assert np.array_equal(l[k], m[k]), k
    assert bytes(P) == bytes(Q)
    assert bytes(inputs_np.default_params()) == bytes(abi.default_params())


def test_reference_arm_maps_no_library_code(tmp_path):
    """bench.py --impl reference runs the reference's CPU path on inputs it builds in numpy:
    its process never maps libhidem_b200.so."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--slab', '20,9,9', "
            "'--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPPED' if 'libhidem_b200.so' in maps else 'CLEAN'); "
            "print('REF' if 'libhidem_ref_fast' in maps else 'NOREF')")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = r.stdout.strip().splitlines()
    if "unavailable" in out[0]:
        pytest.skip("oracle/_ref not built")
    assert out[-2] == "CLEAN" and out[-1] == "REF"

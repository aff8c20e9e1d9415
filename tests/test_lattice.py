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

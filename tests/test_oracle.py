"""The oracle (oracle/hidem_oracle.c) pinned against the reference's own CPU path:
committed golden fixtures (made by tests/golden/make_golden.py from oracle/_ref), live
comparisons with oracle/_ref when it is built, and the known answers of the reference's
grid tests (CatchTests/NeighbourGridTester.cpp:11-165)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_inputs, load_golden
from hidem_b200 import abi, workloads
from oracle import oracle

GOLDEN = ["block6_mixed", "block6_fp64", "slab533_mixed", "slab533_fp64"]
P_OUT = ["xCord", "yCord", "zCord", "xTheta", "yTheta", "zTheta", "xDiff", "yDiff", "zDiff",
         "uDiff", "vDiff", "wDiff"]
L_OUT = ["state", "CT0", "CT1", "CT2", "CT3", "CT4", "CT5"]


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_reproduces_reference_golden_bit_exact(name):
    g = load_golden(name)
    P, p, l = golden_inputs(g)
    port = oracle.port()
    ix, iy, iz, dims, mins = port.cells(P, p)
    assert np.array_equal(np.stack([ix, iy, iz]), g["cells"])
    assert tuple(dims) == tuple(g["dims"]) and np.array_equal(np.array(mins), g["mins"])
    counts, nlist = port.neighbours(P, p)
    assert np.array_equal(counts, g["nbr_counts"]) and np.array_equal(nlist, g["nbr_list"])
    p1, l1, F, events, regen, _ = port.run(P, p, l, int(g["steps"]))
    for k in P_OUT:
        assert np.array_equal(p1[k], g["out_p_" + k]), k
    for k in L_OUT:
        assert np.array_equal(l1[k], g["out_l_" + k]), k
    assert np.array_equal(F, g["out_force"])
    assert np.array_equal(events, g["out_events"])
    assert np.array_equal(regen, g["out_regen"])


needs_ref = pytest.mark.skipif(not (oracle.reference_available(abi.PREC_MIXED)
                                    and oracle.reference_available(abi.PREC_FP64)),
                               reason="oracle/_ref not built (needs the reference sources)")


@needs_ref
@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
@pytest.mark.parametrize("variant", ["block", "bed_front_limits", "regen_rule", "attract"])
def test_oracle_matches_reference_live(precision, variant):
    over = {}
    if variant == "block":
        P, p, l = workloads.ice_block(cells=(5, 4, 6), precision=precision, seed=11)
        steps = 40
    elif variant == "bed_front_limits":
        P, p, l = workloads.calving_slab(size=(7.0, 4.3, 4.3), precision=precision, seed=2,
                                         broken_fraction=0.1, water_level=3.0,
                                         useVelocityLimit=1, maxVel=0.05, maxRot=0.01,
                                         useBoundary=1, lowerLimit=(0.2, 0.2, -9), upperLimit=(5, 3, 9),
                                         boundaryMin=(1, 1, 1), boundaryMax=(1, 1, 0))
        steps = 30
    elif variant == "regen_rule":
        # fast-rising block so the displacement rule triggers rebuilds: the rule takes the
        # signed maximum of the diffs (HiDEMLib.h:436-458), so the motion must be +z
        P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=precision, seed=4,
                                      fixed_bottom=False, g=-9.81e4, waterLevel=-1e3,
                                      firstBalanceTimestep=30)
        steps = 60
    else:
        P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=precision, seed=9, jitter=0.05,
                                      attractDistance=0.05, attractScaleForce=0.3, bendBreak=2.0)
        steps = 30
    port = oracle.port()
    ref = oracle.reference(precision)
    a = port.run(P, p, l, steps)
    b = ref.run(P, p, l, steps)
    for k in P_OUT:
        assert np.array_equal(a[0][k], b[0][k]), k
    for k in L_OUT:
        assert np.array_equal(a[1][k], b[1][k]), k
    assert np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])
    assert np.array_equal(a[4], b[4])
    if variant == "regen_rule":
        assert len(a[4]) > 2  # the rule fired beyond step 0 and firstBalanceTimestep


@needs_ref
@needs_ref
@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_oracle_bed_and_force_maps_match_reference(precision):
    """GlacierDem bed height / friction maps and external force maps: the restatement's
    interpolation and integrate terms against the reference's own Map2d."""
    from conftest import maps_case
    P, p, l, (bed, fric, ext), keep = maps_case(precision)
    port = oracle.port()
    ref = oracle.reference(precision)
    port.set_maps(bed, fric, ext)
    ref.set_maps(bed, fric, ext)
    try:
        a = port.run(P, p, l, 40)
        b = ref.run(P, p, l, 40)
    finally:
        port.set_maps()
        ref.set_maps()
    for k in P_OUT:
        assert np.array_equal(a[0][k], b[0][k]), k
    for k in L_OUT:
        assert np.array_equal(a[1][k], b[1][k]), k
    assert np.array_equal(a[3], b[3])
    # the maps mattered: the same run without them differs
    c = port.run(P, p, l, 40)
    assert not np.array_equal(a[0]["zCord"], c[0]["zCord"])


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_oracle_collision_mesh_matches_reference(precision):
    """Collision mesh of the MeshConstrainedDem sample: the restatement's MeshAccel grid
    (bounds, counts, per-cell triangle lists) equals the reference's own generateAccel;
    trajectories with the closest-triangle force are bit-exact; face forces (atomic sums in
    the reference) agree to rounding."""
    from conftest import mesh_case
    P, p, l, m, keep = mesh_case(precision)
    port = oracle.port()
    ref = oracle.reference(precision)
    port.set_mesh(m)
    ref.set_mesh(m)
    try:
        ga, gb = port.mesh_accel(precision), ref.mesh_accel(precision)
        for k in ("counts", "lower", "upper", "sizes", "starts", "values"):
            assert np.array_equal(ga[k], gb[k]), k
        assert ga["values"].shape[0] > 100 and np.all(np.diff(ga["values"][: ga["sizes"][0]]) > 0)
        a = port.run(P, p, l, 40)
        b = ref.run(P, p, l, 40)
        fa, fb = port.mesh_face_forces(precision), ref.mesh_face_forces(precision)
    finally:
        port.set_mesh()
        ref.set_mesh()
    for k in P_OUT:
        assert np.array_equal(a[0][k], b[0][k]), k
    for k in L_OUT:
        assert np.array_equal(a[1][k], b[1][k]), k
    assert np.array_equal(a[2], b[2])
    tol = (1e-5 if precision == abi.PREC_MIXED else 1e-12) * float(np.abs(fb).max())
    assert (np.abs(fb).sum(axis=1) > 0).sum() >= 10
    assert np.abs(fa.astype(np.float64) - fb).max() <= tol
    # the mesh mattered: the same run without it differs
    c = port.run(P, p, l, 40)
    assert not np.array_equal(a[0]["zCord"], c[0]["zCord"])


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_oracle_collision_mesh_cloud_matches_reference(precision):
    from conftest import mesh_cloud_case
    P, p, l, m, keep = mesh_cloud_case(precision)
    port = oracle.port()
    ref = oracle.reference(precision)
    port.set_mesh(m)
    ref.set_mesh(m)
    try:
        a = port.run(P, p, l, 3)
        b = ref.run(P, p, l, 3)
    finally:
        port.set_mesh()
        ref.set_mesh()
    for k in P_OUT:
        assert np.array_equal(a[0][k], b[0][k]), k


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_oracle_contact_list_matches_reference_on_irregular_input(precision):
    rng = np.random.default_rng(5)
    n = 3000
    p = abi.empty_particles(n, precision)
    p["xCord"][:] = rng.uniform(0, 20, n)
    p["yCord"][:] = rng.uniform(0, 7, n)
    p["zCord"][:] = rng.uniform(-3, 3, n)
    p["radius"][:] = rng.uniform(0.2, 0.5, n)
    p["globalKeys"][:] = np.arange(n)
    P = abi.default_params(precision=precision, maxRadius=0.5, searchDistanceScale=1.3)
    a = oracle.port().neighbours(P, p)
    b = oracle.reference(precision).neighbours(P, p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    ca = oracle.port().cells(P, p)
    cb = oracle.reference(precision).cells(P, p)
    for x, y in zip(ca[:3], cb[:3]):
        assert np.array_equal(x, y)


# ---- known answers of CatchTests/NeighbourGridTester.cpp --------------------------

def lattice_points(nx, ny, nz, shuffle_seed=None):
    pts = np.array([(x, y, z) for x in range(nx) for y in range(ny) for z in range(nz)], float)
    if shuffle_seed is not None:
        pts = pts[np.random.default_rng(shuffle_seed).permutation(len(pts))]
    return pts


def particles_at(pts, precision=abi.PREC_MIXED, radius=0.1):
    n = len(pts)
    p = abi.empty_particles(n, precision)
    p["xCord"][:], p["yCord"][:], p["zCord"][:] = pts[:, 0], pts[:, 1], pts[:, 2]
    p["radius"][:] = radius
    p["globalKeys"][:] = np.arange(n)
    return p


def spacing_params(h):
    # searchDistance = searchDistanceScale * 2 * maxRadius = h
    return abi.default_params(searchDistanceScale=2.0, maxRadius=h / 4.0)


def test_kat_grid_dims_cubic_and_asymmetric():
    ix, iy, iz, dims, _ = oracle.port().cells(spacing_params(1.0), particles_at(lattice_points(3, 3, 3)))
    assert dims == (3, 3, 3)
    _, _, _, dims, _ = oracle.port().cells(spacing_params(1.0), particles_at(lattice_points(2, 3, 4)))
    assert dims == (2, 3, 4)


def test_kat_shuffled_box_spacing_two_gives_27_cells_of_8():
    pts = lattice_points(6, 6, 6, shuffle_seed=1)
    ix, iy, iz, dims, _ = oracle.port().cells(spacing_params(2.0), particles_at(pts))
    assert dims == (3, 3, 3)
    colour = ix + 3 * iy + 9 * iz
    counts = np.bincount(colour, minlength=27)
    assert len(np.unique(colour)) == 27 and counts[0] == 8 and np.all(counts == 8)


def test_kat_iteration_order_groups_by_cell():
    pts = np.array([[0, 0, 0], [1, 0, 0], [0.1, 0, 0], [1.1, 0, 0]], float)
    ix, iy, iz, dims, _ = oracle.port().cells(spacing_params(1.0), particles_at(pts))
    assert dims == (2, 1, 1)
    assert list(ix) == [0, 1, 0, 1]


def test_kat_small_spacing_gives_no_neighbours():
    P = spacing_params(0.2)
    counts, lst = oracle.port().neighbours(P, particles_at(lattice_points(3, 3, 3), radius=0.05))
    assert counts.sum() == 0 and lst.size == 0

"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and the built library; the
rest run on CPU (oracle, host logic, ABI surface)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libhidem_b200.so")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.skip("no CUDA device")
    return 0


def load_golden(name: str) -> dict:
    return dict(np.load(GOLDEN / f"{name}.npz"))


def golden_inputs(g: dict):
    """(params, particles, links) of a golden fixture."""
    from hidem_b200 import abi
    pdict = {k[len("param_"):]: v for k, v in g.items() if k.startswith("param_")}
    over = {}
    for k, v in pdict.items():
        over[k] = v.tolist() if v.ndim else v.item()
    P = abi.default_params(**over)
    p = {k[len("in_p_"):]: v.copy() for k, v in g.items() if k.startswith("in_p_")}
    l = {k[len("in_l_"):]: v.copy() for k, v in g.items() if k.startswith("in_l_")}
    return P, p, l


def maps_case(precision):
    """A 4^3-cell block resting on a GlacierDem bed map (some particles below the bed,
    most within bedInteract), with a friction map and six external force maps; returns
    (params, particles, links, (bed, friction, ext), arrays to keep alive)."""
    from hidem_b200 import abi, workloads
    P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=precision, seed=21, fixed_bottom=False,
                                  useBed=1, bedInteract=2.0, bedFriction=0.3, waterLevel=2.0)
    nx, ny = 13, 9
    xs = np.linspace(-1.0, 7.0, nx)
    ys = np.linspace(-1.0, 7.0, ny)
    X, Y = np.meshgrid(xs, ys)  # [ny][nx], x fastest
    zmin = float(p["zCord"].min())
    bed_v = zmin + 0.3 * np.sin(0.9 * X) + 0.2 * np.cos(1.3 * Y) + 0.1
    fric_v = 0.3 + 0.1 * np.sin(X + Y)
    keep = []
    bed, a = abi.map2d(bed_v, -1.0, -1.0, 7.0, 7.0, precision)
    keep.append(a)
    fric, a = abi.map2d(fric_v, -1.0, -1.0, 7.0, 7.0, precision)
    keep.append(a)
    ext = []
    for k in range(6):
        v = (2000.0 if k < 3 else 50.0) * np.cos(0.7 * X + 0.4 * k) * np.sin(0.5 * Y - 0.3 * k)
        m, a = abi.map2d(v, -1.5, -0.5, 6.5, 7.5, precision)
        ext.append(m)
        keep.append(a)
    return P, p, l, (bed, fric, ext), keep


def mesh_case(precision, cell_size=2.0):
    """A 4^3-cell block in a container mesh (bed with a slope and a bump just under the
    lowest particles, walls 0.3 m from the block's x and y faces), plus one degenerate
    triangle (its three vertices equal); returns (params, particles, links, mesh struct,
    arrays to keep alive)."""
    from hidem_b200 import abi, workloads
    P, p, l = workloads.ice_block(cells=(4, 4, 4), precision=precision, seed=23, fixed_bottom=False,
                                  bedInteract=0.4, waterLevel=2.0)
    lo = (float(p["xCord"].min()) - 0.8, float(p["yCord"].min()) - 0.8)
    hi = (float(p["xCord"].max()) + 0.8, float(p["yCord"].max()) + 0.8, float(p["zCord"].max()) + 2.0)
    z0 = float(p["zCord"].min()) - 0.7

    def bed(x, y):
        return z0 + 0.05 * (x - lo[0]) + 0.2 * np.exp(-((x - 3.0) ** 2 + (y - 2.5) ** 2))

    v, nrm = workloads.container_mesh(lo, hi, bed, nx=6, ny=5)
    v = np.concatenate([v, np.full((1, 3, 3), 2.0)])
    nrm = np.concatenate([nrm, [[0.0, 0.0, -1.0]]])
    m, keep = abi.mesh(v, nrm, cell_size, precision, mesh_force=2e6, mesh_drag=500.0)
    return P, p, l, m, keep


def mesh_cloud_case(precision, seed=5):
    """Unbonded particles on a jittered 1.1 m grid filling the lower part of a container
    mesh with a bumpy bed, many of them near the interaction distance of the bed or a wall
    and near the MeshAccel cell faces (cells of 1.7 m); returns (params, particles, empty
    links, mesh struct, arrays to keep alive)."""
    from hidem_b200 import abi, workloads
    rng = np.random.default_rng(seed)
    lo, hi = (0.0, 0.0), (14.0, 9.0, 8.0)

    def bed(x, y):
        return 0.4 * np.sin(0.7 * x) * np.cos(0.5 * y) + 0.05 * x

    g = np.mgrid[0.6:13.5:1.1, 0.6:8.5:1.1, 0.0:3.3:1.1].reshape(3, -1).T
    g = g + rng.uniform(-0.2, 0.2, g.shape)
    g[:, 2] += bed(g[:, 0], g[:, 1]) + 0.35
    n = g.shape[0]
    p = abi.empty_particles(n, precision)
    p["xCord"][:], p["yCord"][:], p["zCord"][:] = g[:, 0], g[:, 1], g[:, 2]
    p["radius"][:] = 0.5
    p["globalKeys"][:] = np.arange(n)
    P = workloads.block_params(precision, bedInteract=0.15, waterLevel=1.0)
    l = abi.empty_links(0, precision)
    v, nrm = workloads.container_mesh(lo, hi, bed, nx=10, ny=7)
    m, keep = abi.mesh(v, nrm, 1.7, precision, mesh_force=2e5, mesh_drag=300.0)
    return P, p, l, m, keep

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

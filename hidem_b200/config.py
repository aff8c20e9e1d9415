"""TOML run config (the reference's config files and `--section.key=value` overrides) to
``HidemParams`` through the library's ``hidem_params_from_toml``."""
from __future__ import annotations

import ctypes as C

from . import abi


def params_from_toml(path: str | None, overrides: list[str] | None = None):
    """Returns (HidemParams, iteration.timeSteps)."""
    lib = abi.load()
    args = overrides or []
    argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
    p = abi.HidemParams()
    steps = C.c_int64()
    st = lib.hidem_params_from_toml(path.encode() if path else None, len(args), argv,
                                    C.byref(p), C.byref(steps))
    if st != abi.HIDEM_OK:
        raise abi.HidemError(st, lib.hidem_create_error().decode())
    return p, steps.value

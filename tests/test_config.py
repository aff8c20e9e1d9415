"""TOML run-config front-end (hidem_params_from_toml) against Python's tomllib on the
keys the sample main reads, with the reference's command-line override rules."""
from __future__ import annotations

import tomllib

import pytest

from hidem_b200 import abi
from hidem_b200.config import params_from_toml

CONFIG = """
[general]
# same layout as the reference's MeshBlock benchmark configs
scale = 12.0
g = 9.81
beamWidth = 0.5
E = 2e+9
waterLevel = 300.0   # trailing comment
maxVel = 20.0
bedStiffness = 2e+8
damping = 10_000.0
dampingRotation = 10000.0
maxLoad = 5e-4
bendBreak = 0.01
attractDistance = 0.01
attractScaleForce = 1e-5
xBoundaryMin = false
yBoundaryMax = true
dt = 0.0002
breakTime = 5.0
precision = "fp64"
lowerLimit = [ -1.0, -2.0,
               -3.0 ]

[iteration]
timeSteps = 600000

[output]
outWorkingPath = "../Data/#not-a-comment"
statIntervals = [1000,10000,
                 25000,30000]

[grid]
searchDistanceScale = 1.4
gridRegenInterval = -1

[distribution]
firstBalanceTimestep = 200

[lattice]
type = "File"
particleRadius = 0.5
linkGenScale = 1.2

[[iceParameters]]
linkGenerateProbability = 1.0
"""


def test_toml_keys_match_tomllib(tmp_path):
    f = tmp_path / "config.toml"
    f.write_text(CONFIG)
    ref = tomllib.loads(CONFIG)
    p, steps = params_from_toml(str(f))
    g = ref["general"]
    for k in ["scale", "g", "beamWidth", "E", "waterLevel", "maxVel", "bedStiffness", "damping",
              "dampingRotation", "maxLoad", "bendBreak", "attractDistance", "attractScaleForce",
              "dt", "breakTime"]:
        assert getattr(p, k) == g[k], k
    assert p.searchDistanceScale == ref["grid"]["searchDistanceScale"]
    assert p.gridRegenInterval == -1 and p.firstBalanceTimestep == 200
    assert p.maxRadius == ref["lattice"]["particleRadius"] * g["scale"]
    assert steps == 600000
    assert list(p.boundaryMin) == [0, 0, 0] and list(p.boundaryMax) == [0, 1, 0]
    assert list(p.lowerLimit) == [-1.0, -2.0, -3.0]
    assert p.precision == abi.PREC_FP64
    # keys not in the file keep the sample defaults
    assert p.rhoIce == 910.0 and p.airDrag == 1.0 and p.maxRot == 5.0


def test_command_line_overrides_win(tmp_path):
    f = tmp_path / "config.toml"
    f.write_text(CONFIG)
    p, _ = params_from_toml(str(f), ["--general.dt=0.0001", "--grid.gridRegenInterval", "50",
                                     "--general.xBoundaryMin"])
    assert p.dt == 0.0001 and p.gridRegenInterval == 50 and p.boundaryMin[0] == 1


def test_bad_files_are_io_errors(tmp_path):
    with pytest.raises(abi.HidemError) as e:
        params_from_toml(str(tmp_path / "missing.toml"))
    assert e.value.status == 5
    f = tmp_path / "bad.toml"
    f.write_text("[general]\ndt = fast\n")
    with pytest.raises(abi.HidemError) as e:
        params_from_toml(str(f))
    assert e.value.status == 5 and "general.dt" in str(e.value)


def test_overrides_without_file_start_from_defaults():
    p, steps = params_from_toml(None, ["--general.E=3e9"])
    assert p.E == 3e9 and p.dt == 0.0001 and steps == 10000

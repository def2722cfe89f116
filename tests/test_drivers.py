"""The reference's six example executables rebuilt over the C++ facade (drivers/mgp_drivers.cpp,
one per test problem) against the reference's own builds of the same executables
(tests/golden/drivers.json, made by tests/golden/make_driver_golden.py): stdout, the -stats
rows and the SHA-256 of the binary VTK files of u, f and r, with wall-clock times and the
thread count masked.  The CPU test builds the executables and checks that they fail cleanly
without a device."""
import importlib.util
import json
import subprocess
import tempfile
from pathlib import Path

import pytest

from conftest import GOLDEN

spec = importlib.util.spec_from_file_location("make_driver_golden", GOLDEN / "make_driver_golden.py")
mdg = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mdg)

CASES = json.loads((GOLDEN / "drivers.json").read_text())


@pytest.fixture(scope="module")
def drivers(mgp_mod):
    return {p.name: p for p in mgp_mod._build.build_drivers()}


def test_fixture_covers_every_driver_and_problem():
    assert sorted(CASES) == sorted(f"{a}_p{p}" for a in mdg.APPS for p in (1, 2, 3))
    for c in CASES.values():
        assert len(c["vtk_sha256"]) == 3
        assert any(l.startswith("   0: Initial residual:") for l in c["stdout"])


def test_driver_without_device_fails_cleanly(mgp_mod, drivers):
    if mgp_mod.device_count() > 0:
        pytest.skip("a GPU is visible")
    with tempfile.TemporaryDirectory() as d:
        p = subprocess.run([str(drivers["vcycle_p1"]), *mdg.ARGS], cwd=d, capture_output=True, text=True, timeout=120)
    assert p.returncode != 0
    assert "device" in (p.stderr + p.stdout).lower()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_driver_matches_reference_executable(gpu_ready, drivers, name):
    case = CASES[name]
    got = mdg.run_case(drivers[name], case["args"])
    assert got["stdout"] == case["stdout"]
    assert got["stats"] == case["stats"]
    assert got["vtk_sha256"] == case["vtk_sha256"]

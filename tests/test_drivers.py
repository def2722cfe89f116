"""The reference's six example executables rebuilt over the C++ facade (drivers/mgp_drivers.cpp,
one per test problem) against the reference's own builds of the same executables
(tests/golden/drivers.json, made by tests/golden/make_driver_golden.py): stdout, the -stats
rows and the SHA-256 of the binary VTK files of u, f and r, with wall-clock times and the
thread count masked; and a user program written against the facade (tests/cpp/facade_user.cpp)
against the reference's own solver run the same way (tests/golden/facade_user.json).  The CPU
tests build the executables and the program and check that the drivers fail cleanly without a
device."""
import importlib.util
import json
import re
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


# ---- a user program written against the facade (tests/cpp/facade_user.cpp) ---------------------
FACADE_CASE = json.loads((GOLDEN / "facade_user.json").read_text())


@pytest.fixture(scope="module")
def facade_user(mgp_mod, tmp_path_factory):
    """Compiled against the facade headers and libmgp.so, as a user's code would be."""
    b = mgp_mod._build
    b.build()
    exe = tmp_path_factory.mktemp("facade") / "facade_user"
    src = Path(__file__).parent / "cpp" / "facade_user.cpp"
    subprocess.check_call(["g++", "-std=c++17", "-O2", f"-I{b.FACADE}", f"-I{b.INCLUDE}", str(src), f"-L{b.PKG}",
                           "-lmgp", f"-Wl,-rpath,{b.PKG}", "-o", str(exe)])
    return exe


def test_facade_user_program_compiles(facade_user):
    assert facade_user.exists()


@pytest.mark.gpu
def test_facade_user_program_matches_reference(gpu_ready, facade_user, tmp_path):
    """init_zero, get_rhs(0).at[idx], get_top_bc(0).arr, verbose solve with an ofile log,
    to_host, get_solution: the solution's bits, the verbose residual lines and the log's
    residual column equal the reference's own solver run the same way."""
    import hashlib

    import numpy as np

    u_bin, log = tmp_path / "u.bin", tmp_path / "ofile.txt"
    p = subprocess.run([str(facade_user), str(u_bin), str(log)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    u = np.fromfile(u_bin, dtype=np.float64)
    assert hashlib.sha256(u.tobytes()).hexdigest() == FACADE_CASE["u_sha256"]
    verbose = [" ".join(line.split()) for line in p.stdout.splitlines() if re.match(r"^\s*\d+:", line)]
    assert verbose == FACADE_CASE["verbose"]
    lines = log.read_text().splitlines()
    assert lines[0] == FACADE_CASE["ofile_header"]
    assert [line.split()[1] for line in lines[1:]] == FACADE_CASE["ofile_rel_res"]

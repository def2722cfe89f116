"""Generate tests/golden/drivers.json from the reference's own example executables.

Run where the reference sources are present:

    REF_DIR=<reference source dir> python tests/golden/make_driver_golden.py

The executables (its drivers/*.cpp, one per test problem) are built for the CPU by
oracle/build_ref_drivers.sh.  Each case runs one of them in a scratch directory and records
what a user of the reference sees: stdout, the rows appended by -stats, and the SHA-256 of
the VTK files written by -s (binary big-endian doubles, so equal digests mean bit-identical
u, f and r).  Wall-clock times and the OpenMP thread count are masked (see normalise());
everything else must match the B200 build of the same drivers exactly.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent

APPS = ("fcycle", "vcycle", "mixed", "dirichlet", "neumann", "gaussseidel")
ARGS = ["-x", "33", "-y", "17", "-z", "17", "-l", "3", "-maxiter", "4", "-s", "-stats", "stats.txt"]
CASES = {f"{app}_p{p}": (app, p, ARGS) for app in APPS for p in (1, 2, 3)}


def normalise(stdout: str) -> list:
    """stdout without its timings: the per-cycle "... took t seconds" lines are dropped, the
    total time and the thread count are masked."""
    out = []
    for line in stdout.splitlines():
        if re.match(r"^[VF]cycle took ", line):
            continue
        line = re.sub(r"^It took \S+ seconds", "It took <t> seconds", line)
        line = re.sub(r"^MG running on \d+ threads", "MG running on <n> threads", line)
        out.append(line)
    return out


def stats_rows(text: str) -> list:
    """-stats rows with the seconds column (first) and, in the 10-column form, the threads
    column (ninth) removed; header lines kept as they are."""
    rows = []
    for line in text.splitlines():
        if line.startswith("#"):
            rows.append(line)
            continue
        cols = line.split()
        if len(cols) == 10:
            cols = cols[1:8] + cols[9:]
        else:
            cols = cols[1:]
        rows.append(" ".join(cols))
    return rows


def run_case(exe: Path, args: list, env=None) -> dict:
    with tempfile.TemporaryDirectory() as d:
        (Path(d) / "results").mkdir()
        p = subprocess.run([str(exe), *args], cwd=d, capture_output=True, text=True, timeout=600, env=env)
        if p.returncode != 0:
            raise RuntimeError(f"{exe.name} exited {p.returncode}: {p.stderr[-2000:]}")
        stats = ""
        for cand in (Path(d) / "results" / "stats.txt", Path(d) / "stats.txt"):
            if cand.exists():
                stats += cand.read_text()
        vtk = {f.name: hashlib.sha256(f.read_bytes()).hexdigest() for f in sorted((Path(d) / "results").glob("*.vtk"))}
        return {"stdout": normalise(p.stdout), "stats": stats_rows(stats), "vtk_sha256": vtk}


def main():
    ref_dir = os.environ.get("REF_DIR") or (sys.argv[1] if len(sys.argv) > 1 else "")
    if not ref_dir:
        raise SystemExit("set REF_DIR to the reference source directory")
    subprocess.check_call([str(ROOT / "oracle" / "build_ref_drivers.sh"), ref_dir])
    bindir = ROOT / "oracle" / "_ref" / "drivers"
    env = dict(os.environ, OMP_NUM_THREADS="4")
    out = {}
    for name, (app, prob, args) in CASES.items():
        out[name] = {"app": app, "problem": prob, "args": args, **run_case(bindir / f"{app}_p{prob}", args, env)}
        print(name, out[name]["stdout"][-3:])
    (HERE / "drivers.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()

"""Generate tests/golden/drivers.json from the reference's own example executables.

Run where the reference sources are present:

    REF_DIR=<reference source dir> python tests/golden/make_driver_golden.py

The executables (its drivers/*.cpp, one per test problem) are built for the CPU by
oracle/build_ref_drivers.sh.  Each case runs one of them in a scratch directory and records
what a user of the reference sees: stdout, the rows appended by -stats, and the SHA-256 of
the VTK files written by -s (binary big-endian doubles, so equal digests mean bit-identical
u, f and r).  Wall-clock times and the OpenMP thread count are masked (see normalise());
everything else must match the B200 build of the same drivers exactly.  Also writes
tests/golden/facade_user.json: the reference's own solver run the way tests/cpp/facade_user.cpp
runs the facade (solution digest, verbose residual lines, the ofile log's residual column).
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

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

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


# The facade user program (tests/cpp/facade_user.cpp) on the reference's own solver: the same
# settings, init_zero, the same right-hand side and top boundary data loaded into level 0, a
# verbose V-cycle solve with an ofile log.
FACADE = {"dims": (33, 17, 9), "levels": 3, "bc": (1, 1, 1, 1, 0, 0), "cycle": "Vcycle", "nsmooth": 2, "maxiter": 5,
          "h": 1.0 / 32.0}


def facade_values(meta, top_shape):
    """The program's data in the reference's padded host layout (zero in the halos)."""
    f = np.zeros(meta.pad)
    nx, ny, nz = meta.shape
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    f[meta.halo["west"]:meta.halo["west"] + nx, meta.halo["south"]:meta.halo["south"] + ny,
      meta.halo["bottom"]:meta.halo["bottom"] + nz] = ((7 * i + 3 * j + k) % 11) * 0.125 - 0.5
    ti, tj = np.meshgrid(np.arange(top_shape[0]), np.arange(top_shape[1]), indexing="ij")
    top = (((ti + 2 * tj) % 5) * 0.25 - 0.5).reshape(top_shape)
    return f, top


def make_facade_case(ref) -> dict:
    from oracle.oracle import FACES, FIELDS, face_shape

    c = FACADE
    st0 = ref.run(c["dims"], c["levels"], bc=c["bc"], restriction="fw", relaxation="jacobi", mode="ops", ops=(),
                  h=c["h"])
    m = st0.meta[0]
    f, top = facade_values(m, face_shape(m.shape, FACES.index("top")))
    load = {f"L0_{n}": (f if n == "f" else np.zeros(m.pad)) for n in FIELDS}
    for fc, fn in enumerate(FACES):
        load[f"L0_{fn}"] = top if fn == "top" else np.zeros(face_shape(m.shape, fc))
    with tempfile.TemporaryDirectory() as d:
        log = Path(d) / "ofile.txt"
        st = ref.run(c["dims"], c["levels"], bc=c["bc"], restriction="fw", relaxation="jacobi", problem=-1,
                     mode="solve", cycle=c["cycle"], nsmooth=c["nsmooth"], maxiter=c["maxiter"], tol=0.0, h=c["h"],
                     load=load, extra={"ofile": str(log), "verbose": 1})
        ofile = log.read_text().splitlines()
    u = st.fields[(0, "u")][m.halo["west"]:m.halo["west"] + m.shape[0], m.halo["south"]:m.halo["south"] + m.shape[1],
                             m.halo["bottom"]:m.halo["bottom"] + m.shape[2]]
    verbose = [" ".join(t) for t in st.lines if len(t) >= 2 and t[0].rstrip(":").isdigit()]
    return {"u_sha256": hashlib.sha256(np.ascontiguousarray(u, dtype=np.float64).tobytes()).hexdigest(),
            "rel_res": st.stats["rel_res"][0], "iters": st.stats["iters"][0], "verbose": verbose,
            "ofile_header": ofile[0], "ofile_rel_res": [line.split()[1] for line in ofile[1:]]}


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
    from oracle.oracle import RefRun, build_ref

    fc = make_facade_case(RefRun(build_ref()))
    print("facade", fc["rel_res"], fc["verbose"][-2:])
    (HERE / "facade_user.json").write_text(json.dumps(fc, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()

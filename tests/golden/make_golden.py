"""Generate golden vectors from the reference's own code (oracle/_ref/ref_oracle).

Run where the reference sources are present (they are compiled by oracle/build_ref.sh):

    REF_DIR=<reference source dir> python tests/golden/make_golden.py [--only NAME ...]

Writes ``tests/golden/solves.json`` (whole PoissonSolver::solve runs: final relative
residual, reported iterations, and SHA-256 digests of the level-0 solution and residual
over the shape points) and ``tests/golden/ops.npz`` (operator-level input/output pairs on
small random states).  The fixtures pin both the C restatement (oracle/mgp_oracle.c) and
the CUDA engine to the reference's own output.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.oracle import FACES, FIELDS, RefRun, build_ref, face_shape  # noqa: E402

D, N = 0, 1

# name: (dims, levels, bc, restriction, relaxation, problem, cycle, nsmooth, maxiter, h, origin, tol, threads)
SOLVES = {
    # 65^3 all-Dirichlet F-cycle, Injection + red-black GS, 10 cycles (diverges in the reference)
    "c1_fcycle_65": ((65, 65, 65), 5, (D,) * 6, "inj", "gs", 10, "Fcycle", 2, 10, 1 / 64, (0, 0, 0), 0.0, 4),
    "c1_fcycle_17": ((17, 17, 17), 3, (D,) * 6, "inj", "gs", 10, "Fcycle", 2, 4, 1 / 16, (0, 0, 0), 0.0, 1),
    # x^3 y^2 z on [0,1]x[0,.5]x[0,.25], Neumann x (and requested-but-Dirichlet y), FW + Jacobi
    "c2_vcycle_33": ((33, 17, 9), 3, (N, N, N, N, D, D), "fw", "jacobi", 2, "Vcycle", 2, 5, 1 / 32, (0, 0, 0), 0.0, 1),
    "c2_fcycle_65": ((65, 33, 17), 4, (N, N, N, N, D, D), "fw", "jacobi", 2, "Fcycle", 2, 4, 1 / 64, (0, 0, 0), 0.0, 4),
    "c2_fcycle_full": ((513, 257, 129), 6, (N, N, N, N, D, D), "fw", "jacobi", 2, "Fcycle", 2, 2, 1 / 512, (0, 0, 0),
                       0.0, 8),
    "c2_vcycle_full": ((513, 257, 129), 6, (N, N, N, N, D, D), "fw", "jacobi", 2, "Vcycle", 2, 3, 1 / 512, (0, 0, 0),
                       0.0, 8),
    # cos(x z^2) sin(y^3), FW + GS converging F-cycle with the reference stopping rule active
    "c3_fcycle_33": ((33, 33, 17), 4, (D,) * 6, "fw", "gs", 3, "Fcycle", 2, 30, 1 / 32, (0, 0, 0), 1e-10, 4),
    # Neumann east/west/top with Jacobi + Injection, sin problem with the reference origin
    "mixed_fcycle_17": ((17, 17, 17), 3, (D, D, N, N, N, D), "inj", "jacobi", 1, "Fcycle", 3, 4, 0.05,
                        (-0.4, 0.21, 1.23), 0.0, 1),
    "mixed_vcycle_gs": ((33, 17, 17), 3, (D, D, N, D, N, D), "fw", "gs", 1, "Vcycle", 2, 4, 1 / 32, (0.1, 0.2, 0.3),
                        0.0, 1),
    # requested north Neumann: padded y extent even, colour (j+k)&1, columns swept in i order
    # (one thread reproduces the reference's sequential order)
    "gs_column_17": ((17, 17, 17), 3, (N, D, D, D, D, D), "inj", "gs", 1, "Vcycle", 2, 3, 1 / 16, (0, 0, 0), 0.0, 1),
    # pure relaxation, i.e. a one-level V-cycle (results/V100/clang/nvprof_1.txt)
    "relax_only_17": ((17, 17, 17), 1, (N, N, N, N, D, D), "inj", "jacobi", 2, "Vcycle", 4, 3, 1 / 16, (0, 0, 0),
                      0.0, 1),
    # the reference's no-op "relaxation" solver loop
    "relaxation_loop": ((9, 9, 9), 2, (D,) * 6, "inj", "gs", 10, "relaxation", 2, 5, 1 / 8, (0, 0, 0), 0.0, 1),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def interior(m):
    h = m.halo
    nx, ny, nz = m.shape
    return (slice(h["west"], h["west"] + nx), slice(h["south"], h["south"] + ny), slice(h["bottom"], h["bottom"] + nz))


def make_solves(ref: RefRun, only=None) -> dict:
    out = {}
    for name, (dims, levels, bc, rst, rlx, prob, cyc, ns, mi, h, org, tol, thr) in SOLVES.items():
        if only and name not in only:
            continue
        st = ref.run(dims, levels, bc=bc, restriction=rst, relaxation=rlx, problem=prob, mode="solve", cycle=cyc,
                     nsmooth=ns, maxiter=mi, tol=tol, h=h, origin=org, threads=thr, timeout=1800)
        m = st.meta[0]
        u = st.fields[(0, "u")][interior(m)]
        r = st.fields[(0, "r")][interior(m)]
        out[name] = {
            "dims": list(dims), "levels": levels, "bc": list(bc), "restriction": rst, "relaxation": rlx,
            "problem": prob, "cycle": cyc, "nsmooth": ns, "maxiter": mi, "h": h, "origin": list(org), "tol": tol,
            "rel_res": st.stats["rel_res"][0], "iters": st.stats["iters"][0],
            "u_sha256": digest(u), "r_sha256": digest(r),
            "u_sum": float(np.sum(u)), "u_absmax": float(np.max(np.abs(u))),
            "u_sample": [float(x) for x in u.reshape(-1)[:: max(1, u.size // 7)][:8]],
        }
        print(name, out[name]["rel_res"], out[name]["iters"])
    return out


# Operator-level fixtures: random states on small hierarchies, one reference operator each.
OPS = {
    # name: (dims, levels, bc, restriction, relaxation, ops, nsmooth, omega)
    "jacobi_relax": ((17, 9, 9), 2, (N, N, N, N, N, D), "fw", "jacobi", ["relax:0"], 2, -1.0),
    "gs_relax": ((17, 9, 9), 2, (D, D, N, N, N, N), "inj", "gs", ["relax:0"], 1, -1.0),
    # degenerate colouring (padded z even); the engine refuses this layout
    "gs_relax_degenerate": ((17, 9, 9), 2, (D, D, N, N, N, D), "inj", "gs", ["relax:0"], 1, -1.0),
    "gs_relax_column": ((9, 9, 9), 2, (N, D, D, D, D, D), "inj", "gs", ["relax:0"], 2, 1.1),
    "residual": ((17, 9, 9), 2, (N, N, N, N, N, D), "fw", "jacobi", ["residual:0"], 1, -1.0),
    "restrict_inj": ((17, 9, 9), 2, (N, N, N, N, D, D), "inj", "jacobi", ["restrict:0"], 1, -1.0),
    "restrict_fw": ((17, 9, 9), 2, (N, N, N, N, D, D), "fw", "jacobi", ["restrict:0"], 1, -1.0),
    "bc_restrict_fw": ((17, 9, 9), 2, (D, D, N, N, N, D), "fw", "jacobi", ["bcrestrict:0"], 1, -1.0),
    "bc_restrict_inj": ((17, 9, 9), 2, (D, D, N, N, N, N), "inj", "gs", ["bcrestrict:0"], 1, -1.0),
    "prolong": ((17, 9, 9), 2, (N, N, N, N, D, D), "fw", "jacobi", ["prolong:0"], 1, -1.0),
    "prolong_add": ((17, 9, 9), 2, (D, D, N, N, N, D), "fw", "jacobi", ["prolong:0", "add:0"], 1, -1.0),
    "write_bc": ((9, 9, 9), 2, (D, D, N, D, D, D), "fw", "jacobi", ["writebc:0"], 1, -1.0),
    "vcycle": ((17, 17, 9), 3, (N, N, N, N, N, D), "fw", "jacobi", ["vcycle:0"], 2, -1.0),
    "fcycle_gs": ((17, 17, 9), 3, (D, D, N, N, D, D), "inj", "gs", ["fcycle:0"], 2, -1.0),
}


def make_ops(ref: RefRun) -> dict:
    arrays = {}
    rng = np.random.default_rng(20261203)
    for name, (dims, levels, bc, rst, rlx, ops, ns, om) in OPS.items():
        # First run with no ops to learn the layout.
        st0 = ref.run(dims, levels, bc=bc, restriction=rst, relaxation=rlx, mode="ops", ops=(), h=0.0625)
        load = {}
        for l in range(levels):
            m = st0.meta[l]
            for fname in FIELDS:
                if fname == "uprev" and rlx != "jacobi":
                    continue
                a = rng.uniform(-1, 1, size=m.pad)
                load[f"L{l}_{fname}"] = a
            for fc, fn in enumerate(FACES):
                load[f"L{l}_{fn}"] = rng.uniform(-1, 1, size=face_shape(m.shape, fc))
        st = ref.run(dims, levels, bc=bc, restriction=rst, relaxation=rlx, mode="ops", ops=ops, load=load,
                     nsmooth=ns, omega=om, h=0.0625)
        arrays[f"{name}/meta"] = np.array([json.dumps({"dims": dims, "levels": levels, "bc": bc, "restriction": rst,
                                                       "relaxation": rlx, "ops": ops, "nsmooth": ns, "omega": om,
                                                       "h": 0.0625})])
        for k, v in load.items():
            arrays[f"{name}/in/{k}"] = v
        for (l, fname), v in st.fields.items():
            arrays[f"{name}/out/L{l}_{fname}"] = v
        for (l, fn), v in st.faces.items():
            arrays[f"{name}/out/L{l}_{fn}"] = v
        print(name, "ok")
    return arrays


def main():
    binary = build_ref()
    if binary is None or not Path(binary).exists():
        raise SystemExit("reference sources not available: cannot generate golden vectors")
    ref = RefRun(binary)
    # `--only NAME ...` regenerates the named solves and keeps every other fixture as it is
    only = sys.argv[sys.argv.index("--only") + 1:] if "--only" in sys.argv else None
    solves = make_solves(ref, only)
    if only:
        kept = json.loads((HERE / "solves.json").read_text())
        kept.update(solves)
        solves = kept
    (HERE / "solves.json").write_text(json.dumps(solves, indent=1, sort_keys=True) + "\n")
    if only:
        return
    ops = make_ops(ref)
    np.savez_compressed(HERE / "ops.npz", **ops)


if __name__ == "__main__":
    main()

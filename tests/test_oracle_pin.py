"""CPU: pin the oracle (oracle/mgp_oracle.c, the C restatement) to the reference.

* against the committed golden vectors generated by the reference's own build
  (tests/golden/make_golden.py): whole solves by SHA-256 of the level-0 solution/residual
  and operator-level input/output pairs, all bit-exact;
* live against the reference build (oracle/_ref/ref_oracle) on seeded random states when
  that binary is present.
"""
import json

import numpy as np
import pytest

from _util import digest, golden_cfg, load_ops, make_oracle
from oracle.oracle import FACES, FIELDS, REF_BIN, RefRun

SOLVES = json.loads((__import__("pathlib").Path(__file__).parent / "golden" / "solves.json").read_text())
FULL = ("c2_fcycle_full", "c2_vcycle_full")
QUICK = [k for k in SOLVES if k not in FULL]


def run_oracle_solve(cfg):
    o = make_oracle(cfg)
    o.init_problem(cfg["problem"], tuple(cfg["origin"]))
    o.write_bc(0)
    rr, it, _, hist = o.solve(cfg["cycle"], cfg["nsmooth"], -1.0, cfg["maxiter"], 1, cfg["tol"])
    return o, rr, it, hist


@pytest.mark.parametrize("name", QUICK)
def test_oracle_matches_reference_solve(name):
    cfg = golden_cfg(SOLVES[name])
    o, rr, it, _ = run_oracle_solve(cfg)
    assert rr == cfg["rel_res"]
    assert it == cfg["iters"]
    assert digest(o.shape_view("u", 0)) == cfg["u_sha256"]
    assert digest(o.shape_view("r", 0)) == cfg["r_sha256"]


@pytest.mark.slow
@pytest.mark.parametrize("name", FULL)
def test_oracle_matches_reference_full_size_c2(name):
    cfg = golden_cfg(SOLVES[name])
    o, rr, it, _ = run_oracle_solve(cfg)
    assert rr == cfg["rel_res"] and it == cfg["iters"]
    assert digest(o.shape_view("u", 0)) == cfg["u_sha256"]


OPS = load_ops(np.load(__import__("pathlib").Path(__file__).parent / "golden" / "ops.npz"))


def apply_ops(o, ops, omega, nsmooth):
    om = o.default_omega() if omega < 0 else omega
    for spec in ops:
        op, lvl = spec.split(":")
        lvl = int(lvl)
        if op == "relax":
            o.relax(lvl, om, nsmooth)
        elif op == "residual":
            o.residual(lvl)
        elif op == "restrict":
            o.restrict(lvl)
        elif op == "bcrestrict":
            o.restrict_bc(lvl)
        elif op == "prolong":
            o.prolong(lvl)
        elif op == "add":
            o.add(lvl)
        elif op == "writebc":
            o.write_bc(lvl)
        elif op == "vcycle":
            o.vcycle(lvl, om, nsmooth)
        elif op == "fcycle":
            o.fcycle(lvl, om, nsmooth)
        else:
            raise ValueError(op)


def load_inputs(o, case):
    for l in range(o.levels):
        for name in FIELDS:
            key = f"in/L{l}_{name}"
            if key in case:
                o.field(name, l)[...] = case[key]
        for fc, fn in enumerate(FACES):
            o.face(fc, l)[...] = case[f"in/L{l}_{fn}"]


@pytest.mark.parametrize("name", sorted(OPS))
def test_oracle_matches_reference_operator(name):
    case = OPS[name]
    m = case["meta"]
    cfg = {"dims": tuple(m["dims"]), "levels": m["levels"], "bc": tuple(m["bc"]), "restriction": m["restriction"],
           "relaxation": m["relaxation"], "h": m["h"]}
    o = make_oracle(cfg)
    load_inputs(o, case)
    apply_ops(o, m["ops"], m["omega"], m["nsmooth"])
    for l in range(o.levels):
        mm = o.meta[l]
        for name_f in FIELDS:
            want = case[f"out/L{l}_{name_f}"][mm.interior]
            got = o.field(name_f, l)[mm.interior]
            assert np.array_equal(got, want), (name_f, l)
        for fc, fn in enumerate(FACES):
            assert np.array_equal(o.face(fc, l), case[f"out/L{l}_{fn}"]), (fn, l)


live = pytest.mark.skipif(not REF_BIN.exists(), reason="reference build (oracle/_ref) not present")


@live
@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("rst,rlx,bc", [("fw", "jacobi", (1, 1, 1, 1, 1, 0)), ("inj", "gs", (0, 0, 1, 1, 1, 0)),
                                        ("fw", "gs", (0, 0, 0, 0, 0, 0))])
def test_oracle_matches_reference_live_fcycle(seed, rst, rlx, bc):
    """A random state through one F-cycle, oracle vs the reference build."""
    rng = np.random.default_rng(seed)
    cfg = {"dims": (17, 9, 17), "levels": 3, "bc": bc, "restriction": rst, "relaxation": rlx, "h": 0.1}
    o = make_oracle(cfg)
    load = {}
    for l in range(3):
        for name in FIELDS:
            if name == "uprev" and rlx != "jacobi":
                continue
            a = rng.uniform(-1, 1, size=o.meta[l].pad)
            o.field(name, l)[...] = a
            load[f"L{l}_{name}"] = a
        for fc, fn in enumerate(FACES):
            a = rng.uniform(-1, 1, size=o.face(fc, l).shape)
            o.face(fc, l)[...] = a
            load[f"L{l}_{fn}"] = a
    st = RefRun().run(cfg["dims"], 3, bc=bc, restriction=rst, relaxation=rlx, mode="ops", ops=["fcycle:0"],
                      load=load, nsmooth=2, h=0.1)
    o.fcycle(0, o.default_omega(), 2)
    for l in range(3):
        mm = o.meta[l]
        assert np.array_equal(o.field("u", l)[mm.interior], st.fields[(l, "u")][mm.interior])

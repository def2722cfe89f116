"""GPU: the CUDA engine, called through the C ABI, against the oracle and the reference's
golden vectors.  FP64 results are required to be bit-identical (the engine keeps the
reference's operand order and is compiled without multiply-add contraction)."""
import json
from pathlib import Path

import numpy as np
import pytest

from _util import (assert_face_equal, assert_field_equal, digest, golden_cfg, load_ops, make_engine, make_oracle,
                   push, randomize)
from oracle.oracle import FACES, FIELDS

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).parent / "golden"
SOLVES = json.loads((GOLD / "solves.json").read_text())
OPS = load_ops(np.load(GOLD / "ops.npz"))

CONFIGS = [
    # dims, levels, bc (N S E W T B), restriction, relaxation
    ((17, 9, 9), 2, (1, 1, 1, 1, 0, 0), "fw", "jacobi"),
    ((33, 17, 9), 3, (0, 0, 1, 1, 1, 0), "inj", "jacobi"),
    ((33, 17, 17), 3, (0, 0, 1, 1, 1, 1), "fw", "gs"),  # top/bottom requested N: padded z odd
    ((17, 17, 17), 3, (0, 0, 0, 0, 0, 0), "inj", "gs"),
    ((17, 9, 17), 2, (1, 0, 0, 0, 0, 0), "inj", "gs"),  # padded y even: column order
    ((65, 33, 33), 4, (1, 1, 1, 1, 0, 0), "fw", "jacobi"),
    ((33, 33, 33), 3, (1, 1, 0, 1, 1, 1), "fw", "jacobi"),
]
STRICT_CONFIGS = [
    ((17, 17, 9), 2, (1, 1, 1, 0, 1, 1), "fw", "jacobi"),
    ((17, 17, 17), 3, (1, 1, 1, 1, 1, 1), "inj", "jacobi"),
]


def cfg_of(c, h=0.0625, strict=False):
    return {"dims": c[0], "levels": c[1], "bc": c[2], "restriction": c[3], "relaxation": c[4], "h": h,
            "strict_bc": strict}


def pair(mgp, cfg, seed):
    o = make_oracle(cfg)
    randomize(o, seed)
    e = make_engine(mgp, cfg)
    push(o, e)
    return o, e


def live_faces(o, level):
    """Faces whose data the cycle reads at this level: every face on the finest level, the
    Neumann faces below it.  Coarse Dirichlet face arrays are never read; the reference
    re-zeroes them on every visit (dirichlet.h:101-107) while the engine keeps them zero
    from allocation, so they are not compared after a random start."""
    return [fc for fc in range(6) if level == 0 or o.face_types[fc] == 1]


def check_all(o, e, fields=("u", "f", "r"), faces=True):
    for l in range(o.levels):
        for name in fields:
            assert_field_equal(o, e, name, l)
        if faces:
            for fc in live_faces(o, l):
                assert_face_equal(o, e, fc, l)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_relax_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 10 + ci)
    om = o.default_omega()
    for l in range(o.levels):
        o.relax(l, om, 2)
        e.relax(l, om, 2)
    check_all(o, e, fields=("u", "uprev"))


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_residual_and_norm_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 20 + ci)
    for l in range(o.levels):
        o.residual(l)
        e.residual(l)
        assert_field_equal(o, e, "r", l)
        assert e.norm("r", l) == o.norm("r", l)
        assert e.norm("f", l) == o.norm("f", l)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_restriction_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 30 + ci)
    for l in range(o.levels - 1):
        o.restrict(l)
        e.restrict(l)
        assert_field_equal(o, e, "f", l + 1)
        o.restrict_bc(l)
        e.restrict_bc(l)
        for fc in range(6):
            assert_face_equal(o, e, fc, l + 1)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_prolongation_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 40 + ci)
    for l in range(o.levels - 1):
        o.prolong(l)
        e.prolong(l)
        assert_field_equal(o, e, "r", l)
        o.add(l)
        e.add(l)
        assert_field_equal(o, e, "u", l)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_fused_prolong_add_matches_prolong_then_add(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 50 + ci)
    for l in range(o.levels - 1):
        o.prolong(l)
        o.add(l)
        e.prolong_add(l)
        assert_field_equal(o, e, "u", l)
        # r keeps P e outside the relaxation bounds, as the reference's r does
        lv = e.level[l]
        nx, ny, nz = lv.shape
        kinds = lv.face_kind
        mask = np.zeros((nx, ny, nz), dtype=bool)
        x0, x1 = int(kinds[3] == 0), nx - int(kinds[2] == 0)
        y0, y1 = int(kinds[1] == 0), ny - int(kinds[0] == 0)
        z0, z1 = int(kinds[5] == 0), nz - int(kinds[4] == 0)
        mask[...] = True
        mask[x0:x1, y0:y1, z0:z1] = False
        assert_field_equal(o, e, "r", l, where=mask)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
@pytest.mark.parametrize("cycle", ["vcycle", "fcycle"])
def test_cycle_bit_exact(mgp_mod, gpu_ready, ci, cycle):
    cfg = cfg_of(CONFIGS[ci])
    o, e = pair(mgp_mod, cfg, 60 + ci)
    om = o.default_omega()
    getattr(o, cycle)(0, om, 2)
    getattr(e, cycle)(0, om, 2)
    for l in range(o.levels):
        assert_field_equal(o, e, "u", l)
        assert_field_equal(o, e, "f", l)
        for fc in live_faces(o, l):
            assert_face_equal(o, e, fc, l)


FUSED_LARGE = [
    # coarse levels wider than one k tile of the fused kernel (31 coarse points) and taller
    # than one j tile
    ((33, 33, 129), 3, (1, 1, 1, 1, 0, 0), "fw", "jacobi"),
    ((65, 17, 97), 3, (0, 0, 1, 1, 1, 1), "fw", "gs"),
    ((33, 65, 65), 3, (0, 0, 1, 1, 1, 1), "inj", "gs"),
    # long x: each block of the fused kernel marches several coarse planes, carrying the
    # FullWeighting partial sums from one fine plane to the next
    ((257, 33, 65), 3, (1, 1, 1, 1, 0, 0), "fw", "jacobi"),
    ((513, 17, 33), 3, (0, 0, 1, 1, 1, 1), "fw", "gs"),
    ((257, 17, 33), 3, (1, 1, 0, 0, 0, 0), "inj", "jacobi"),
]


@pytest.mark.parametrize("ci", range(len(FUSED_LARGE)))
def test_fused_setup_large_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(FUSED_LARGE[ci], h=1.0 / 128)
    o = make_oracle(cfg)
    randomize(o, 90 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_FUSED_SETUP)
    push(o, e)
    om = o.default_omega()
    o.fcycle(0, om, 2)
    e.fcycle(0, om, 2)
    for l in range(o.levels):
        assert_field_equal(o, e, "u", l)
        assert_field_equal(o, e, "f", l)


@pytest.mark.parametrize("ci", [0, 3])
def test_fused_setup_float_matches_unfused(mgp_mod, gpu_ready, ci):
    """FP32: the one-kernel set-up gives the same bits as residual + restriction kernels."""
    cfg = cfg_of(FUSED_LARGE[ci], h=1.0 / 128)
    o = make_oracle(cfg)
    randomize(o, 95 + ci)
    engines = [make_engine(mgp_mod, cfg, dtype=mgp_mod.F32, flags=fl) for fl in (0, mgp_mod.FLAG_FUSED_SETUP)]
    for e in engines:
        for l in range(o.levels):
            for name in ("u", "uprev", "f", "r"):
                if name == "uprev" and o.relaxation != 0:
                    continue
                e.upload(name, o.field(name, l).astype(np.float32), l)
            for fc in range(6):
                e.upload_face(fc, o.face(fc, l).astype(np.float32), l)
        e.fcycle(0, o.default_omega(), 2)
    for l in range(o.levels):
        for name in ("u", "f"):
            a, b = engines[0].download(name, l), engines[1].download(name, l)
            assert np.array_equal(a, b), (name, l)


@pytest.mark.parametrize("ci", range(len(CONFIGS)))
def test_fused_setup_cycle_bit_exact(mgp_mod, gpu_ready, ci):
    """The one-kernel residual+restriction form of the coarse-grid set-up."""
    cfg = cfg_of(CONFIGS[ci])
    o = make_oracle(cfg)
    randomize(o, 80 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_FUSED_SETUP)
    push(o, e)
    om = o.default_omega()
    o.fcycle(0, om, 2)
    e.fcycle(0, om, 2)
    for l in range(o.levels):
        assert_field_equal(o, e, "u", l)
        assert_field_equal(o, e, "f", l)


@pytest.mark.parametrize("ci", range(len(STRICT_CONFIGS)))
def test_strict_bc_cycle_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(STRICT_CONFIGS[ci], strict=True)
    o, e = pair(mgp_mod, cfg, 70 + ci)
    om = o.default_omega()
    o.fcycle(0, om, 2)
    e.fcycle(0, om, 2)
    for l in range(o.levels):
        assert_field_equal(o, e, "u", l)


def run_engine_solve(mgp, cfg, o_init, flags=0):
    """Solve with the engine from the oracle's initial state (problem data computed on the
    host by the oracle, as PoissonSolver::init does)."""
    e = make_engine(mgp, cfg, maxiter=cfg["maxiter"], tol=cfg["tol"], flags=flags)
    for name in ("u", "uprev", "f", "r"):
        if name == "uprev" and o_init.relaxation != 0:
            continue
        e.upload(name, o_init.field(name, 0), 0)
    for fc in range(6):
        e.upload_face(fc, o_init.face(fc, 0), 0)
    e.write_bc(0)
    st = e.solve(cfg["cycle"], cfg["nsmooth"], -1.0)
    return e, st


@pytest.mark.parametrize("name", sorted(SOLVES))
def test_solve_matches_reference_golden(mgp_mod, gpu_ready, name):
    cfg = golden_cfg(SOLVES[name])
    o = make_oracle(cfg)
    o.init_problem(cfg["problem"], tuple(cfg["origin"]))
    pad_z = cfg["dims"][2] + (cfg["bc"][4] != 0) + (cfg["bc"][5] != 0)
    if cfg["relaxation"] == "gs" and pad_z % 2 == 0:
        # degenerate red-black colouring: the engine refuses the layout (the reference's
        # parallel result depends on thread timing; the fixture is its one-thread run)
        with pytest.raises(mgp_mod.MgpError) as ei:
            make_engine(mgp_mod, cfg)
        assert ei.value.status == mgp_mod.ERR_UNSUPPORTED
        return
    e, st = run_engine_solve(mgp_mod, cfg, o)
    u = e.download("u", 0)[e.level[0].interior]
    r = e.download("r", 0)[e.level[0].interior]
    assert st.rel_res == cfg["rel_res"]
    assert st.iterations == cfg["iters"]
    assert digest(u) == cfg["u_sha256"]
    assert digest(r) == cfg["r_sha256"]


def test_solve_matches_oracle_history_and_state(mgp_mod, gpu_ready):
    cfg = {"dims": (33, 17, 17), "levels": 3, "bc": (1, 1, 1, 1, 1, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 32, "problem": 2, "cycle": "Fcycle", "nsmooth": 3, "maxiter": 6,
           "tol": 0.0, "origin": (0.0, 0.0, 0.0)}
    o = make_oracle(cfg)
    o.init_problem(2, (0.0, 0.0, 0.0))
    e, st = run_engine_solve(mgp_mod, cfg, o)
    o.write_bc(0)
    rr, it, _, _ = o.solve("Fcycle", 3, -1.0, 6, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    assert_field_equal(o, e, "u", 0)
    assert_field_equal(o, e, "uprev", 0)
    assert_field_equal(o, e, "r", 0)


@pytest.mark.parametrize("name", sorted(OPS))
def test_operator_matches_reference_golden(mgp_mod, gpu_ready, name):
    case = OPS[name]
    m = case["meta"]
    cfg = {"dims": tuple(m["dims"]), "levels": m["levels"], "bc": tuple(m["bc"]), "restriction": m["restriction"],
           "relaxation": m["relaxation"], "h": m["h"]}
    pad_z = cfg["dims"][2] + (cfg["bc"][4] != 0) + (cfg["bc"][5] != 0)
    if cfg["relaxation"] == "gs" and pad_z % 2 == 0:
        with pytest.raises(mgp_mod.MgpError) as ei:
            make_engine(mgp_mod, cfg)
        assert ei.value.status == mgp_mod.ERR_UNSUPPORTED
        return
    e = make_engine(mgp_mod, cfg)
    for l in range(m["levels"]):
        for f in FIELDS:
            key = f"in/L{l}_{f}"
            if key in case:
                e.upload(f, case[key], l)
        for fc, fn in enumerate(FACES):
            e.upload_face(fc, case[f"in/L{l}_{fn}"], l)
    om = m["omega"]
    for spec in m["ops"]:
        op, lvl = spec.split(":")
        lvl = int(lvl)
        {"relax": lambda: e.relax(lvl, om, m["nsmooth"]), "residual": lambda: e.residual(lvl),
         "restrict": lambda: e.restrict(lvl), "bcrestrict": lambda: e.restrict_bc(lvl),
         "prolong": lambda: e.prolong(lvl), "add": lambda: e.add(lvl), "writebc": lambda: e.write_bc(lvl),
         "vcycle": lambda: e.vcycle(lvl, om, m["nsmooth"]), "fcycle": lambda: e.fcycle(lvl, om, m["nsmooth"])}[op]()
    for l in range(m["levels"]):
        lv = e.level[l]
        for f in ("u", "f") + (("r",) if m["ops"][0].split(":")[0] not in ("vcycle", "fcycle") else ()):
            got = e.download(f, l)[lv.interior]
            want = case[f"out/L{l}_{f}"][lv.interior]
            assert np.array_equal(got, want), (name, f, l, float(np.max(np.abs(got - want))))
        kinds = e.level[l].face_kind
        for fc, fn in enumerate(FACES):
            if l > 0 and kinds[fc] == 0 and m["ops"][0].split(":")[0] in ("vcycle", "fcycle"):
                continue  # coarse Dirichlet data: never read, see live_faces()
            assert np.array_equal(e.download_face(fc, l), case[f"out/L{l}_{fn}"]), (name, fn, l)


def test_fp32_engine_tracks_fp64_oracle(mgp_mod, gpu_ready):
    """T=float solver: the same cycle in single precision stays within FP32 rounding of the
    FP64 oracle (relative 1e-4 after one V-cycle on a smooth problem)."""
    cfg = {"dims": (33, 33, 33), "levels": 4, "bc": (0, 0, 1, 1, 0, 0), "restriction": "fw", "relaxation": "jacobi",
           "h": 1 / 32}
    o = make_oracle(cfg)
    o.init_problem(3, (0.0, 0.0, 0.0))
    o.write_bc(0)
    e = make_engine(mgp_mod, cfg, dtype=mgp_mod.F32)
    for name in ("u", "uprev", "f", "r"):
        e.upload(name, o.field(name, 0).astype(np.float32), 0)
    for fc in range(6):
        e.upload_face(fc, o.face(fc, 0).astype(np.float32), 0)
    o.vcycle(0, o.default_omega(), 2)
    e.vcycle(0, -1.0, 2)
    assert_field_equal(o, e, "u", 0, exact=False, rtol=1e-4)


FW_EDGES = [
    # coarse extents even and odd in j and k, Neumann and Dirichlet faces
    ((65, 33, 33), 2, (1, 1, 1, 1, 0, 0)),
    ((33, 65, 17), 2, (0, 0, 1, 1, 1, 1)),
    ((17, 9, 65), 2, (1, 0, 0, 1, 0, 1)),
    ((129, 65, 129), 2, (1, 1, 1, 1, 0, 0)),
]


@pytest.mark.parametrize("ci", range(len(FW_EDGES)))
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_fullweighting_edges_bit_exact(mgp_mod, gpu_ready, ci, dtype):
    """FullWeighting over coarse extents even and odd in j and k, on faces of every kind: f on
    the coarse level bit-identical to the oracle (FP64), and within FP32 rounding of it (FP32)."""
    dims, levels, bc = FW_EDGES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": "fw", "relaxation": "jacobi", "h": 1 / 64,
           "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 900 + ci)
    if dtype == "f64":
        e = make_engine(mgp_mod, cfg)
        push(o, e)
        o.restrict(0)
        e.restrict(0)
        assert_field_equal(o, e, "f", 1)
    else:
        e = make_engine(mgp_mod, cfg, dtype=mgp_mod.F32)
        for l in range(o.levels):
            for name in ("u", "uprev", "f", "r"):
                o.field(name, l)[...] = o.field(name, l).astype(np.float32)
                e.upload(name, o.field(name, l).astype(np.float32), l)
        o.restrict(0)
        e.restrict(0)
        assert_field_equal(o, e, "f", 1, exact=False, rtol=1e-6)
    e.close()

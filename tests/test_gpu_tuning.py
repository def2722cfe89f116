"""GPU: launch-shape tuning (mgp_set_tuning / mgp_autotune).  The tuned parameters only cut the
kernels' work differently, so every tuned solve must leave the oracle's bits; the search must
leave the solver's fields as it found them and answer a second call from its cache."""
import numpy as np
import pytest

from _util import assert_field_equal, make_engine, make_oracle, randomize
from test_gpu_parity import run_engine_solve

pytestmark = pytest.mark.gpu

SOLVE_CFGS = [
    {"dims": (129, 65, 65), "levels": 4, "bc": (1, 1, 0, 1, 0, 0), "restriction": "fw", "relaxation": "jacobi",
     "h": 1 / 128, "cycle": "Fcycle", "nsmooth": 2, "maxiter": 3, "tol": 0.0, "strict_bc": True},
    {"dims": (65, 65, 33), "levels": 4, "bc": (0, 0, 0, 0, 0, 0), "restriction": "inj", "relaxation": "gs",
     "h": 1 / 64, "cycle": "Vcycle", "nsmooth": 2, "maxiter": 3, "tol": 0.0},
    {"dims": (129, 129, 65), "levels": 5, "bc": (1, 1, 1, 1, 0, 0), "restriction": "fw", "relaxation": "jacobi",
     "h": 1 / 128, "cycle": "Vcycle", "nsmooth": 3, "maxiter": 3, "tol": 0.0},
]

# (relax planes, residual planes, norm planes, set-up form, set-up planes) on every level
SHAPES = [(1, 1, 1, 1, 0), (5, 7, 3, 2, 1), (1 << 20, 2, 1 << 20, 2, 7), (3, 1 << 20, 2, 1, 3)]


@pytest.mark.parametrize("si", range(len(SHAPES)))
@pytest.mark.parametrize("ci", range(len(SOLVE_CFGS)))
def test_tuned_shapes_solve_bit_exact(mgp_mod, gpu_ready, ci, si):
    cfg = SOLVE_CFGS[ci]
    o = make_oracle(cfg)
    o.init_problem(2, (0.0, 0.0, 0.0))
    e = make_engine(mgp_mod, cfg, maxiter=cfg["maxiter"], tol=cfg["tol"])
    for l in range(cfg["levels"]):
        for p, v in enumerate(SHAPES[si]):
            e.set_tuning(l, p, v)
    assert e.get_tuning(0, mgp_mod.TUNE_SETUP_FORM) == SHAPES[si][3]
    for name in ("u", "uprev", "f", "r"):
        if name == "uprev" and o.relaxation != 0:
            continue
        e.upload(name, o.field(name, 0), 0)
    for fc in range(6):
        e.upload_face(fc, o.face(fc, 0), 0)
    e.write_bc(0)
    st = e.solve(cfg["cycle"], cfg["nsmooth"], -1.0)
    o.write_bc(0)
    rr, it, _, _ = o.solve(cfg["cycle"], cfg["nsmooth"], -1.0, cfg["maxiter"], 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    for name in ("u", "r"):
        assert_field_equal(o, e, name, 0)
    e.close()


def test_autotune_keeps_fields_caches_and_stays_exact(mgp_mod, gpu_ready):
    cfg = SOLVE_CFGS[2]
    o = make_oracle(cfg)
    randomize(o, 91)
    e = make_engine(mgp_mod, cfg, maxiter=3, tol=0.0)
    for l in range(o.levels):
        for name in ("u", "uprev", "f", "r"):
            e.upload(name, o.field(name, l), l)
        for fc in range(6):
            e.upload_face(fc, o.face(fc, l), l)
    before = {(n, l): e.download(n, l) for l in range(o.levels) for n in ("u", "uprev", "f", "r")}
    res = e.autotune("Vcycle", 3, force=True)
    assert res["tuned_ms"] > 0 and res["untuned_ms"] > 0
    assert res["tuned_ms"] <= res["untuned_ms"]
    for (n, l), a in before.items():
        assert np.array_equal(e.download(n, l), a), f"{n}@L{l} changed by the search"
    # a second solver of the same configuration takes the cached result without a search
    e2 = make_engine(mgp_mod, cfg, maxiter=3, tol=0.0)
    res2 = e2.autotune("Vcycle", 3)
    assert res2["untuned_ms"] == 0 and res2["tuned_ms"] == 0
    assert res2["params"] == res["params"]
    # and the tuned solver still solves bit-identically to the oracle
    o.init_problem(2, (0.0, 0.0, 0.0))
    for name in ("u", "uprev", "f", "r"):
        e2.upload(name, o.field(name, 0), 0)
    for fc in range(6):
        e2.upload_face(fc, o.face(fc, 0), 0)
    e2.write_bc(0)
    st = e2.solve("Vcycle", 3, -1.0)
    o.write_bc(0)
    rr, it, _, _ = o.solve("Vcycle", 3, -1.0, 3, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    for name in ("u", "r"):
        assert_field_equal(o, e2, name, 0)
    e.close()
    e2.close()


def test_autotune_refinement_solver_tunes_correction_hierarchy(mgp_mod, gpu_ready):
    cfg = {"dims": (129, 65, 65), "levels": 4, "bc": (0, 0, 0, 0, 0, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 128, "cycle": "Fcycle", "nsmooth": 2, "maxiter": 30, "tol": 1e-9}
    o = make_oracle(cfg)
    o.init_problem(3, (0.0, 0.0, 0.0))
    plain = make_engine(mgp_mod, cfg, maxiter=30, tol=1e-9, flags=mgp_mod.FLAG_REFINE_F32)
    tuned = make_engine(mgp_mod, cfg, maxiter=30, tol=1e-9, flags=mgp_mod.FLAG_REFINE_F32)
    tuned.autotune("Fcycle", 2, force=True)
    stats = []
    for e in (plain, tuned):
        for name in ("u", "f"):
            e.upload(name, o.field(name, 0), 0)
        for fc in range(6):
            e.upload_face(fc, o.face(fc, 0), 0)
        e.write_bc(0)
        stats.append(e.solve("Fcycle", 2, -1.0))
    assert (stats[0].rel_res, stats[0].iterations) == (stats[1].rel_res, stats[1].iterations)
    assert np.array_equal(plain.download("u", 0), tuned.download("u", 0))
    plain.close()
    tuned.close()


def test_tuning_rejects_bad_arguments(mgp_mod, gpu_ready):
    cfg = SOLVE_CFGS[0]
    e = make_engine(mgp_mod, cfg)
    for level, param, value in ((-1, 0, 1), (4, 0, 1), (0, mgp_mod.TUNE_PARAMS, 1), (0, -1, 1), (0, 0, -1), (0, 3, 3),
                                (0, 5, 2), (0, 6, 2), (1, 7, 3)):
        with pytest.raises(mgp_mod.MgpError) as ei:
            e.set_tuning(level, param, value)
        assert ei.value.status == mgp_mod.ERR_INVALID_ARG
    with pytest.raises(mgp_mod.MgpError):
        e.autotune("relaxation", 2)
    e.close()

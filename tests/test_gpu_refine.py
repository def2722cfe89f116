"""GPU: iterative refinement (FP64 residual and update on level 0, correction cycles on an
FP32 or FP64 hierarchy).  Results are checked against the FP64 oracle solution (the
reference's plain FP64 F-cycle driven to machine precision) and against the analytic
solution, including second-order convergence under grid refinement."""
import numpy as np
import pytest

from _util import make_engine, make_oracle
from oracle.oracle import problem_u

pytestmark = pytest.mark.gpu


def analytic(problem, shape, h, origin=(0.0, 0.0, 0.0)):
    nx, ny, nz = shape
    x = origin[0] + np.arange(nx) * h
    y = origin[1] + np.arange(ny) * h
    z = origin[2] + np.arange(nz) * h
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    if problem == 2:
        return X ** 3 * Y ** 2 * Z
    if problem == 3:
        return np.cos(X * Z * Z) * np.sin(Y ** 3)
    raise ValueError(problem)


def refined_solve(mgp, cfg, flags, tol, maxiter=60, cycle="Fcycle", nsmooth=2):
    o = make_oracle(cfg)
    o.init_problem(cfg["problem"], (0.0, 0.0, 0.0))
    o.write_bc(0)
    e = mgp.Solver(cfg["dims"], cfg["levels"], cfg["h"], cfg["bc"], cfg["restriction"], cfg["relaxation"], mgp.F64,
                   maxiter, 1, tol, (0.0, 0.0, 0.0), 0, False, flags=flags)
    e.upload("u", o.field("u", 0), 0)
    e.upload("f", o.field("f", 0), 0)
    for fc in range(6):
        e.upload_face(fc, o.face(fc, 0), 0)
    e.write_bc(0)
    st = e.solve(cycle, nsmooth)
    u = e.download("u", 0)[e.level[0].interior]
    return o, e, st, u


def oracle_converged(cfg, cycles=40):
    o = make_oracle(cfg)
    o.init_problem(cfg["problem"], (0.0, 0.0, 0.0))
    o.write_bc(0)
    o.solve("Fcycle", 2, -1.0, cycles, cycles, 0.0)  # fixed count: miniter = maxiter
    return o


DIRICHLET = {"dims": (65, 65, 33), "levels": 5, "bc": (0,) * 6, "restriction": "fw", "relaxation": "gs",
             "h": 1 / 64, "problem": 3}


@pytest.mark.parametrize("flag", ["FLAG_REFINE_F32", "FLAG_REFINE_F64"])
def test_refinement_reaches_tolerance_and_oracle_solution(mgp_mod, gpu_ready, flag):
    tol = 1e-10
    o, e, st, u = refined_solve(mgp_mod, DIRICHLET, getattr(mgp_mod, flag), tol)
    assert st.rel_res < tol, st.rel_res
    assert st.iterations <= 20
    ref = oracle_converged(DIRICHLET)
    uref = ref.shape_view("u", 0)
    err = np.max(np.abs(u - uref))
    rel_l2 = np.linalg.norm(u - uref) / np.linalg.norm(uref)
    assert err <= 1e-8 * np.max(np.abs(uref)), err
    assert rel_l2 <= 1e-8, rel_l2
    # the returned residual is the FP64 residual of the returned u
    r = e.download("r", 0)[e.level[0].interior]
    assert np.max(np.abs(r)) / o.norm("f", 0) == pytest.approx(st.rel_res, rel=1e-12)


def test_refinement_converges_on_neumann_problem(mgp_mod, gpu_ready):
    """x^3 y^2 z with Neumann x faces: the reference's own cycle stagnates near 1e-3 relative
    residual; the refinement drives the FP64 residual below 1e-10."""
    cfg = {"dims": (65, 33, 17), "levels": 4, "bc": (1, 1, 1, 1, 0, 0), "restriction": "fw", "relaxation": "jacobi",
           "h": 1 / 64, "problem": 2}
    o, e, st, u = refined_solve(mgp_mod, cfg, mgp_mod.FLAG_REFINE_F64, 1e-10, maxiter=200)
    assert st.rel_res < 1e-10, (st.rel_res, st.iterations)
    o2, e2, st2, u2 = refined_solve(mgp_mod, cfg, mgp_mod.FLAG_REFINE_F32, 1e-8, maxiter=200)
    assert st2.rel_res < 1e-8, (st2.rel_res, st2.iterations)
    # the plain reference cycle on the same problem stalls well above 1e-8
    ref = make_oracle(cfg)
    ref.init_problem(2, (0.0, 0.0, 0.0))
    ref.write_bc(0)
    rr, _, _, _ = ref.solve("Fcycle", 2, -1.0, 30, 30, 0.0)
    assert rr > 1e-6
    # both refinements agree with each other to the FP32 tolerance scale
    assert np.max(np.abs(u - u2)) <= 1e-6 * np.max(np.abs(u))


def test_refinement_keeps_second_order_accuracy(mgp_mod, gpu_ready):
    """Max error against the analytic solution falls ~4x per halving of h (README 'Verifying
    the Order of Accuracy')."""
    errs = []
    for n, lv in ((17, 3), (33, 4), (65, 5)):
        cfg = dict(DIRICHLET, dims=(n, n, n), levels=lv, h=1.0 / (n - 1))
        _, e, st, u = refined_solve(mgp_mod, cfg, mgp_mod.FLAG_REFINE_F32, 1e-10)
        assert st.rel_res < 1e-10
        errs.append(np.max(np.abs(u - analytic(3, u.shape, cfg["h"]))))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    assert all(1.8 < r < 2.3 for r in rates), (errs, rates)


STEP_CASES = [
    # (dims, levels, bc, restriction, relaxation, cycle, inner dtype)
    ((33, 33, 17), 4, (0,) * 6, "fw", "gs", "Fcycle", "f64"),
    ((33, 33, 17), 4, (0,) * 6, "fw", "gs", "Fcycle", "f32"),
    ((65, 33, 17), 4, (1, 1, 1, 1, 0, 0), "fw", "jacobi", "Vcycle", "f32"),
    ((33, 17, 17), 3, (0, 0, 1, 0, 1, 0), "inj", "jacobi", "Fcycle", "f64"),
]


@pytest.mark.parametrize("ci", range(len(STEP_CASES)))
def test_refinement_step_matches_composed_step(mgp_mod, gpu_ready, ci):
    """One refinement step (correction cycle, u += e, new FP64 residual) against the same step
    composed from plain solvers: r0 from an FP64 residual of u0, e from
    one correction cycle of a zero-boundary solver of the inner precision started at u = 0,
    u1 = u0 + e at the relaxed points (numpy), r1 from an FP64 residual of u1.  u1 and r1 must
    be bit-identical, for two steps in a row."""
    dims, levels, bc, rst, rlx, cyc, idt = STEP_CASES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": rlx, "h": 1.0 / (dims[0] - 1)}
    o = make_oracle(cfg)
    rng = np.random.default_rng(500 + ci)
    u0 = rng.uniform(-1, 1, size=o.meta[0].pad)
    f = rng.uniform(-1, 1, size=o.meta[0].pad)
    faces = [rng.uniform(-1, 1, size=o.face(fc, 0).shape) for fc in range(6)]
    flag = mgp_mod.FLAG_REFINE_F64 if idt == "f64" else mgp_mod.FLAG_REFINE_F32
    R = make_engine(mgp_mod, cfg, maxiter=1, tol=0.0, flags=flag)
    P = make_engine(mgp_mod, cfg)  # FP64: residuals
    inner_dt = mgp_mod.F64 if idt == "f64" else mgp_mod.F32
    npdt = np.float64 if idt == "f64" else np.float32
    Q = make_engine(mgp_mod, cfg, dtype=inner_dt)  # the correction cycle, zero boundary data
    for e in (R, P):
        e.upload("u", u0, 0)
        e.upload("f", f, 0)
        for fc in range(6):
            e.upload_face(fc, faces[fc], 0)
        e.write_bc(0)
    lv = R.level[0]
    inner = lv.interior
    # the relaxation bounds of level 0 (Dirichlet faces excluded) inside the host layout
    fk = dict(zip(("north", "south", "east", "west", "top", "bottom"), lv.face_kind))
    rb = tuple(slice(h + (fk[lo_f] == 0), h + n - (fk[hi_f] == 0))
               for h, n, lo_f, hi_f in zip((lv.halo["west"], lv.halo["south"], lv.halo["bottom"]), lv.shape,
                                           ("west", "south", "bottom"), ("east", "north", "top")))
    ucur = P.download("u", 0)
    for step in range(2):
        P.upload("u", ucur, 0)
        P.residual(0)
        r0 = P.download("r", 0)
        # correction: zero-guess cycle on f = (Ti) r0 over the relaxed points
        fi = np.zeros(lv.pad, dtype=npdt)
        fi[rb] = r0[rb].astype(npdt)
        for l in range(levels):
            for name in ("u", "uprev", "f", "r"):
                if name == "uprev" and rlx != "jacobi":
                    continue
                Q.upload(name, np.zeros(Q.level[l].pad, dtype=npdt), l)
        Q.upload("f", fi, 0)
        getattr(Q, cyc.lower())(0, -1.0, 2)
        ecorr = Q.download("u", 0)
        ucur = ucur.copy()
        ucur[rb] = ucur[rb] + ecorr[rb].astype(np.float64)
        st = R.solve(cyc, 2)
        assert st.cycles_run == 1
        u1 = R.download("u", 0)
        assert np.array_equal(u1[inner], ucur[inner]), f"step {step}: u differs at {np.count_nonzero(u1[inner] != ucur[inner])} points"
        P.upload("u", ucur, 0)
        P.residual(0)
        r1 = P.download("r", 0)
        assert np.array_equal(R.download("r", 0)[rb], r1[rb])
    for e in (R, P, Q):
        e.close()

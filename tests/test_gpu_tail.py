"""GPU: the coarsest levels of a cycle in one CTA (mgp_tail.cuh, on request: MGP_TUNE_TAIL = 1).
With the tail and without it, V- and F-cycles leave the same bits in u, u_prev, f, r and the face data of
every level, in FP64 and FP32, for Jacobi and red-black SOR, FullWeighting and Injection, and
Dirichlet and Neumann faces; and with the tail, the FP64 cycles equal the oracle's."""
import numpy as np
import pytest

from _util import make_oracle, randomize

pytestmark = pytest.mark.gpu

CASES = [
    # dims, levels, bc (strict), relaxation, restriction
    ((129, 65, 65), 4, (0, 0, 0, 0, 0, 0), "jacobi", "fw"),
    ((129, 65, 65), 4, (1, 1, 1, 1, 0, 0), "jacobi", "fw"),
    ((129, 65, 65), 4, (0, 0, 0, 0, 0, 0), "gs", "fw"),
    ((65, 33, 65), 4, (1, 0, 0, 1, 0, 1), "jacobi", "inj"),
    ((65, 65, 33), 3, (0, 0, 1, 1, 1, 1), "gs", "inj"),
    ((33, 17, 9), 3, (1, 1, 1, 1, 1, 0), "jacobi", "fw"),
]


@pytest.mark.parametrize("cycle", ["vcycle", "fcycle"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_tail_matches_grid_path(mgp_mod, gpu_ready, ci, dtype, cycle):
    dims, levels, bc, rlx, rst = CASES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": rlx,
           "h": 1.0 / (dims[0] - 1), "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 40 + ci)
    dt = mgp_mod.F64 if dtype == "f64" else mgp_mod.F32
    npdt = np.float64 if dtype == "f64" else np.float32
    jac = rlx == "jacobi"
    names = ("u", "uprev", "f", "r") if jac else ("u", "f", "r")
    engines = []
    for tail_on in (1, 0):
        e = mgp_mod.Solver(dims, levels, cfg["h"], bc, mgp_mod.FULLWEIGHTING if rst == "fw" else mgp_mod.INJECTION,
                           mgp_mod.JACOBI if jac else mgp_mod.GAUSSSEIDEL, dt, 10, 1, 0.0, strict_bc=True)
        e.set_tuning(0, mgp_mod.TUNE_TAIL, tail_on)
        for l in range(levels):
            for name in names:
                e.upload(name, o.field(name, l).astype(npdt), l)
            for fc in range(6):
                e.upload_face(fc, o.face(fc, l).astype(npdt), l)
        for ns in (2, 3):
            getattr(e, cycle)(0, -1.0, ns)
        engines.append(e)
    for l in range(levels):
        for name in names:
            a, b = engines[0].download(name, l), engines[1].download(name, l)
            assert np.array_equal(a, b), f"{name}@L{l}: {np.count_nonzero(a != b)} points differ"
        for fc in range(6):
            assert np.array_equal(engines[0].download_face(fc, l), engines[1].download_face(fc, l)), (fc, l)
    for e in engines:
        e.close()


@pytest.mark.parametrize("cycle", ["vcycle", "fcycle"])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_tail_cycles_match_oracle(mgp_mod, gpu_ready, ci, cycle):
    from _util import assert_field_equal, make_engine, push

    dims, levels, bc, rlx, rst = CASES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": rlx,
           "h": 1.0 / (dims[0] - 1), "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 80 + ci)
    e = make_engine(mgp_mod, cfg)
    e.set_tuning(0, mgp_mod.TUNE_TAIL, 1)
    push(o, e)
    om = o.default_omega()
    for ns in (2, 3):
        getattr(o, cycle)(0, om, ns)
        getattr(e, cycle)(0, om, ns)
    for l in range(levels):
        assert_field_equal(o, e, "u", l)
        assert_field_equal(o, e, "f", l)

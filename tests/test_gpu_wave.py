"""GPU: the wavefront passes of large Jacobi levels (k_wave: two sweeps per pass, and the
residual after the last sweep in the same pass) against the oracle's operation-by-operation
relaxation, cycles and solves, and against the engine's default single-sweep path (the passes
are opt-in: MGP_FLAG_WAVE).

FP64 results must be bit-identical.  The random states differ between u and u_prev at the
Dirichlet points, so the values a sweep leaves alone (u_prev's for sweep 1, u's for sweep 2)
are checked too."""
import numpy as np
import pytest

from _util import assert_field_equal, make_engine, make_oracle, push, randomize
from test_gpu_parity import run_engine_solve

pytestmark = pytest.mark.gpu

# (dims, bc N S E W T B) with strict kinds; each level-0 shape has >= 2^20 points.  Tiles with a
# short last tile, odd nz (a half-filled last k vector), every face kind.
RELAX = [
    ((97, 131, 83), (1, 1, 1, 1, 1, 1)),   # all Neumann
    ((97, 131, 83), (0, 0, 0, 0, 0, 0)),   # all Dirichlet
    ((65, 257, 129), (1, 1, 1, 1, 0, 0)),  # the bench's kinds
    ((129, 129, 65), (0, 1, 1, 0, 1, 0)),  # mixed
    ((33, 65, 513), (1, 0, 0, 1, 0, 1)),   # nz 513: wider than one box row, single sweeps
    ((65, 129, 255), (1, 0, 0, 1, 0, 1)),  # nz 255: the widest box row
]


def relax_cfg(dims, bc, levels=1):
    return {"dims": dims, "levels": levels, "bc": bc, "restriction": "fw", "relaxation": "jacobi", "h": 1 / 64,
            "strict_bc": True}


@pytest.mark.parametrize("ns", [1, 2, 3, 4])
@pytest.mark.parametrize("ci", range(len(RELAX)))
def test_wave_relaxation_matches_oracle(mgp_mod, gpu_ready, ci, ns):
    dims, bc = RELAX[ci]
    cfg = relax_cfg(dims, bc)
    o = make_oracle(cfg)
    randomize(o, 300 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_WAVE)
    push(o, e)
    om = o.default_omega()
    o.relax(0, om, ns)
    e.relax(0, om, ns)
    assert_field_equal(o, e, "u", 0)
    assert_field_equal(o, e, "uprev", 0)
    e.close()


CYCLES = [
    # level 0 (and level 1 for the first) large enough for the wavefront passes
    ((257, 257, 129), 4, (1, 0, 1, 1, 0, 1), "fw"),
    ((129, 129, 129), 3, (0, 0, 0, 0, 0, 0), "inj"),
    ((193, 97, 65), 3, (1, 1, 1, 1, 1, 1), "fw"),
]


@pytest.mark.parametrize("cycle", ["fcycle", "vcycle"])
@pytest.mark.parametrize("ci", range(len(CYCLES)))
def test_wave_cycles_match_oracle(mgp_mod, gpu_ready, ci, cycle):
    """A cycle's set-up residual formed inside the pre-smoothing pass: u, u_prev and f on
    every level bit-identical to the oracle."""
    dims, levels, bc, rst = CYCLES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": "jacobi", "h": 1 / 128,
           "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 500 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_WAVE)
    push(o, e)
    for ns in (2, 3):
        getattr(o, cycle)(0, o.default_omega(), ns)
        getattr(e, cycle)(0, o.default_omega(), ns)
    for l in range(o.levels):
        for name in ("u", "uprev", "f"):
            assert_field_equal(o, e, name, l)
    e.close()


@pytest.mark.parametrize("cycle", ["Fcycle", "Vcycle"])
def test_wave_solve_matches_oracle(mgp_mod, gpu_ready, cycle):
    """Solve iterations (captured graphs, the solve loop's residual and max-norm inside the last
    pass): residual history, u, u_prev and r bit-identical to the oracle, with fewer launches
    than the single-sweep path."""
    cfg = {"dims": (129, 129, 129), "levels": 5, "bc": (1, 1, 1, 1, 0, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 128, "cycle": cycle, "nsmooth": 2, "maxiter": 4, "tol": 0.0}
    o = make_oracle(cfg)
    o.init_problem(2, (0.0, 0.0, 0.0))
    e, st = run_engine_solve(mgp_mod, cfg, o, flags=mgp_mod.FLAG_WAVE)
    single, st1 = run_engine_solve(mgp_mod, cfg, o)
    o.write_bc(0)
    rr, it, _, _ = o.solve(cycle, 2, -1.0, 4, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    assert (st1.rel_res, st1.iterations) == (rr, it)
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    assert st.kernel_launches < st1.kernel_launches
    e.close()
    single.close()


def test_wave_solve_dirichlet_norm_counts_stored_residual(mgp_mod, gpu_ready):
    """All-Dirichlet faces: the residual norm includes the stored r on the boundary planes, which
    the pass reads instead of computing (random r there, larger than the interior residual)."""
    cfg = {"dims": (129, 129, 97), "levels": 3, "bc": (0, 0, 0, 0, 0, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 128, "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 41, lo=-5.0, hi=5.0)
    e = make_engine(mgp_mod, cfg, maxiter=3, tol=0.0, flags=mgp_mod.FLAG_WAVE)
    push(o, e)
    st = e.solve("Vcycle", 2, -1.0)
    rr, it, _, _ = o.solve("Vcycle", 2, -1.0, 3, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    e.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_wave_matches_single_sweeps(mgp_mod, gpu_ready, dtype):
    """Two levels with wavefront passes (257x257x129 and 129x129x65): F- and V-cycles by
    MGP_FLAG_WAVE and by default leave the same bits in u, u_prev and r on every level."""
    cfg = {"dims": (257, 257, 129), "levels": 4, "bc": (1, 0, 1, 1, 0, 1), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 256, "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 77)
    dt = mgp_mod.F64 if dtype == "f64" else mgp_mod.F32
    npdt = np.float64 if dtype == "f64" else np.float32
    engines = [make_engine(mgp_mod, cfg, dtype=dt, flags=fl) for fl in (mgp_mod.FLAG_WAVE, 0)]
    for e in engines:
        for l in range(o.levels):
            for name in ("u", "uprev", "f", "r"):
                e.upload(name, o.field(name, l).astype(npdt), l)
            for fc in range(6):
                e.upload_face(fc, o.face(fc, l).astype(npdt), l)
        e.fcycle(0, -1.0, 2)
        e.vcycle(0, -1.0, 3)
        e.fcycle(0, -1.0, 1)
    for l in range(o.levels):
        for name in ("u", "uprev", "r"):
            a, b = engines[0].download(name, l), engines[1].download(name, l)
            assert np.array_equal(a, b), f"{name}@L{l} differs ({np.count_nonzero(a != b)} points)"
    for e in engines:
        e.close()


@pytest.mark.parametrize("ns", [1, 2, 3])
@pytest.mark.parametrize("ci", [0, 1, 2, 3])
def test_relax_residual_matches_oracle(mgp_mod, gpu_ready, ci, ns):
    """mgp_relax_residual (relax, residual and max-norm; one pass for the last sweeps on large
    levels) against the oracle's relax, residual and norm in turn."""
    dims, bc = RELAX[ci]
    cfg = relax_cfg(dims, bc)
    o = make_oracle(cfg)
    randomize(o, 700 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_WAVE)
    push(o, e)
    om = o.default_omega()
    o.relax(0, om, ns)
    o.residual(0)
    got = e.relax_residual(0, om, ns, norm=True)
    assert got == o.norm("r", 0)
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    o.relax(0, om, ns)
    o.residual(0)
    assert e.relax_residual(0, om, ns, norm=False) is None
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    e.close()


def test_wave_wait_timeout_reports_and_recovers(mgp_mod, gpu_ready):
    """Failure detection without a GPU fault: with a bound of one poll, the consumers of the
    wavefront passes give up on plane copies that have not landed yet (the producer keeps its
    normal bound and lets every copy it issued land before the CTA exits).  The solve reports
    MGP_ERR_TIMEOUT instead of returning wrong numbers, and the same solver, with the default
    bound again, then solves bit-identically to the oracle."""
    cfg = {"dims": (257, 257, 129), "levels": 3, "bc": (1, 1, 1, 1, 0, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 256, "cycle": "Vcycle", "nsmooth": 2, "maxiter": 2, "tol": 0.0}
    o = make_oracle(cfg)
    o.init_problem(2, (0.0, 0.0, 0.0))
    e = make_engine(mgp_mod, cfg, maxiter=2, tol=0.0, flags=mgp_mod.FLAG_WAVE)
    e.set_wait_polls(1)
    for name in ("u", "uprev", "f", "r"):
        e.upload(name, o.field(name, 0), 0)
    for fc in range(6):
        e.upload_face(fc, o.face(fc, 0), 0)
    e.write_bc(0)
    with pytest.raises(mgp_mod.MgpError) as ei:
        e.solve("Vcycle", 2, -1.0)
    assert ei.value.status == mgp_mod.ERR_TIMEOUT
    # the context is intact: reload the initial state and solve with the default bound
    e.set_wait_polls(0)
    for l in range(o.levels):
        for name in ("u", "uprev", "f", "r"):
            e.upload(name, o.field(name, l), l)
    for fc in range(6):
        e.upload_face(fc, o.face(fc, 0), 0)
    e.write_bc(0)
    st = e.solve("Vcycle", 2, -1.0)
    o.write_bc(0)
    rr, it, _, _ = o.solve("Vcycle", 2, -1.0, 2, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    e.close()

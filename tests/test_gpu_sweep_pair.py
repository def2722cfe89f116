"""GPU: two weighted-Jacobi sweeps in one pass (k_jacobi_pair, MGP_FLAG_SWEEP_PAIRS, levels
of at least 2^20 points) against the oracle's sweep-by-sweep relaxation and against the
engine's default single-sweep path.  u and u_prev are required to be bit-identical:
the pair keeps the reference's values at Dirichlet points of both buffers (random, and
different in u and u_prev, in these tests) and writes u_prev's relaxed points when nothing
later in the cycle overwrites them."""
import numpy as np
import pytest

from _util import assert_field_equal, make_engine, make_oracle, push, randomize
from test_gpu_parity import run_engine_solve

pytestmark = pytest.mark.gpu

# (dims, bc N S E W T B) with strict kinds; each level-0 shape has >= 2^20 points.  Row tiles
# with a short last tile, odd nz (a half-filled last k vector), every face kind.
RELAX = [
    ((97, 131, 83), (1, 1, 1, 1, 1, 1)),   # all Neumann
    ((97, 131, 83), (0, 0, 0, 0, 0, 0)),   # all Dirichlet
    ((65, 257, 129), (1, 1, 1, 1, 0, 0)),  # the bench's kinds: 13-row tiles, the last of 10
    ((129, 129, 65), (0, 1, 1, 0, 1, 0)),  # mixed
    ((33, 65, 513), (1, 0, 0, 1, 0, 1)),   # nz 513: too wide for a pair tile, single sweeps
    ((257, 65, 257), (1, 0, 0, 1, 0, 1)),  # nz 257: 5-row tiles
]


def relax_cfg(dims, bc, levels=1):
    return {"dims": dims, "levels": levels, "bc": bc, "restriction": "fw", "relaxation": "jacobi", "h": 1 / 64,
            "strict_bc": True}


@pytest.mark.parametrize("ns", [2, 3, 4])
@pytest.mark.parametrize("ci", range(len(RELAX)))
def test_pair_relaxation_matches_oracle(mgp_mod, gpu_ready, ci, ns):
    dims, bc = RELAX[ci]
    cfg = relax_cfg(dims, bc)
    o = make_oracle(cfg)
    randomize(o, 300 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_SWEEP_PAIRS)
    push(o, e)
    om = o.default_omega()
    o.relax(0, om, ns)
    e.relax(0, om, ns)
    assert_field_equal(o, e, "u", 0)
    assert_field_equal(o, e, "uprev", 0)


def test_pair_fcycle_solve_matches_oracle(mgp_mod, gpu_ready):
    """F-cycle solve on 129^3 (level 0 relaxes in pairs): residual history, u, u_prev and r
    bit-identical to the oracle after 4 iterations (graphs for both buffer arrangements are
    captured and replayed), with fewer launches than the single-sweep path."""
    cfg = {"dims": (129, 129, 129), "levels": 5, "bc": (1, 1, 1, 1, 0, 0), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 128, "cycle": "Fcycle", "nsmooth": 2, "maxiter": 4, "tol": 0.0}
    o = make_oracle(cfg)
    o.init_problem(2, (0.0, 0.0, 0.0))
    e, st = run_engine_solve(mgp_mod, cfg, o, flags=mgp_mod.FLAG_SWEEP_PAIRS)
    o.write_bc(0)
    rr, it, _, _ = o.solve("Fcycle", 2, -1.0, 4, 1, 0.0)
    assert (st.rel_res, st.iterations) == (rr, it)
    for name in ("u", "uprev", "r"):
        assert_field_equal(o, e, name, 0)
    o2 = make_oracle(cfg)
    o2.init_problem(2, (0.0, 0.0, 0.0))
    single = make_engine(mgp_mod, cfg, maxiter=4, tol=0.0)
    for name in ("u", "uprev", "f", "r"):
        single.upload(name, o2.field(name, 0), 0)
    for fc in range(6):
        single.upload_face(fc, o2.face(fc, 0), 0)
    single.write_bc(0)
    st1 = single.solve("Fcycle", 2, -1.0)
    assert (st1.rel_res, st1.iterations) == (rr, it)
    assert st.kernel_launches < st1.kernel_launches
    e.close()
    single.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_pair_cycles_match_single_sweeps(mgp_mod, gpu_ready, dtype):
    """Two levels with pairs (257x257x129 and 129x129x65): F- and V-cycles with
    MGP_FLAG_SWEEP_PAIRS and with the default single sweeps leave the same bits in u, u_prev
    and r on every level."""
    cfg = {"dims": (257, 257, 129), "levels": 4, "bc": (1, 0, 1, 1, 0, 1), "restriction": "fw",
           "relaxation": "jacobi", "h": 1 / 256, "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 77)
    dt = mgp_mod.F64 if dtype == "f64" else mgp_mod.F32
    npdt = np.float64 if dtype == "f64" else np.float32
    engines = [make_engine(mgp_mod, cfg, dtype=dt, flags=fl) for fl in (mgp_mod.FLAG_SWEEP_PAIRS, 0)]
    for e in engines:
        for l in range(o.levels):
            for name in ("u", "uprev", "f", "r"):
                e.upload(name, o.field(name, l).astype(npdt), l)
            for fc in range(6):
                e.upload_face(fc, o.face(fc, l).astype(npdt), l)
        e.fcycle(0, -1.0, 2)
        e.vcycle(0, -1.0, 3)
        e.fcycle(0, -1.0, 2)
    for l in range(o.levels):
        for name in ("u", "uprev", "r"):
            a, b = engines[0].download(name, l), engines[1].download(name, l)
            assert np.array_equal(a, b), f"{name}@L{l} differs ({np.count_nonzero(a != b)} points)"
    for e in engines:
        e.close()

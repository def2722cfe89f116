"""GPU: the x-slab decomposition (mgp/decomp.py) with engine solvers as the slabs -- all slabs in
one process on one GPU, halo planes copied between them (the path the multi-GPU form runs
with one slab per GPU, planes sent by NCCL instead).  The decomposed solve must reproduce the
one-domain oracle solve bit for bit at every owned plane, with Jacobi and with red-black
Gauss-Seidel (one-colour half-sweeps, mgp_relax_colour, exchanged in between)."""
import numpy as np
import pytest

from mgp import decomp
from test_decomp import CASES, RLX, RST, fields_of, global_state

pytestmark = pytest.mark.gpu


def engine_slab(mgp, slab, g, dims, bc, levels, h, rst, rlx="jacobi"):
    e = decomp.EngineSlab(mgp, slab, dims, levels, h, bc, RST[rst], relaxation=RLX[rlx])
    lv, gm = e.solver.level[0], g.meta[0]
    off = slab.lo + gm.halo["west"] - lv.halo["west"]
    for name in fields_of(rlx):
        e.solver.upload(name, np.ascontiguousarray(g.field(name, 0)[off:off + lv.pad[0]]), 0)
    for fc in range(6):
        gf = g.face(fc, 0)
        if fc in (0, 1, 4, 5):
            a = gf[slab.lo:slab.hi + 1]
        elif fc == decomp.WEST:
            a = gf if slab.rank == 0 else g.shape_view("u", 0)[slab.lo][None]
        else:
            a = gf if slab.rank == slab.parts - 1 else g.shape_view("u", 0)[slab.hi][None]
        e.solver.upload_face(fc, np.ascontiguousarray(a), 0)
    e.solver.write_bc(0)
    return e


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_engine_slabs_match_global_solve(mgp_mod, gpu_ready, ci):
    dims, levels, bc, rst, cycle, ns, parts, rlx = CASES[ci]
    g, h = global_state(dims, levels, bc, rst, 700 + ci, rlx)
    slabs = decomp.plan_slabs(dims[0], levels, parts)
    ex = {s.rank: engine_slab(mgp_mod, s, g, dims, bc, levels, h, rst, rlx) for s in slabs}
    omega = g.default_omega()
    west = decomp.global_west_halo(mgp_mod, dims, levels, h, bc, RST[rst], RLX[rlx])
    assert west == g.meta[0].halo["west"]
    solver = decomp.SlabSolver(slabs, decomp.LocalExchange(ex), levels, omega, maxiter=3, relaxation=rlx,
                               west_halo=west)
    rel, it, hist = solver.solve(cycle, ns)
    rr, it_g, _, hist_g = g.solve(cycle, ns, omega, 3, 1, 0.0)
    assert rel == rr and it == it_g
    assert hist[1:] == list(hist_g)
    for name in ("u", "r"):
        whole = g.shape_view(name, 0)
        for s in slabs:
            _, _, olo, ohi = s.at(0)
            lv = ex[s.rank].solver.level[0]
            got = ex[s.rank].solver.download(name, 0)[lv.interior][s.local(0, olo):s.local(0, ohi)]
            assert np.array_equal(got, whole[olo:ohi]), (name, s.rank)
    for e in ex.values():
        e.close()


@pytest.mark.parametrize("bc", [(1, 1, 1, 1, 0, 0), (1, 0, 1, 1, 0, 0), (0, 0, 0, 1, 1, 1)])
def test_relax_colour_matches_oracle(mgp_mod, gpu_ready, bc):
    """mgp_relax_colour: one half-sweep of the named colour, alternate flag untouched -- the
    same bits as the oracle's, for colours in either order (P_y even: the column-ordered
    sweep)."""
    from _util import assert_field_equal, make_engine, make_oracle, push, randomize

    cfg = {"dims": (33, 17, 17), "levels": 2, "bc": bc, "restriction": "fw", "relaxation": "gs", "h": 1 / 32}
    o = make_oracle(cfg)
    randomize(o, 31)
    e = make_engine(mgp_mod, cfg)
    push(o, e)
    for colour in (1, 1, 0, 1, 0, 0):
        o.relax_colour(0, 0.9, colour)
        e.relax_colour(0, 0.9, colour)
        assert_field_equal(o, e, "u", 0)
    # the alternate flag was not touched: a full relaxation still starts with colour 0
    o.relax(0, 0.9, 1)
    e.relax(0, 0.9, 1)
    assert_field_equal(o, e, "u", 0)
    e.close()


def test_relax_colour_refused_for_jacobi(mgp_mod, gpu_ready):
    e = mgp_mod.Solver((17, 9, 9), 2, 1 / 16, (0,) * 6, mgp_mod.FULLWEIGHTING, mgp_mod.JACOBI, mgp_mod.F64)
    with pytest.raises(mgp_mod.MgpError) as ei:
        e.relax_colour(0, -1.0, 0)
    assert ei.value.status == mgp_mod.ERR_UNSUPPORTED
    e.close()

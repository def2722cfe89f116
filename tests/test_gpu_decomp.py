"""GPU: the x-slab decomposition (mgp/decomp.py) with engine solvers as the slabs -- all slabs in
one process on one GPU, halo planes copied between them (the path the multi-GPU form runs
with one slab per GPU, planes sent by NCCL instead).  The decomposed solve must reproduce the
one-domain oracle solve bit for bit at every owned plane."""
import numpy as np
import pytest

from mgp import decomp
from test_decomp import CASES, RST, global_state

pytestmark = pytest.mark.gpu


def engine_slab(mgp, slab, g, dims, bc, levels, h, rst):
    e = decomp.EngineSlab(mgp, slab, dims, levels, h, bc, RST[rst])
    lv, gm = e.solver.level[0], g.meta[0]
    off = slab.lo + gm.halo["west"] - lv.halo["west"]
    for name in ("u", "uprev", "f", "r"):
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
    dims, levels, bc, rst, cycle, ns, parts = CASES[ci]
    g, h = global_state(dims, levels, bc, rst, 700 + ci)
    slabs = decomp.plan_slabs(dims[0], levels, parts)
    ex = {s.rank: engine_slab(mgp_mod, s, g, dims, bc, levels, h, rst) for s in slabs}
    omega = g.default_omega()
    rel, it, hist = decomp.SlabSolver(slabs, decomp.LocalExchange(ex), levels, omega, maxiter=3).solve(cycle, ns)
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

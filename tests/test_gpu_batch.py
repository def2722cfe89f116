"""GPU: batches.  Problems of different sizes, level counts and boundary kinds solved
together (one persistent launch per level operation over a (problem, tile) work list) must
reproduce, bit for bit, the same problems solved one at a time by the refinement solver:
the batch runs the same per-tile kernels in each problem's own F-cycle order."""
import numpy as np
import pytest

from _util import make_oracle

pytestmark = pytest.mark.gpu

PROBLEMS = [
    # dims, levels, bc, problem
    ((17, 17, 17), 3, (0,) * 6, 3),
    ((33, 33, 33), 4, (0,) * 6, 1),
    ((33, 17, 17), 3, (0, 0, 1, 1, 0, 0), 2),
    ((65, 33, 33), 5, (0,) * 6, 3),
    ((9, 9, 9), 2, (0,) * 6, 1),
]


def init_problem(dims, levels, bc, problem, h):
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": "fw", "relaxation": "gs", "h": h}
    o = make_oracle(cfg)
    o.init_problem(problem, (0.0, 0.0, 0.0))
    o.write_bc(0)
    return o


def load(solver, o):
    solver.upload("u", o.field("u", 0), 0)
    solver.upload("f", o.field("f", 0), 0)
    for fc in range(6):
        solver.upload_face(fc, o.face(fc, 0), 0)
    solver.write_bc(0)


@pytest.mark.parametrize("inner", ["F32", "F64"])
@pytest.mark.parametrize("cycle", ["Fcycle", "Vcycle"])
def test_batch_matches_single_problem_solves(mgp_mod, gpu_ready, inner, cycle):
    mgp = mgp_mod
    dt = getattr(mgp, inner)
    flag = mgp.FLAG_REFINE_F32 if inner == "F32" else mgp.FLAG_REFINE_F64
    tol = 1e-9
    batch = mgp.Batch(mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, dt, cycle, 2)
    ids, oracles = [], []
    for dims, levels, bc, prob in PROBLEMS:
        h = 1.0 / (dims[0] - 1)
        o = init_problem(dims, levels, bc, prob, h)
        pid = batch.add(dims, levels, h, bc)
        load(batch.problem(pid), o)
        ids.append(pid)
        oracles.append((o, h))
    steps = batch.solve(tol, 100)
    assert steps > 0
    assert batch.launches_per_step() >= 0
    for (dims, levels, bc, prob), pid, (o, h) in zip(PROBLEMS, ids, oracles):
        st = batch.status(pid)
        assert st.rel_res < tol, (dims, st.rel_res)
        single = mgp.Solver(dims, levels, h, bc, mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, mgp.F64, 100, 1, tol,
                            flags=flag)
        load(single, o)
        s1 = single.solve(cycle, 2)
        assert s1.iterations == st.iterations, (dims, s1.iterations, st.iterations)
        assert s1.rel_res == st.rel_res
        ub = batch.problem(pid).download("u", 0)
        us = single.download("u", 0)
        assert np.array_equal(ub, us), (dims, float(np.max(np.abs(ub - us))))
        rb = batch.problem(pid).download("r", 0)
        rs = single.download("r", 0)
        assert np.array_equal(rb, rs)


def test_batch_add_remove_and_continue(mgp_mod, gpu_ready):
    """Problems join and leave between steps (the continuous-batching primitive)."""
    mgp = mgp_mod
    batch = mgp.Batch(mgp.FULLWEIGHTING, mgp.GAUSSSEIDEL, mgp.F32, "Fcycle", 2, max_problems=4)
    a = batch.add((33, 33, 33), 4, 1 / 32)
    o = init_problem((33, 33, 33), 4, (0,) * 6, 3, 1 / 32)
    load(batch.problem(a), o)
    assert batch.step() == 1
    assert batch.step() == 1
    b = batch.add((17, 17, 17), 3, 1 / 16)
    load(batch.problem(b), init_problem((17, 17, 17), 3, (0,) * 6, 1, 1 / 16))
    assert batch.step() == 2
    batch.remove(a)
    assert batch.step() == 1
    assert batch.status(b).iterations == 2
    with pytest.raises(mgp.MgpError):
        batch.status(a)

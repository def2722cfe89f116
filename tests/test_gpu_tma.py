"""GPU: the TMA-fed stencil sweeps (MGP_FLAG_TMA_SWEEPS: levels of 2^20 points and more sweep
with shared-memory plane rings filled by cp.async.bulk.tensor).  Every sweep kind -- Jacobi, red-black and
column-ordered Gauss-Seidel, residual with and without its max-norm -- is compared bit for
bit with the oracle on random states, over layouts with and without halos, several k tiles
and partial j tiles; FP32 sweeps are compared with the FP64 oracle within FP32 rounding."""
import numpy as np
import pytest

from _util import assert_field_equal, make_engine, make_oracle, push, randomize

pytestmark = pytest.mark.gpu

LARGE = [
    # dims, bc (N S E W T B), relaxation, strict
    ((129, 129, 65), (1, 1, 1, 1, 0, 0), "jacobi", False),
    ((65, 65, 257), (1, 1, 1, 1, 1, 1), "jacobi", True),    # two k tiles, Neumann everywhere
    ((129, 65, 129), (0, 0, 1, 1, 1, 1), "gs", False),      # red-black
    ((129, 129, 65), (1, 1, 1, 1, 0, 0), "gs", False),      # red-black, halo in x and y
    ((129, 65, 129), (1, 0, 0, 0, 1, 1), "gs", False),      # padded y even: column order
    ((129, 129, 65), (0, 0, 0, 0, 1, 1), "gs", False),      # no halo in x, y
    ((33, 65, 513), (1, 1, 0, 0, 0, 0), "jacobi", False),   # long k rows: three k tiles (FP32: two)
]


def cfg_of(c):
    return {"dims": c[0], "levels": 2, "bc": c[1], "restriction": "fw", "relaxation": c[2],
            "h": 1.0 / (max(c[0]) - 1), "strict_bc": c[3]}


@pytest.mark.parametrize("ci", range(len(LARGE)))
def test_sweeps_bit_exact(mgp_mod, gpu_ready, ci):
    cfg = cfg_of(LARGE[ci])
    o = make_oracle(cfg)
    randomize(o, 300 + ci)
    e = make_engine(mgp_mod, cfg, flags=mgp_mod.FLAG_TMA_SWEEPS)
    push(o, e)
    om = o.default_omega()
    o.relax(0, om, 2)
    e.relax(0, om, 2)
    assert_field_equal(o, e, "u", 0)
    if cfg["relaxation"] == "jacobi":
        assert_field_equal(o, e, "uprev", 0)
    o.residual(0)
    e.residual(0)
    assert_field_equal(o, e, "r", 0)
    assert e.norm("r", 0) == o.norm("r", 0)
    e.close()


@pytest.mark.parametrize("ci", [0, 2, 4])
def test_solve_iteration_residual_norm(mgp_mod, gpu_ready, ci):
    """A captured solve iteration ends with the fused residual + max-norm sweep (NORM=true):
    two V-cycle iterations, history and state identical to the oracle."""
    cfg = cfg_of(LARGE[ci])
    o = make_oracle(cfg)
    randomize(o, 400 + ci)
    e = make_engine(mgp_mod, cfg, maxiter=2, tol=0.0, flags=mgp_mod.FLAG_TMA_SWEEPS)
    push(o, e)
    rel, iters, _, hist = o.solve("Vcycle", 2, o.default_omega(), 2, 1, 0.0, 1e9)
    st = e.solve("Vcycle", nsmooth=2)
    assert st.iterations == iters
    assert st.rel_res == rel
    assert_field_equal(o, e, "u", 0)
    assert_field_equal(o, e, "r", 0)
    e.close()


@pytest.mark.parametrize("ci", range(len(LARGE)))
def test_fp32_tma_matches_oracle_scale(mgp_mod, gpu_ready, ci):
    """FP32 sweeps on the TMA path stay within FP32 rounding of the FP64 oracle."""
    cfg = cfg_of(LARGE[ci])
    o = make_oracle(cfg)
    randomize(o, 500 + ci)
    e = make_engine(mgp_mod, cfg, dtype=mgp_mod.F32, flags=mgp_mod.FLAG_TMA_SWEEPS)
    push(o, e)
    om = o.default_omega()
    o.relax(0, om, 1)
    e.relax(0, om, 1)
    assert_field_equal(o, e, "u", 0, exact=False, rtol=1e-5)
    o.residual(0)
    e.residual(0)
    # the residual of random data is O(1/h^2); compare on that scale
    assert_field_equal(o, e, "r", 0, exact=False, rtol=1e-5)
    e.close()

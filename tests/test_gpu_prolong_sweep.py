"""GPU: prolongation + add fused with the first Jacobi sweep after it (k_prolong_sweep, levels >= 1,
nsmooth even; odd nsmooth keeps the separate passes and is checked too).  Fused and separate (MGP_TUNE_PROLONG_SWEEP = 1) V- and F-cycles leave
the same bits in u, u_prev, f, r and the face data of every level, in FP64 and FP32, with
Dirichlet and Neumann faces; the FP64 cycles with the fused pass also equal the oracle's (the
cycle tests of tests/test_gpu_parity.py run it with nsmooth 2)."""
import numpy as np
import pytest

from _util import assert_field_equal, make_engine, make_oracle, push, randomize

pytestmark = pytest.mark.gpu

CASES = [
    ((129, 65, 65), 4, (0, 0, 0, 0, 0, 0), "fw"),
    ((129, 65, 65), 4, (1, 1, 1, 1, 0, 0), "fw"),
    ((65, 33, 65), 4, (1, 0, 0, 1, 0, 1), "inj"),
    ((97, 49, 33), 3, (1, 1, 1, 1, 1, 1), "fw"),
]


@pytest.mark.parametrize("ns", [2, 3, 4])
@pytest.mark.parametrize("cycle", ["vcycle", "fcycle"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_fused_matches_separate(mgp_mod, gpu_ready, ci, dtype, cycle, ns):
    dims, levels, bc, rst = CASES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": "jacobi",
           "h": 1.0 / (dims[0] - 1), "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 120 + ci)
    dt = mgp_mod.F64 if dtype == "f64" else mgp_mod.F32
    npdt = np.float64 if dtype == "f64" else np.float32
    engines = []
    for mode in (2, 1):  # fused on every eligible level, separate passes
        e = make_engine(mgp_mod, cfg, dtype=dt)
        for l in range(levels):
            e.set_tuning(l, mgp_mod.TUNE_PROLONG_SWEEP, mode)
            for name in ("u", "uprev", "f", "r"):
                e.upload(name, o.field(name, l).astype(npdt), l)
            for fc in range(6):
                e.upload_face(fc, o.face(fc, l).astype(npdt), l)
        getattr(e, cycle)(0, -1.0, ns)
        getattr(e, cycle)(0, -1.0, ns)
        engines.append(e)
    for l in range(levels):
        for name in ("u", "uprev", "f", "r"):
            a, b = engines[0].download(name, l), engines[1].download(name, l)
            assert np.array_equal(a, b), f"{name}@L{l}: {np.count_nonzero(a != b)} points differ"
        for fc in range(6):
            assert np.array_equal(engines[0].download_face(fc, l), engines[1].download_face(fc, l)), (fc, l)
    for e in engines:
        e.close()


@pytest.mark.parametrize("cycle", ["vcycle", "fcycle"])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_fused_cycles_match_oracle(mgp_mod, gpu_ready, ci, cycle):
    dims, levels, bc, rst = CASES[ci]
    cfg = {"dims": dims, "levels": levels, "bc": bc, "restriction": rst, "relaxation": "jacobi",
           "h": 1.0 / (dims[0] - 1), "strict_bc": True}
    o = make_oracle(cfg)
    randomize(o, 140 + ci)
    e = make_engine(mgp_mod, cfg)
    for l in range(levels):
        e.set_tuning(l, mgp_mod.TUNE_PROLONG_SWEEP, 2)
    push(o, e)
    om = o.default_omega()
    for ns in (3, 2):
        getattr(o, cycle)(0, om, ns)
        getattr(e, cycle)(0, om, ns)
    for l in range(levels):
        for name in ("u", "f"):
            assert_field_equal(o, e, name, l)
    e.close()

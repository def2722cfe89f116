"""CPU: the C ABI library loads, exports every symbol include/mgp.h declares, and its
device-free planning entry point reproduces the reference's level geometry, halo widths,
strides and boundary-kind resolution (checked against the oracle's own layout)."""
import ctypes
import itertools
import re

import pytest

from conftest import ROOT
from oracle.oracle import Oracle

HEADER = ROOT / "include" / "mgp.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s+(mgp_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("mgp_create", "mgp_destroy", "mgp_solve", "mgp_upload_field", "mgp_download_field",
                 "mgp_relax", "mgp_residual", "mgp_restrict", "mgp_prolong", "mgp_norm", "mgp_plan_level"):
        assert must in names


def test_library_exports_every_declared_symbol(mgp_mod):
    lib = mgp_mod.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"libmgp.so lacks {missing}"


def plan(mgp, dims, levels, bc, relaxation=0, strict=False, level=0, dtype=0):
    d = mgp.Desc()
    d.dims[:] = list(dims)
    d.levels, d.maxiter, d.miniter, d.tolerance, d.h = levels, 10, 1, 0.0, 1.0 / max(1, dims[0] - 1)
    d.bc[:] = list(bc)
    d.restriction, d.prolongation, d.relaxation, d.dtype, d.device = 0, 0, relaxation, dtype, 0
    d.flags = 1 if strict else 0
    li = mgp.LevelInfo()
    st = mgp.lib().mgp_plan_level(ctypes.byref(d), level, ctypes.byref(li))
    return st, li


@pytest.mark.parametrize("bc", list(itertools.product((0, 1), repeat=6))[::5])
@pytest.mark.parametrize("strict", [False, True])
def test_plan_matches_oracle_layout(mgp_mod, bc, strict):
    dims, levels = (33, 17, 9), 3
    o = Oracle(dims, levels, 1 / 32, bc, 0, 0, strict)
    for l in range(levels):
        st, li = plan(mgp_mod, dims, levels, bc, 0, strict, l)
        assert st == 0, mgp_mod.lib().mgp_last_error()
        m = o.meta[l]
        assert tuple(li.shape) == m.shape
        assert tuple(li.pad) == m.pad
        assert tuple(li.stride) == m.stride
        assert li.size == m.size
        assert li.h == m.h
        halo = dict(zip(("east", "west", "north", "south", "top", "bottom"), li.halo))
        assert halo == m.halo
        assert list(li.face_kind) == list(o.face_types)


def test_plan_resolves_boundaries_like_reference(mgp_mod):
    # BoundaryCondition {N,N,N,N,D,D}: north/south become Dirichlet (domain.h:191-192) but keep
    # their halo layers; bottom is always Dirichlet (domain.h:140-145).
    st, li = plan(mgp_mod, (513, 257, 129), 6, (1, 1, 1, 1, 0, 0))
    assert st == 0
    assert list(li.face_kind) == [0, 0, 1, 1, 0, 0]
    assert tuple(li.pad) == (515, 259, 129)
    assert tuple(li.stride) == (259 * 129, 129, 1)
    st, li = plan(mgp_mod, (17, 17, 17), 3, (0, 0, 0, 0, 0, 1))
    assert list(li.face_kind) == [0] * 6 and li.halo[5] == 1
    st, li = plan(mgp_mod, (17, 17, 17), 3, (1, 1, 0, 0, 0, 1), strict=True)
    assert list(li.face_kind) == [1, 1, 0, 0, 0, 1]


def test_plan_level_geometry(mgp_mod):
    for l, want in enumerate([(513, 257, 129), (257, 129, 65), (129, 65, 33), (65, 33, 17), (33, 17, 9), (17, 9, 5)]):
        st, li = plan(mgp_mod, (513, 257, 129), 6, (1, 1, 1, 1, 0, 0), level=l)
        assert st == 0 and tuple(li.shape) == want
        assert li.h == pytest.approx(2.0 ** l / 512, rel=0, abs=0)


def test_plan_rejects_non_coarsenable_dims(mgp_mod):
    st, _ = plan(mgp_mod, (64, 33, 33), 3, (0,) * 6)
    assert st == mgp_mod.ERR_INVALID_ARG
    assert "Invalid grid of size" in mgp_mod.lib().mgp_last_error().decode()


def test_plan_rejects_bad_descriptor(mgp_mod):
    assert plan(mgp_mod, (1, 9, 9), 1, (0,) * 6)[0] == mgp_mod.ERR_INVALID_ARG
    assert plan(mgp_mod, (9, 9, 9), 0, (0,) * 6)[0] == mgp_mod.ERR_INVALID_ARG
    assert plan(mgp_mod, (9, 9, 9), 2, (0, 0, 0, 0, 0, 2))[0] == mgp_mod.ERR_INVALID_ARG


def test_plan_detects_degenerate_gauss_seidel_colouring(mgp_mod):
    # exactly one of top/bottom requested non-Dirichlet: padded z extent even, the
    # reference's idx%2 colouring becomes z-plane parity (racy in the reference)
    st, _ = plan(mgp_mod, (17, 17, 17), 3, (0, 0, 0, 0, 1, 0), relaxation=1)
    assert st == mgp_mod.ERR_UNSUPPORTED
    assert "degenerate" in mgp_mod.lib().mgp_last_error().decode()
    # padded y extent even only: supported (column order), and Jacobi is never affected
    assert plan(mgp_mod, (17, 17, 17), 3, (1, 0, 0, 0, 0, 0), relaxation=1)[0] == 0
    assert plan(mgp_mod, (17, 17, 17), 3, (0, 0, 0, 0, 1, 0), relaxation=0)[0] == 0
    # a single-level even grid degenerates too
    assert plan(mgp_mod, (16, 16, 16), 1, (0,) * 6, relaxation=1)[0] == mgp_mod.ERR_UNSUPPORTED


def test_status_strings(mgp_mod):
    lib = mgp_mod.lib()
    assert lib.mgp_status_string(0) == b"ok"
    assert lib.mgp_status_string(7) == b"unsupported"
    assert lib.mgp_abi_version() == 1


def test_create_without_device_reports_no_device_or_succeeds(mgp_mod):
    """On a CPU-only machine mgp_create must fail cleanly with NO_DEVICE (never crash)."""
    if mgp_mod.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(mgp_mod.MgpError) as ei:
        mgp_mod.Solver((9, 9, 9), 2, 0.125)
    assert ei.value.status == mgp_mod.ERR_NO_DEVICE


def test_missing_engine_library_fails_loudly(mgp_mod, monkeypatch, tmp_path):
    """No CPU fallback: without libmgp.so every entry point of the Python layer raises."""
    monkeypatch.setattr(mgp_mod, "_lib", None)
    monkeypatch.setattr(mgp_mod, "LIB_PATH", tmp_path / "libmgp.so")
    monkeypatch.setattr(mgp_mod._build, "needs_build", lambda: False)
    with pytest.raises(RuntimeError, match="library missing"):
        mgp_mod.lib()
    with pytest.raises(RuntimeError, match="library missing"):
        mgp_mod.Solver((9, 9, 9), 2, 0.125)

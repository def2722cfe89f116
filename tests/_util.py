"""Shared helpers for the parity tests: build an oracle/engine pair on the same hierarchy,
fill the oracle with a seeded random state, mirror it into the engine and compare."""
from __future__ import annotations

import hashlib
import json

import numpy as np

from oracle.oracle import FACES, FIELDS, Oracle

BC_D, BC_N = 0, 1


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def rst_id(name: str) -> int:
    return {"inj": 0, "fw": 1}[name]


def rlx_id(name: str) -> int:
    return {"jacobi": 0, "gs": 1}[name]


def make_oracle(cfg: dict) -> Oracle:
    return Oracle(cfg["dims"], cfg["levels"], cfg["h"], tuple(cfg["bc"]), rst_id(cfg["restriction"]),
                  rlx_id(cfg["relaxation"]), cfg.get("strict_bc", False))


def make_engine(mgp, cfg: dict, dtype=None, maxiter=None, tol=None, flags=0):
    return mgp.Solver(cfg["dims"], cfg["levels"], cfg["h"], tuple(cfg["bc"]), rst_id(cfg["restriction"]),
                      rlx_id(cfg["relaxation"]), dtype if dtype is not None else mgp.F64,
                      maxiter if maxiter is not None else cfg.get("maxiter", 10), 1,
                      tol if tol is not None else cfg.get("tol", 0.0), tuple(cfg.get("origin", (0, 0, 0))),
                      0, cfg.get("strict_bc", False), flags=flags)


def randomize(o: Oracle, seed: int, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    for l in range(o.levels):
        for name in FIELDS:
            if name == "uprev" and o.relaxation != 0:
                continue
            o.field(name, l)[...] = rng.uniform(lo, hi, size=o.meta[l].pad)
        for fc in range(6):
            o.face(fc, l)[...] = rng.uniform(lo, hi, size=o.face(fc, l).shape)


def push(o: Oracle, e, levels=None, fields=FIELDS):
    """Copy the oracle's state (all levels by default) into the engine."""
    for l in range(o.levels) if levels is None else levels:
        for name in fields:
            if name == "uprev" and o.relaxation != 0:
                continue
            e.upload(name, o.field(name, l), l)
        for fc in range(6):
            e.upload_face(fc, o.face(fc, l), l)


def shape_of(arr_padded: np.ndarray, meta) -> np.ndarray:
    return arr_padded[meta.interior]


def assert_field_equal(o: Oracle, e, name: str, level: int, where=None, exact=True, rtol=0.0):
    got = shape_of(e.download(name, level), e.level[level])
    want = shape_of(o.field(name, level), o.meta[level])
    if where is not None:
        got, want = got[where], want[where]
    if exact:
        if not np.array_equal(got, want):
            d = np.abs(got.astype(np.float64) - want)
            idx = np.unravel_index(np.argmax(d), d.shape)
            raise AssertionError(f"{name}@L{level} differs: max|d|={d.max():.3e} at {idx} "
                                 f"got={got[idx]!r} want={want[idx]!r} ({np.count_nonzero(d)} points)")
    else:
        scale = max(1e-300, float(np.max(np.abs(want))))
        err = float(np.max(np.abs(got.astype(np.float64) - want))) / scale
        assert err <= rtol, f"{name}@L{level}: relative max error {err:.3e} > {rtol:.1e}"


def assert_face_equal(o: Oracle, e, fc: int, level: int):
    got = e.download_face(fc, level)
    want = o.face(fc, level)
    if not np.array_equal(got, want):
        d = np.abs(got - want)
        raise AssertionError(f"face {FACES[fc]}@L{level} differs: max|d|={d.max():.3e}")


def golden_cfg(entry: dict) -> dict:
    cfg = dict(entry)
    cfg["dims"] = tuple(entry["dims"])
    cfg["bc"] = tuple(entry["bc"])
    return cfg


def load_ops(npz) -> dict:
    cases = {}
    for key in npz.files:
        name, rest = key.split("/", 1)
        cases.setdefault(name, {})[rest] = npz[key]
    for name, d in cases.items():
        d["meta"] = json.loads(str(d["meta"][0]))
    return cases

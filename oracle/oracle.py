"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live here, and nothing in the product path imports this module:

* ``Oracle``: ctypes wrapper over ``oracle/mgp_oracle.c`` (the C restatement of the
  reference's PoissonSolver hot path, built into ``oracle/liborc.so``).
* ``RefRun``: runs ``oracle/_ref/ref_oracle`` -- the reference's own code compiled from its
  sources by ``oracle/build_ref.sh`` with ``oracle/ref_harness.cpp`` -- and reads back the
  level hierarchy it dumps.  Only available where that binary was built.

Arrays are numpy views/copies in the reference's halo-padded layout
(include/array.h:70-77 of the reference): shape ``pad`` = shape + halo, k unit-stride.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liborc.so"
REF_BIN = HERE / "_ref" / "ref_oracle"

FACES = ("north", "south", "east", "west", "top", "bottom")  # reference Location_t order
FIELDS = ("u", "uprev", "f", "r")
D, N = 0, 1
INJECTION, FULLWEIGHTING = 0, 1
JACOBI, GAUSSSEIDEL = 0, 1
CYCLES = {"relaxation": 0, "Relaxation": 0, "vcycle": 1, "Vcycle": 1, "fcycle": 2, "Fcycle": 2}


def build_oracle(force: bool = False) -> Path:
    """Compile the C restatement (plain IEEE double, no contraction)."""
    src = HERE / "mgp_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        tmp = LIB_PATH.with_suffix(".so.tmp")
        subprocess.check_call(
            ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(tmp), "-lm"]
        )
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def build_ref(ref_dir: str | None = None) -> Path | None:
    """Compile the reference's own CPU path where its sources are present: `ref_dir`, else the
    REF_DIR environment variable, else the installed copy under baseline/_ref.  Without any of
    them the binary built earlier (if any) is returned."""
    candidates = [ref_dir, os.environ.get("REF_DIR"), str(HERE.parent / "baseline" / "_ref")]
    found = next((c for c in candidates if c and Path(c, "include", "libpoisson.h").exists()), None)
    if found is None:
        return REF_BIN if REF_BIN.exists() else None
    src = HERE / "ref_harness.cpp"
    if not REF_BIN.exists() or REF_BIN.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["bash", str(HERE / "build_ref.sh"), found])
    return REF_BIN


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, dp, lp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long)
        L.orc_create.argtypes = [lp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
        L.orc_create.restype = ctypes.c_int
        L.orc_destroy.argtypes = [vp]
        L.orc_level_meta.argtypes = [vp, ctypes.c_int, lp]
        L.orc_level_h.argtypes = [vp, ctypes.c_int]
        L.orc_level_h.restype = ctypes.c_double
        L.orc_face_type.argtypes = [vp, ctypes.c_int]
        L.orc_field.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.orc_field.restype = dp
        L.orc_face.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.orc_face.restype = dp
        L.orc_init_problem.argtypes = [vp, ctypes.c_int, dp]
        L.orc_problem_u.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_problem_u.restype = ctypes.c_double
        for name in ("orc_write_bc", "orc_residual", "orc_restrict", "orc_zero_u", "orc_restrict_bc",
                     "orc_prolong", "orc_add"):
            getattr(L, name).argtypes = [vp, ctypes.c_int]
        L.orc_relax.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_long]
        L.orc_relax_colour.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_vcycle.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_long]
        L.orc_fcycle.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_long]
        L.orc_norm.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.orc_norm.restype = ctypes.c_double
        L.orc_default_omega.argtypes = [vp]
        L.orc_default_omega.restype = ctypes.c_double
        L.orc_solve.argtypes = [vp, ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_long, ctypes.c_long,
                                ctypes.c_double, ctypes.c_double, dp, dp, dp, dp, ctypes.c_long]
        L.orc_solve.restype = ctypes.c_long
        _lib = L
    return _lib


@dataclass
class LevelMeta:
    shape: tuple
    pad: tuple
    stride: tuple
    size: int
    halo: dict  # east west north south top bottom
    h: float

    @property
    def interior(self):
        """Slices selecting the shape points inside the padded array."""
        hw, hs, hb = self.halo["west"], self.halo["south"], self.halo["bottom"]
        nx, ny, nz = self.shape
        return (slice(hw, hw + nx), slice(hs, hs + ny), slice(hb, hb + nz))


def face_shape(shape, fc: int):
    nx, ny, nz = shape
    return [(nx, 1, nz), (nx, 1, nz), (1, ny, nz), (1, ny, nz), (nx, ny, 1), (nx, ny, 1)][fc]


class Oracle:
    """The C restatement of PoissonSolver<double,R,TrilinearInterpolation,S> (one device)."""

    def __init__(self, dims, levels, h, bc=(D,) * 6, restriction=INJECTION, relaxation=GAUSSSEIDEL,
                 strict_bc=False):
        L = lib()
        self._h = ctypes.c_void_p()
        d = (ctypes.c_long * 3)(*dims)
        b = (ctypes.c_int * 6)(*bc)
        rc = L.orc_create(d, levels, h, b, restriction, relaxation, int(strict_bc), ctypes.byref(self._h))
        if rc == 2:
            raise ValueError(f"Invalid grid of size {tuple(dims)} for {levels} levels")
        if rc != 0:
            raise ValueError("oracle create failed")
        self.levels = levels
        self.relaxation = relaxation
        self.meta = []
        m = (ctypes.c_long * 16)()
        for l in range(levels):
            L.orc_level_meta(self._h, l, m)
            self.meta.append(LevelMeta(tuple(m[0:3]), tuple(m[3:6]), tuple(m[6:9]), m[9],
                                       dict(zip(("east", "west", "north", "south", "top", "bottom"), m[10:16])),
                                       L.orc_level_h(self._h, l)))
        self.face_types = [L.orc_face_type(self._h, f) for f in range(6)]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_destroy(self._h)
            self._h = None

    # numpy views (live, writable)
    def field(self, name: str, level: int = 0) -> np.ndarray:
        p = lib().orc_field(self._h, FIELDS.index(name), level)
        return np.ctypeslib.as_array(p, shape=self.meta[level].pad)

    def face(self, fc, level: int = 0) -> np.ndarray:
        fc = FACES.index(fc) if isinstance(fc, str) else fc
        p = lib().orc_face(self._h, fc, level)
        return np.ctypeslib.as_array(p, shape=face_shape(self.meta[level].shape, fc))

    def shape_view(self, name: str, level: int = 0) -> np.ndarray:
        return self.field(name, level)[self.meta[level].interior]

    def init_problem(self, problem: int, origin=(0.0, 0.0, 0.0)):
        o = (ctypes.c_double * 3)(*origin)
        lib().orc_init_problem(self._h, problem, o)

    def write_bc(self, level=0):
        lib().orc_write_bc(self._h, level)

    def default_omega(self):
        return lib().orc_default_omega(self._h)

    def relax(self, level, omega, nsmooth):
        lib().orc_relax(self._h, level, omega, nsmooth)

    def relax_colour(self, level, omega, colour):
        """One red-black half-sweep of one colour; the alternate flag is left as it was."""
        lib().orc_relax_colour(self._h, level, omega, colour)

    def residual(self, level):
        lib().orc_residual(self._h, level)

    def restrict(self, level):
        lib().orc_restrict(self._h, level)

    def zero_u(self, level):
        lib().orc_zero_u(self._h, level)

    def restrict_bc(self, level):
        lib().orc_restrict_bc(self._h, level)

    def prolong(self, level):
        lib().orc_prolong(self._h, level)

    def add(self, level):
        lib().orc_add(self._h, level)

    def vcycle(self, level, omega, nsmooth):
        lib().orc_vcycle(self._h, level, omega, nsmooth)

    def fcycle(self, level, omega, nsmooth):
        lib().orc_fcycle(self._h, level, omega, nsmooth)

    def norm(self, name, level=0):
        return lib().orc_norm(self._h, FIELDS.index(name), level)

    def solve(self, cycle="Vcycle", nsmooth=10, omega=-1.0, maxiter=100, miniter=1, tol=1e-6, maxtime=1200.0):
        """PoissonSolver::solve; returns (rel_res, iterations, seconds, per-iteration history)."""
        rr, it, tm = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        hist = np.zeros(max(1, maxiter), dtype=np.float64)
        n = lib().orc_solve(self._h, CYCLES[cycle], nsmooth, omega, maxiter, miniter, tol, maxtime,
                            ctypes.byref(rr), ctypes.byref(it), ctypes.byref(tm),
                            hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(hist))
        return rr.value, it.value, tm.value, hist[:n].copy()


def problem_u(problem: int, x: float, y: float, z: float) -> float:
    return lib().orc_problem_u(problem, x, y, z)


# ----------------------------------------------------------------------------------------
@dataclass
class RefState:
    meta: list
    fields: dict = field(default_factory=dict)  # (level, name) -> padded array
    faces: dict = field(default_factory=dict)   # (level, face) -> array
    stats: dict = field(default_factory=dict)
    lines: list = field(default_factory=list)


class RefRun:
    """Run the reference's own code (oracle/_ref/ref_oracle) on one spec."""

    def __init__(self, binary: Path | None = None):
        self.binary = Path(binary) if binary else REF_BIN
        if not self.binary.exists():
            raise FileNotFoundError(f"reference oracle binary not built: {self.binary}")

    @staticmethod
    def _bc_str(bc):
        return " ".join("N" if b else "D" for b in bc)

    def run(self, dims, levels, bc=(D,) * 6, restriction="inj", relaxation="gs", problem=0, mode="solve",
            cycle="Fcycle", nsmooth=2, omega=-1.0, maxiter=10, tol=0.0, h=None, origin=(0.0, 0.0, 0.0),
            ops=(), load: dict | None = None, threads=1, extra: dict | None = None, dump=True, timeout=600):
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            out = td / "out"
            out.mkdir()
            spec = [f"dims {dims[0]} {dims[1]} {dims[2]}", f"levels {levels}", f"maxiter {maxiter}",
                    f"tolerance {tol!r}", f"origin {origin[0]!r} {origin[1]!r} {origin[2]!r}",
                    f"bc {self._bc_str(bc)}", f"restriction {restriction}", f"relaxation {relaxation}",
                    f"problem {problem}", f"mode {mode}", f"cycle {cycle}", f"nsmooth {nsmooth}",
                    f"omega {omega!r}", f"out {out}"]
            if h is not None:
                spec.append(f"h {h!r}")
            if ops:
                spec.append("ops " + " ".join(ops))
            for k, v in (extra or {}).items():
                spec.append(f"{k} {v}")
            if load:
                ld = td / "load"
                ld.mkdir()
                for name, arr in load.items():
                    np.ascontiguousarray(arr, dtype=np.float64).tofile(ld / f"{name}.bin")
                spec.append(f"load {ld}")
            (td / "spec").write_text("\n".join(spec) + "\n")
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            env.pop("OMP_TARGET_OFFLOAD", None)
            p = subprocess.run([str(self.binary), str(td / "spec")], capture_output=True, text=True, env=env,
                               timeout=timeout)
            if p.returncode != 0:
                raise RuntimeError(f"ref_oracle failed: {p.stderr}")
            return self._read(out, levels, p.stdout, dump and mode != "time")

    @staticmethod
    def _read(out: Path, levels: int, stdout: str, dump: bool) -> RefState:
        meta = []
        if dump:
            for line in (out / "meta.txt").read_text().splitlines():
                t = line.split()
                shape = tuple(int(x) for x in t[3:6])
                halo = dict(zip(("east", "west", "north", "south", "top", "bottom"), (int(x) for x in t[7:13])))
                stride = tuple(int(x) for x in t[14:17])
                size = int(t[18])
                hval = float(t[20])
                faces = t[22:28]
                pad = (shape[0] + halo["east"] + halo["west"], shape[1] + halo["north"] + halo["south"],
                       shape[2] + halo["top"] + halo["bottom"])
                lm = LevelMeta(shape, pad, stride, size, halo, hval)
                lm.face_kinds = faces
                meta.append(lm)
        st = RefState(meta)
        for line in stdout.splitlines():
            t = line.split()
            st.lines.append(t)
            if len(t) >= 2 and t[0] in ("rel_res", "iters", "time", "threads", "fnorm", "unorm"):
                st.stats.setdefault(t[0], []).append(float(t[1]))
            if len(t) >= 4 and t[0] == "rnorm":
                st.stats.setdefault("rnorm", []).append(float(t[1]))
                st.stats.setdefault("rel", []).append(float(t[3]))
        if dump:
            for l in range(levels):
                m = meta[l]
                for name in FIELDS:
                    st.fields[(l, name)] = np.fromfile(out / f"L{l}_{name}.bin", dtype=np.float64).reshape(m.pad)
                for fc, fname in enumerate(FACES):
                    st.faces[(l, fname)] = np.fromfile(out / f"L{l}_{fname}.bin", dtype=np.float64).reshape(
                        face_shape(m.shape, fc))
        return st

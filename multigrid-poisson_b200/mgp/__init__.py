"""mgp -- Python binding of the B200 multigrid Poisson engine (libmgp.so, C ABI in include/mgp.h).

Two layers:

* ``Solver``: a thin ctypes wrapper over the C ABI (create / upload / operators / solve).
* ``PoissonSolver``: the reference's public solver API, Poisson::PoissonSolver<T,R,P,S>
  (include/libpoisson.h:28-67 of eljens/multigrid-poisson), with host arrays kept as numpy
  arrays in the reference's halo-padded layout, so code written against the reference's
  ``init_zero / get_rhs / get_top_bc / to_device / solve / to_host / get_solution`` flow
  reads the same.

There is no CPU fallback: every compute call goes to the CUDA engine, and importing this
module on a machine without the built library raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field as dc_field
from pathlib import Path

import numpy as np

from . import _build

LIB_PATH = _build.LIB

OK, ERR_INVALID_ARG, ERR_OOM, ERR_NO_DEVICE, ERR_CUDA, ERR_TIMEOUT, ERR_DIVERGED, ERR_UNSUPPORTED, ERR_STATE = range(9)
DIRICHLET, NEUMANN = 0, 1
NORTH, SOUTH, EAST, WEST, TOP, BOTTOM = range(6)
FACES = ("north", "south", "east", "west", "top", "bottom")
INJECTION, FULLWEIGHTING = 0, 1
TRILINEAR = 0
JACOBI, GAUSSSEIDEL = 0, 1
F64, F32 = 0, 1
FIELD_U, FIELD_UPREV, FIELD_F, FIELD_R = range(4)
FIELDS = ("u", "uprev", "f", "r")
CYCLE_RELAXATION, CYCLE_V, CYCLE_F = 0, 1, 2
FLAG_STRICT_BC = 1
FLAG_FUSED_SETUP = 8
FLAG_REFINE_F32 = 16
FLAG_REFINE_F64 = 32
FLAG_WAVE = 256
SOLVE_VERBOSE, SOLVE_PRINT_CYCLE_TIME = 1, 2
# launch-shape tuning parameters (mgp_set_tuning / mgp_autotune)
(TUNE_RELAX_PLANES, TUNE_RESID_PLANES, TUNE_NORM_PLANES, TUNE_SETUP_FORM, TUNE_SETUP_PLANES, TUNE_WAVE, TUNE_TAIL,
 TUNE_PROLONG_SWEEP) = range(8)
TUNE_PARAMS = 8
AUTOTUNE_FORCE = 1

_RESTRICTIONS = {"Injection": INJECTION, "injection": INJECTION, "inj": INJECTION,
                 "FullWeighting": FULLWEIGHTING, "fullweighting": FULLWEIGHTING, "fw": FULLWEIGHTING}
_RELAXATIONS = {"Jacobi": JACOBI, "jacobi": JACOBI, "GaussSeidel": GAUSSSEIDEL, "gaussseidel": GAUSSSEIDEL,
                "gs": GAUSSSEIDEL}
_CYCLES = {"relaxation": CYCLE_RELAXATION, "Relaxation": CYCLE_RELAXATION, "vcycle": CYCLE_V, "Vcycle": CYCLE_V,
           "fcycle": CYCLE_F, "Fcycle": CYCLE_F}


class MgpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Desc(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int64 * 3), ("levels", ctypes.c_int64), ("maxiter", ctypes.c_int64),
                ("miniter", ctypes.c_int64), ("tolerance", ctypes.c_double), ("h", ctypes.c_double),
                ("origin", ctypes.c_double * 3), ("bc", ctypes.c_int32 * 6), ("restriction", ctypes.c_int32),
                ("prolongation", ctypes.c_int32), ("relaxation", ctypes.c_int32), ("dtype", ctypes.c_int32),
                ("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class LevelInfo(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int64 * 3), ("halo", ctypes.c_int64 * 6), ("pad", ctypes.c_int64 * 3),
                ("stride", ctypes.c_int64 * 3), ("size", ctypes.c_int64), ("h", ctypes.c_double),
                ("origin", ctypes.c_double * 3), ("face_kind", ctypes.c_int32 * 6),
                ("face_shape", (ctypes.c_int64 * 3) * 6)]


class Stats(ctypes.Structure):
    _fields_ = [("rel_res", ctypes.c_double), ("iterations", ctypes.c_double), ("seconds", ctypes.c_double),
                ("cycles_run", ctypes.c_int64), ("first_rel_res", ctypes.c_double),
                ("kernel_launches", ctypes.c_int64)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("restriction", ctypes.c_int32), ("relaxation", ctypes.c_int32), ("inner_dtype", ctypes.c_int32),
                ("cycle", ctypes.c_int32), ("nsmooth", ctypes.c_int64), ("omega", ctypes.c_double),
                ("max_problems", ctypes.c_int64), ("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]


_lib = None


def lib():
    """Load libmgp.so (building it first when sources are newer).  Raises if unavailable."""
    global _lib
    if _lib is None:
        if _build.needs_build():
            _build.build()
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA engine library missing: {LIB_PATH}")
        L = ctypes.CDLL(str(LIB_PATH))
        vp, i64, dbl, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        L.mgp_status_string.restype = ctypes.c_char_p
        L.mgp_status_string.argtypes = [i32]
        L.mgp_last_error.restype = ctypes.c_char_p
        L.mgp_abi_version.restype = i32
        L.mgp_device_count.argtypes = [ctypes.POINTER(i32)]
        L.mgp_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(vp)]
        L.mgp_destroy.argtypes = [vp]
        L.mgp_level_info_get.argtypes = [vp, i32, ctypes.POINTER(LevelInfo)]
        L.mgp_num_levels.argtypes = [vp]
        for n in ("mgp_upload_field", "mgp_download_field", "mgp_upload_face", "mgp_download_face"):
            getattr(L, n).argtypes = [vp, i32, i32, vp, i64]
        L.mgp_field_device.argtypes = [vp, i32, i32, ctypes.POINTER(vp), ctypes.POINTER(i64)]
        L.mgp_face_device.argtypes = [vp, i32, i32, ctypes.POINTER(vp), ctypes.POINTER(i64)]
        L.mgp_write_bc.argtypes = [vp, i32]
        L.mgp_solve.argtypes = [vp, i32, i64, dbl, ctypes.c_char_p, dbl, ctypes.c_uint32, ctypes.POINTER(Stats)]
        L.mgp_set_iteration_limits.argtypes = [vp, i64, i64, dbl]
        L.mgp_relax.argtypes = [vp, i32, dbl, i64]
        L.mgp_relax_colour.argtypes = [vp, i32, dbl, i32]
        L.mgp_set_wait_polls.argtypes = [vp, i64]
        L.mgp_set_tuning.argtypes = [vp, i32, i32, i64]
        L.mgp_get_tuning.argtypes = [vp, i32, i32, ctypes.POINTER(i64)]
        L.mgp_autotune.argtypes = [vp, i32, i64, dbl, ctypes.c_uint32, ctypes.POINTER(dbl), ctypes.POINTER(dbl)]
        L.mgp_relax_residual.argtypes = [vp, i32, dbl, i64, ctypes.POINTER(ctypes.c_double)]
        for n in ("mgp_residual", "mgp_restrict", "mgp_zero_u", "mgp_restrict_bc", "mgp_prolong", "mgp_add",
                  "mgp_prolong_add"):
            getattr(L, n).argtypes = [vp, i32]
        L.mgp_vcycle.argtypes = [vp, i32, dbl, i64]
        L.mgp_fcycle.argtypes = [vp, i32, dbl, i64]
        L.mgp_norm.argtypes = [vp, i32, i32, ctypes.POINTER(dbl)]
        L.mgp_synchronize.argtypes = [vp]
        L.mgp_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.mgp_batch_create.argtypes = [ctypes.POINTER(BatchDesc), ctypes.POINTER(vp)]
        L.mgp_batch_destroy.argtypes = [vp]
        L.mgp_batch_problem_bytes.argtypes = [ctypes.POINTER(BatchDesc), ctypes.POINTER(Desc), ctypes.POINTER(i64)]
        L.mgp_batch_add.argtypes = [vp, ctypes.POINTER(Desc), ctypes.POINTER(i32)]
        L.mgp_batch_problem.argtypes = [vp, i32, ctypes.POINTER(vp)]
        L.mgp_batch_remove.argtypes = [vp, i32]
        L.mgp_batch_set_active.argtypes = [vp, i32, i32]
        L.mgp_batch_step.argtypes = [vp, ctypes.POINTER(i32)]
        L.mgp_batch_status.argtypes = [vp, i32, ctypes.POINTER(Stats)]
        L.mgp_batch_solve.argtypes = [vp, dbl, i64, ctypes.POINTER(i64)]
        L.mgp_batch_kernel_launches.argtypes = [vp, ctypes.POINTER(i64)]
        L.mgp_batch_mem_info.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
        L.mgp_batch_reserve.argtypes = [vp, ctypes.c_size_t]
        L.mgp_mem_info.argtypes = [i32, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
        dp = ctypes.POINTER(dbl)
        L.mgp_fill_sine_modes.argtypes = [vp, i32, dp, dp, dp, dp, dp]
        L.mgp_fill_uniform.argtypes = [vp, ctypes.c_uint64, dbl, dbl]
        L.mgp_fill_problem.argtypes = [vp, i32]
        L.mgp_u_error.argtypes = [vp, vp, i32, ctypes.POINTER(dbl)]
        L.mgp_batch_restart.argtypes = [vp, i32]
        L.mgp_host_alloc.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t]
        L.mgp_host_free.argtypes = [vp]
        _lib = L
    return _lib


def _check(st: int):
    if st != OK:
        raise MgpError(st, lib().mgp_last_error().decode())


def mem_info(device=0):
    """(free, total) device bytes."""
    f, t = ctypes.c_size_t(), ctypes.c_size_t()
    _check(lib().mgp_mem_info(device, ctypes.byref(f), ctypes.byref(t)))
    return f.value, t.value


def device_count() -> int:
    n = ctypes.c_int()
    _check(lib().mgp_device_count(ctypes.byref(n)))
    return n.value


def _np_dtype(dtype: int):
    return np.float64 if dtype == F64 else np.float32


def host_array(shape, dtype, pinned: bool = False) -> np.ndarray:
    """A zeroed numpy array; with pinned=True its memory is page-locked (mgp_host_alloc) and
    released when the array is garbage-collected."""
    if not pinned:
        return np.zeros(shape, dtype=dtype)
    import weakref

    n = int(np.prod(shape))
    nbytes = max(1, n * np.dtype(dtype).itemsize)
    p = ctypes.c_void_p()
    _check(lib().mgp_host_alloc(ctypes.byref(p), nbytes))
    ctype = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float
    buf = (ctype * n).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dtype).reshape(shape)
    arr[...] = 0
    weakref.finalize(buf, lib().mgp_host_free, p.value)
    return arr


# ----------------------------------------------------------------------------------------
@dataclass
class Level:
    shape: tuple
    halo: dict
    pad: tuple
    stride: tuple
    size: int
    h: float
    face_kind: tuple
    face_shape: tuple

    @property
    def interior(self):
        """Slices selecting the shape points of a padded host array."""
        hw, hs, hb = self.halo["west"], self.halo["south"], self.halo["bottom"]
        nx, ny, nz = self.shape
        return (slice(hw, hw + nx), slice(hs, hs + ny), slice(hb, hb + nz))


class DeviceView:
    """A solver's device buffer described by __cuda_array_interface__ (version 3); keeps the
    solver alive while the view exists."""

    def __init__(self, ptr, shape, strides, dtype, owner):
        self.ptr, self.shape, self.strides, self.dtype, self._owner = ptr, shape, strides, np.dtype(dtype), owner

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "strides": self.strides, "typestr": self.dtype.str, "data": (self.ptr, False),
                "version": 3, "stream": None}


class Solver:
    """One level hierarchy on one GPU, driven through the C ABI."""

    def __init__(self, dims, levels, h, bc=(DIRICHLET,) * 6, restriction=INJECTION, relaxation=GAUSSSEIDEL,
                 dtype=F64, maxiter=100, miniter=1, tolerance=1e-6, origin=(0.0, 0.0, 0.0), device=0,
                 strict_bc=False, flags=0, _handle=None):
        L = lib()
        self._owned = _handle is None
        d = make_desc(dims, levels, h, bc, restriction, relaxation, dtype, maxiter, miniter, tolerance, origin, device,
                      strict_bc, flags)
        if _handle is not None:
            self._h = ctypes.c_void_p(_handle)
            self._init_levels(d, levels)
            return
        self._h = ctypes.c_void_p()
        _check(L.mgp_create(ctypes.byref(d), ctypes.byref(self._h)))
        self._init_levels(d, levels)

    def _init_levels(self, d, levels):
        L = lib()
        self.desc = d
        self.dtype = d.dtype
        self.np_dtype = _np_dtype(d.dtype)
        self.levels = levels
        self.level = []
        for l in range(L.mgp_num_levels(self._h)):
            li = LevelInfo()
            _check(L.mgp_level_info_get(self._h, l, ctypes.byref(li)))
            self.level.append(Level(tuple(li.shape), dict(zip(("east", "west", "north", "south", "top", "bottom"),
                                                                   li.halo)),
                                    tuple(li.pad), tuple(li.stride), li.size, li.h, tuple(li.face_kind),
                                    tuple(tuple(li.face_shape[f]) for f in range(6))))

    def close(self):
        if not getattr(self, "_owned", True):
            return
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.mgp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- data movement (reference layout on the host) ----
    def _fid(self, name):
        return FIELDS.index(name) if isinstance(name, str) else name

    def _face_id(self, fc):
        return FACES.index(fc) if isinstance(fc, str) else fc

    def empty_field(self, level=0):
        return np.zeros(self.level[level].pad, dtype=self.np_dtype)

    def upload(self, name, arr, level=0):
        a = np.ascontiguousarray(arr, dtype=self.np_dtype)
        assert a.size == self.level[level].size, (a.shape, self.level[level].pad)
        _check(lib().mgp_upload_field(self._h, self._fid(name), level, a.ctypes.data, a.size))

    def download(self, name, level=0, out=None):
        a = out if out is not None else self.empty_field(level)
        assert a.flags.c_contiguous and a.dtype == self.np_dtype and a.size == self.level[level].size
        _check(lib().mgp_download_field(self._h, self._fid(name), level, a.ctypes.data, a.size))
        return a

    def upload_face(self, fc, arr, level=0):
        a = np.ascontiguousarray(arr, dtype=self.np_dtype)
        _check(lib().mgp_upload_face(self._h, self._face_id(fc), level, a.ctypes.data, a.size))

    def download_face(self, fc, level=0):
        fcid = self._face_id(fc)
        a = np.zeros(self.level[level].face_shape[fcid], dtype=self.np_dtype)
        _check(lib().mgp_download_face(self._h, fcid, level, a.ctypes.data, a.size))
        return a

    def device_field(self, name, level=0) -> "DeviceView":
        """The device buffer holding field `name` of `level`, as an object with
        __cuda_array_interface__ (torch.as_tensor / cupy.asarray wrap it without a copy):
        shape (nx, ny, nz), k unit-stride, the engine's row and plane pitches.  For u / uprev of
        a Jacobi solver it is the buffer that holds the field now; every sweep swaps the pair."""
        p = ctypes.c_void_p()
        lay = (ctypes.c_int64 * 5)()
        _check(lib().mgp_field_device(self._h, self._fid(name), level, ctypes.byref(p), lay))
        es = np.dtype(self.np_dtype).itemsize
        return DeviceView(p.value, (lay[0], lay[1], lay[2]), (lay[3] * es, lay[4] * es, es), self.np_dtype, self)

    def device_face(self, fc, level=0) -> "DeviceView":
        """The device face array `fc` of `level` (dense, the reference's face layout)."""
        p = ctypes.c_void_p()
        shp = (ctypes.c_int64 * 3)()
        _check(lib().mgp_face_device(self._h, self._face_id(fc), level, ctypes.byref(p), shp))
        es = np.dtype(self.np_dtype).itemsize
        shape = (shp[0], shp[1], shp[2])
        return DeviceView(p.value, shape, (shape[1] * shape[2] * es, shape[2] * es, es), self.np_dtype, self)

    def write_bc(self, level=0):
        _check(lib().mgp_write_bc(self._h, level))

    # ---- operators ----
    def relax(self, level, omega=-1.0, nsmooth=1):
        _check(lib().mgp_relax(self._h, level, omega, nsmooth))

    def relax_colour(self, level, omega=-1.0, colour=0):
        """One red-black half-sweep of one colour (mgp_relax_colour); alternate flag untouched."""
        _check(lib().mgp_relax_colour(self._h, level, omega, colour))

    def set_wait_polls(self, polls):
        """Bound of the wavefront passes' waits for a plane copy (0: the default)."""
        _check(lib().mgp_set_wait_polls(self._h, polls))

    def set_tuning(self, level, param, value):
        """Launch shape of one level's kernels (TUNE_*; 0 = the built-in choice)."""
        _check(lib().mgp_set_tuning(self._h, level, param, value))

    def get_tuning(self, level, param):
        v = ctypes.c_int64()
        _check(lib().mgp_get_tuning(self._h, level, param, ctypes.byref(v)))
        return v.value

    def tuning(self):
        """All levels' tuning parameters: one list of TUNE_PARAMS values per level."""
        return [[self.get_tuning(l, p) for p in range(TUNE_PARAMS)] for l in range(self.levels)]

    def autotune(self, cycle="Fcycle", nsmooth=2, omega=-1.0, force=False):
        """Searches the launch shapes for the fastest solve iteration of (cycle, nsmooth) and keeps
        them (fields restored afterwards).  Returns {"untuned_ms", "tuned_ms", "params"}; the two
        times are 0 when the process cache answered."""
        cyc = cycle if isinstance(cycle, int) else _CYCLES[cycle]
        u, t = ctypes.c_double(), ctypes.c_double()
        _check(lib().mgp_autotune(self._h, cyc, nsmooth, omega, AUTOTUNE_FORCE if force else 0, ctypes.byref(u),
                                  ctypes.byref(t)))
        return {"untuned_ms": u.value, "tuned_ms": t.value, "params": self.tuning()}

    def relax_residual(self, level, omega=-1.0, nsmooth=1, norm=True):
        """relax, then residual (and the max-norm of r when `norm`): returns the norm or None."""
        out = ctypes.c_double()
        _check(lib().mgp_relax_residual(self._h, level, omega, nsmooth, ctypes.byref(out) if norm else None))
        return out.value if norm else None

    def residual(self, level):
        _check(lib().mgp_residual(self._h, level))

    def restrict(self, level):
        _check(lib().mgp_restrict(self._h, level))

    def zero_u(self, level):
        _check(lib().mgp_zero_u(self._h, level))

    def restrict_bc(self, level):
        _check(lib().mgp_restrict_bc(self._h, level))

    def prolong(self, level):
        _check(lib().mgp_prolong(self._h, level))

    def prolong_add(self, level):
        _check(lib().mgp_prolong_add(self._h, level))

    def add(self, level):
        _check(lib().mgp_add(self._h, level))

    def vcycle(self, level=0, omega=-1.0, nsmooth=2):
        _check(lib().mgp_vcycle(self._h, level, omega, nsmooth))

    def fcycle(self, level=0, omega=-1.0, nsmooth=2):
        _check(lib().mgp_fcycle(self._h, level, omega, nsmooth))

    def norm(self, name, level=0):
        out = ctypes.c_double()
        _check(lib().mgp_norm(self._h, self._fid(name), level, ctypes.byref(out)))
        return out.value

    def synchronize(self):
        _check(lib().mgp_synchronize(self._h))

    def fill_sine_modes(self, amp, kx, ky, kz, L):
        """Device-side level-0 f = sum_m amp sin(kx pi x/Lx) sin(ky pi y/Ly) sin(kz pi z/Lz)."""
        n = len(amp)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (amp, kx, ky, kz, L)]
        ptr = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in arrs]
        _check(lib().mgp_fill_sine_modes(self._h, n, *ptr))

    def fill_problem(self, problem):
        """Device-side init() for the reference's test problems 1, 2, 3 (f, faces, u = 0 + Dirichlet data)."""
        _check(lib().mgp_fill_problem(self._h, problem))

    def u_error(self, ref=None, problem=0):
        """(max-abs error, relative L2 error, max |v|) of level-0 u against `ref` (a Solver) or the
        analytic solution of test problem `problem`."""
        out = (ctypes.c_double * 4)()
        _check(lib().mgp_u_error(self._h, ref._h if ref is not None else None, problem, out))
        return out[0], (out[1] / out[2] if out[2] > 0 else float("nan")), out[3]

    def fill_uniform(self, seed, lo=-1.0, hi=1.0):
        """Device-side level-0 f: independent uniform values in [lo, hi) (splitmix64 counter)."""
        _check(lib().mgp_fill_uniform(self._h, int(seed) & (2 ** 64 - 1), lo, hi))

    @property
    def stream_handle(self) -> int:
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        out = ctypes.c_void_p()
        _check(lib().mgp_get_stream(self._h, ctypes.byref(out)))
        return out.value or 0

    def set_iteration_limits(self, maxiter, miniter=1, tolerance=1e-6):
        _check(lib().mgp_set_iteration_limits(self._h, maxiter, miniter, tolerance))

    def solve(self, cycle="Vcycle", nsmooth=10, omega=-1.0, ofile="", maxtime=20 * 60.0, verbose=False,
              print_cycle_time=False):
        st = Stats()
        flags = (SOLVE_VERBOSE if verbose else 0) | (SOLVE_PRINT_CYCLE_TIME if print_cycle_time else 0)
        cyc = cycle if isinstance(cycle, int) else _CYCLES.get(cycle)
        if cyc is None:
            raise ValueError(f'solver must be "Relaxation", "Vcycle" of "Fcycle" but was "{cycle}"')
        _check(lib().mgp_solve(self._h, cyc, nsmooth, omega, (ofile or "").encode(), maxtime, flags,
                               ctypes.byref(st)))
        return st


def make_desc(dims, levels, h, bc=(DIRICHLET,) * 6, restriction=INJECTION, relaxation=GAUSSSEIDEL, dtype=F64,
              maxiter=100, miniter=1, tolerance=1e-6, origin=(0.0, 0.0, 0.0), device=0, strict_bc=False, flags=0):
    d = Desc()
    d.dims[:] = list(dims)
    d.levels, d.maxiter, d.miniter, d.tolerance, d.h = levels, maxiter, miniter, tolerance, h
    d.origin[:] = list(origin)
    d.bc[:] = list(bc)
    d.restriction = restriction if isinstance(restriction, int) else _RESTRICTIONS[restriction]
    d.prolongation = TRILINEAR
    d.relaxation = relaxation if isinstance(relaxation, int) else _RELAXATIONS[relaxation]
    d.dtype = dtype
    d.device = device
    d.flags = (FLAG_STRICT_BC if strict_bc else 0) | flags
    return d


class Batch:
    """Many independent problems solved together (C ABI mgp_batch_*): every level operation
    of every problem at the same depth runs as one persistent kernel over a (problem, tile)
    work list.  Each problem is a refinement solver: FP64 level 0, correction hierarchy in
    `inner_dtype`."""

    def __init__(self, restriction=FULLWEIGHTING, relaxation=GAUSSSEIDEL, inner_dtype=F32, cycle="Fcycle",
                 nsmooth=2, omega=-1.0, max_problems=256, device=0):
        bd = BatchDesc()
        bd.restriction = restriction if isinstance(restriction, int) else _RESTRICTIONS[restriction]
        bd.relaxation = relaxation if isinstance(relaxation, int) else _RELAXATIONS[relaxation]
        bd.inner_dtype = inner_dtype
        bd.cycle = cycle if isinstance(cycle, int) else _CYCLES[cycle]
        bd.nsmooth, bd.omega, bd.max_problems, bd.device, bd.flags = nsmooth, omega, max_problems, device, 0
        self.bdesc = bd
        self._h = ctypes.c_void_p()
        _check(lib().mgp_batch_create(ctypes.byref(bd), ctypes.byref(self._h)))
        self._views = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.mgp_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        self.close()

    def problem_bytes(self, dims, levels, h, bc=(DIRICHLET,) * 6, strict_bc=False) -> int:
        d = make_desc(dims, levels, h, bc, strict_bc=strict_bc)
        out = ctypes.c_int64()
        _check(lib().mgp_batch_problem_bytes(ctypes.byref(self.bdesc), ctypes.byref(d), ctypes.byref(out)))
        return out.value

    def add(self, dims, levels, h, bc=(DIRICHLET,) * 6, origin=(0.0, 0.0, 0.0), strict_bc=False) -> int:
        d = make_desc(dims, levels, h, bc, self.bdesc.restriction, self.bdesc.relaxation, F64, origin=origin,
                      device=self.bdesc.device, strict_bc=strict_bc)
        pid = ctypes.c_int()
        _check(lib().mgp_batch_add(self._h, ctypes.byref(d), ctypes.byref(pid)))
        hp = ctypes.c_void_p()
        _check(lib().mgp_batch_problem(self._h, pid.value, ctypes.byref(hp)))
        self._views[pid.value] = Solver(dims, levels, h, bc, self.bdesc.restriction, self.bdesc.relaxation, F64,
                                        origin=origin, _handle=hp.value)
        return pid.value

    def problem(self, pid) -> "Solver":
        """The problem's solver (uploads, downloads, write_bc); owned by the batch."""
        return self._views[pid]

    def remove(self, pid):
        self._views.pop(pid, None)
        _check(lib().mgp_batch_remove(self._h, pid))

    def restart(self, pid):
        _check(lib().mgp_batch_restart(self._h, pid))

    def set_active(self, pid, active=True):
        _check(lib().mgp_batch_set_active(self._h, pid, int(active)))

    def step(self) -> int:
        n = ctypes.c_int()
        _check(lib().mgp_batch_step(self._h, ctypes.byref(n)))
        return n.value

    def status(self, pid) -> Stats:
        st = Stats()
        _check(lib().mgp_batch_status(self._h, pid, ctypes.byref(st)))
        return st

    def solve(self, tol, maxiter=100) -> int:
        k = ctypes.c_int64()
        _check(lib().mgp_batch_solve(self._h, tol, maxiter, ctypes.byref(k)))
        return k.value

    def launches_per_step(self) -> int:
        k = ctypes.c_int64()
        _check(lib().mgp_batch_kernel_launches(self._h, ctypes.byref(k)))
        return k.value

    def reserve(self, nbytes: int):
        """Reserve nbytes of device memory in the batch's pool up front (kept by the pool)."""
        _check(lib().mgp_batch_reserve(self._h, int(nbytes)))

    def mem_info(self):
        """(free, total) device bytes available to this batch: the device's free memory plus
        what the batch's memory pool keeps from retired problems."""
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib().mgp_batch_mem_info(self._h, ctypes.byref(f), ctypes.byref(t)))
        return f.value, t.value


# ----------------------------------------------------------------------------------------
# The reference's public API (include/libpoisson.h, include/settings.h, include/boundary.h)
@dataclass
class Settings:
    """Poisson::Settings (include/settings.h:14-39)."""
    levels: int = 1
    dims: list = dc_field(default_factory=lambda: [3, 3, 3])
    maxiter: int = 100
    miniter: int = 1
    tolerance: float = 1e-6
    lengthx: float = 3.1415
    h: float = 0.33
    origin: list = dc_field(default_factory=lambda: [-0.4, 0.21, 1.23])
    dev: int = 0


@dataclass
class BoundaryCondition:
    """Poisson::BoundaryCondition (include/boundary.h:23-30)."""
    north: int = NEUMANN
    south: int = NEUMANN
    east: int = NEUMANN
    west: int = NEUMANN
    top: int = DIRICHLET
    bottom: int = DIRICHLET

    def as_list(self):
        return [self.north, self.south, self.east, self.west, self.top, self.bottom]


class HostArray:
    """Host side of a DeviceArray<T> (include/devicearray.h): ``at`` is the padded buffer
    and ``idx(i,j,k)`` the reference's halo-aware index (include/array.h:85-87)."""

    def __init__(self, lvl: Level, dtype, pinned: bool = False):
        self.shape = lvl.shape
        self.stride = lvl.stride
        self.halo = lvl.halo
        self.size = lvl.size
        self.arr = host_array(lvl.pad, dtype, pinned)
        self.at = self.arr.reshape(-1)
        self._lvl = lvl

    def idx(self, i, j, k):
        h = self.halo
        return (i + h["west"]) * self.stride[0] + (j + h["south"]) * self.stride[1] + (k + h["bottom"])

    @property
    def view(self):
        """The shape points as an (nx,ny,nz) view."""
        return self.arr[self._lvl.interior]


class BoundaryArray:
    """Host side of Boundary<T>::arr (a face array, no halo)."""

    def __init__(self, shape, dtype, pinned: bool = False):
        self.shape = tuple(shape)
        self.arr = host_array(tuple(shape), dtype, pinned)
        self.at = self.arr.reshape(-1)

    def idx(self, i, j, k):
        return (i * self.shape[1] + j) * self.shape[2] + k


class PoissonSolver:
    """Poisson::PoissonSolver<T, R, TrilinearInterpolation, S> on one B200."""

    def __init__(self, settings: Settings, bc: BoundaryCondition | None = None, restriction="Injection",
                 prolongation="TrilinearInterpolation", relaxation="GaussSeidel", dtype=F64, strict_bc=False,
                 pinned=False, flags=0):
        if prolongation not in ("TrilinearInterpolation", TRILINEAR):
            raise ValueError(f"unknown prolongation {prolongation}")
        self.settings = settings
        self.BC = bc if bc is not None else BoundaryCondition()
        self.engine = Solver(settings.dims, settings.levels, settings.h, self.BC.as_list(), restriction, relaxation,
                             dtype, settings.maxiter, settings.miniter, settings.tolerance, settings.origin,
                             settings.dev, strict_bc, flags=flags)
        lv0 = self.engine.level[0]
        dt = self.engine.np_dtype
        self._fields = {n: HostArray(lv0, dt, pinned) for n in FIELDS}
        self._faces = [BoundaryArray(lv0.face_shape[f], dt, pinned) for f in range(6)]
        self._verbose = False
        self._stats = Stats()

    def verbose(self, onoff: bool):
        self._verbose = bool(onoff)

    def init_zero(self):
        for a in self._fields.values():
            a.arr[...] = 0
        for b in self._faces:
            b.arr[...] = 0

    def init(self, ufun, ffun, dudxfun, dudyfun, dudzfun):
        """PoissonSolver::init with host problem functions (vectorised numpy callables of x, y, z)."""
        st, lv = self.settings, self.engine.level[0]
        x0, y0, z0 = st.origin
        h = st.h
        nx, ny, nz = lv.shape
        self.init_zero()
        I, J, K = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64),
                              np.arange(nz, dtype=np.float64), indexing="ij")
        self._fields["f"].view[...] = ffun(x0 + I * h, y0 + J * h, z0 + K * h)
        offs = [(0, ny - 1, 0), (0, 0, 0), (nx - 1, 0, 0), (0, 0, 0), (0, 0, nz - 1), (0, 0, 0)]
        for fc in range(6):
            fs = lv.face_shape[fc]
            a, b, c = np.meshgrid(np.arange(fs[0], dtype=np.float64), np.arange(fs[1], dtype=np.float64),
                                  np.arange(fs[2], dtype=np.float64), indexing="ij")
            X = x0 + (a + offs[fc][0]) * h
            Y = y0 + (b + offs[fc][1]) * h
            Z = z0 + (c + offs[fc][2]) * h
            if lv.face_kind[fc] == DIRICHLET:
                fn = ufun
            else:
                fn = dudxfun if fc in (EAST, WEST) else dudyfun if fc in (NORTH, SOUTH) else dudzfun
            self._faces[fc].arr[...] = fn(X, Y, Z)

    def to_device(self):
        """Domain::to_device (include/domain.h:245-263): every field, every face, then the
        Dirichlet data into u and u_prev."""
        for n in FIELDS:
            if n == "uprev" and self.engine.desc.relaxation != JACOBI:
                continue
            self.engine.upload(n, self._fields[n].arr)
        for fc in range(6):
            self.engine.upload_face(fc, self._faces[fc].arr)
        self.engine.write_bc(0)

    def to_host(self):
        """Domain::to_host (include/domain.h:265-272): r, u and u_prev."""
        for n in ("r", "u", "uprev"):
            self.engine.download(n, 0, out=self._fields[n].arr)

    def solve(self, solver="Vcycle", nsmooth=10, omega=-1.0, ofile="", maxtime=20 * 60.0):
        if solver not in _CYCLES:
            raise ValueError(f'solver must be "Relaxation", "Vcycle" of "Fcycle" but was "{solver}"')
        self._stats = self.engine.solve(solver, nsmooth, omega, ofile, maxtime, verbose=self._verbose)

    def relative_residual(self):
        return self._stats.rel_res

    def solve_time(self):
        return self._stats.seconds

    def solve_iterations(self):
        return self._stats.iterations

    def get_rhs(self, gpuid=0) -> HostArray:
        return self._fields["f"]

    def get_solution(self, gpuid=0) -> HostArray:
        return self._fields["u"]

    def get_residual(self, gpuid=0) -> HostArray:
        return self._fields["r"]

    def get_top_bc(self, gpuid=0) -> BoundaryArray:
        return self._faces[TOP]

    def get_bottom_bc(self, gpuid=0) -> BoundaryArray:
        return self._faces[BOTTOM]

    def get_bc(self, face) -> BoundaryArray:
        return self._faces[FACES.index(face) if isinstance(face, str) else face]

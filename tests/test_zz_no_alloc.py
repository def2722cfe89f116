"""GPU: mgp_norm_device, the max-norm over a caller-owned device array that allocates nothing
(its scratch is a static device array).  Its result is compared with mgp_norm -- the
solver entry point whose kernel reduces into solver-allocated scratch -- on the same values.
A max-norm is exact in floating point (no rounding), so the tolerance is 0: equal bits.

Named to be collected last, so it also runs after every other GPU test in one process."""
import ctypes

import numpy as np
import pytest

from _util import BC_D, BC_N, make_engine

pytestmark = pytest.mark.gpu

LIMIT = 1 << 28  # points; the static scratch holds 32768 block maxima of 8192 points


def _bind(mgp):
    L = mgp.lib()
    f = L.mgp_norm_device
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                  ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    return f


def _norm_device(mgp, t, dtype, shape=None):
    """mgp_norm_device over torch tensor t (3-D, last axis unit-stride) on t's current stream."""
    import torch

    f = _bind(mgp)
    shp = (ctypes.c_int64 * 3)(*(shape if shape is not None else t.shape))
    st = (ctypes.c_int64 * 2)(t.stride(0), t.stride(1))
    out = ctypes.c_double(-1.0)
    stream = torch.cuda.current_stream(t.device).cuda_stream
    rc = f(t.device.index, t.data_ptr(), dtype, shp, st, stream, ctypes.byref(out))
    return rc, out.value


def _engine_and_values(mgp, dims, dtype, seed, scale=1.0):
    cfg = dict(dims=dims, levels=2, h=1.0 / (max(dims) - 1), bc=(BC_D, BC_D, BC_N, BC_N, BC_N, BC_N),
               restriction="fw", relaxation="jacobi")
    e = make_engine(mgp, cfg, dtype=dtype)
    lv = e.level[0]
    rng = np.random.default_rng(seed)
    host = np.zeros(lv.pad, dtype=e.np_dtype)
    vals = (scale * rng.uniform(-1.0, 1.0, size=lv.shape)).astype(e.np_dtype)
    # plant a negative extreme so |.| matters
    vals[tuple(int(x) for x in rng.integers(0, lv.shape))] = -3.5 * scale
    host[lv.interior] = vals
    e.upload("f", host, 0)
    return e, vals


def _device_copy(vals, pad_z=5):
    """vals on the GPU in a (nx, ny, nz+pad_z) buffer; the padding holds 1e30, which must not
    be read."""
    import torch

    nx, ny, nz = vals.shape
    t = torch.full((nx, ny, nz + pad_z), 1e30, dtype=torch.from_numpy(vals).dtype, device="cuda:0")
    t[:, :, :nz] = torch.from_numpy(vals).to("cuda:0")
    return t[:, :, :nz]


@pytest.mark.parametrize("dtype_name", ["F64", "F32"])
def test_matches_solver_norm_two_calls(mgp_mod, gpu_ready, dtype_name):
    import torch

    dt = getattr(mgp_mod, dtype_name)
    e, vals = _engine_and_values(mgp_mod, (65, 33, 47), dt, seed=11)
    want = e.norm("f", 0)
    t = _device_copy(vals)
    torch.cuda.synchronize()
    got = [_norm_device(mgp_mod, t, dt) for _ in range(2)]
    for rc, v in got:
        assert rc == 0, mgp_mod.lib().mgp_last_error()
        assert v == want, (v, want)
    assert want == float(np.max(np.abs(vals.astype(np.float64))))
    e.close()


def test_sizes_in_a_row_and_multi_block(mgp_mod, gpu_ready):
    """A large array (many blocks, larger maximum) then a small one: the small call must not
    see the large call's block maxima."""
    import torch

    dt = mgp_mod.F64
    e_big, big = _engine_and_values(mgp_mod, (129, 129, 65), dt, seed=5, scale=4.0)
    e_small, small = _engine_and_values(mgp_mod, (17, 9, 33), dt, seed=6)
    tb, ts = _device_copy(big, pad_z=3), _device_copy(small, pad_z=7)
    torch.cuda.synchronize()
    for _ in range(2):
        rc, v = _norm_device(mgp_mod, tb, dt)
        assert rc == 0 and v == e_big.norm("f", 0)
        rc, v = _norm_device(mgp_mod, ts, dt)
        assert rc == 0 and v == e_small.norm("f", 0)
    e_big.close()
    e_small.close()


def test_empty_shape_and_limit(mgp_mod, gpu_ready):
    import torch

    dt = mgp_mod.F64
    t = torch.zeros((4, 4, 4), dtype=torch.float64, device="cuda:0")
    rc, v = _norm_device(mgp_mod, t, dt, shape=(0, 4, 4))
    assert rc == 0 and v == 0.0
    # one point over the static limit: refused on the host before any launch
    rc, _ = _norm_device(mgp_mod, t, dt, shape=(LIMIT // (4 * 4) + 1, 4, 4))
    assert rc == mgp_mod.ERR_INVALID_ARG
    assert b"static scratch limit" in mgp_mod.lib().mgp_last_error()


def test_calls_leave_free_device_memory_unchanged(mgp_mod, gpu_ready):
    """The property the entry point exists for: after its one-time set-up (an empty-shape
    call), many calls on a large array and a small one take no device memory."""
    import torch

    dt = mgp_mod.F64
    e_big, big = _engine_and_values(mgp_mod, (257, 129, 65), dt, seed=8, scale=2.0)
    e_small, small = _engine_and_values(mgp_mod, (17, 9, 33), dt, seed=9)
    tb, ts = _device_copy(big, pad_z=3), _device_copy(small, pad_z=7)
    rc, _ = _norm_device(mgp_mod, tb, dt, shape=(0, 1, 1))
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    want_big, want_small = e_big.norm("f", 0), e_small.norm("f", 0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    for _ in range(50):
        rc, v = _norm_device(mgp_mod, tb, dt)
        assert rc == 0 and v == want_big
    rc, v = _norm_device(mgp_mod, ts, dt)
    assert rc == 0 and v == want_small
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info(0)
    assert free2 == free1, f"free device memory changed by {free1 - free2} bytes over the calls"
    assert free1 == free0
    e_big.close()
    e_small.close()


def test_rejects_a_stream_of_another_device_and_overflowing_strides(mgp_mod, gpu_ready):
    import torch

    dt = mgp_mod.F64
    t = torch.zeros((4, 4, 4), dtype=torch.float64, device="cuda:0")
    f = _bind(mgp_mod)
    out = ctypes.c_double(-1.0)
    shp = (ctypes.c_int64 * 3)(4, 4, 4)
    huge = (ctypes.c_int64 * 2)(1 << 62, 1 << 61)  # stride[1] * ny overflows 64 bits
    rc = f(0, t.data_ptr(), dt, shp, huge, None, ctypes.byref(out))
    assert rc == mgp_mod.ERR_INVALID_ARG
    assert b"overflow" in mgp_mod.lib().mgp_last_error()
    if torch.cuda.device_count() > 1:
        s1 = torch.cuda.Stream(device="cuda:1")
        ok = (ctypes.c_int64 * 2)(16, 4)
        rc = f(0, t.data_ptr(), dt, shp, ok, s1.cuda_stream, ctypes.byref(out))
        assert rc == mgp_mod.ERR_INVALID_ARG

"""GPU: field transfers.  Fields of 8 MiB and more cross PCIe through a device staging copy
of the host layout (one contiguous upload, a repack kernel, long-run download); smaller ones
use a strided 3-D copy.  Both must move exactly the shape points: uploads ignore the host
halo, downloads leave it untouched."""
import zlib

import numpy as np
import pytest

from _util import BC_D, BC_N, make_engine

pytestmark = pytest.mark.gpu

BCS = [
    (BC_N, BC_N, BC_N, BC_N, BC_D, BC_D),   # halo in x and y: downloads in whole (j,k) planes
    (BC_D,) * 6,                              # no halo: one contiguous run
    (BC_N,) * 6,                              # halo everywhere: k rows
    (BC_D, BC_D, BC_D, BC_D, BC_N, BC_D),   # halo in z only
]


@pytest.mark.parametrize("dims", [(129, 129, 129), (33, 17, 17)])
@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("dtype_name", ["F64", "F32"])
def test_round_trip_shape_points_only(mgp_mod, gpu_ready, dims, bc, dtype_name):
    dt = getattr(mgp_mod, dtype_name)
    cfg = dict(dims=dims, levels=2, h=1.0 / (max(dims) - 1), bc=bc, restriction="fw", relaxation="jacobi")
    e = make_engine(mgp_mod, cfg, dtype=dt)
    lv = e.level[0]
    rng = np.random.default_rng(zlib.crc32(repr((dims, bc, dtype_name)).encode()))
    for name in ("u", "f", "r", "uprev"):
        src = rng.uniform(-1, 1, size=lv.pad).astype(e.np_dtype)
        e.upload(name, src, 0)
        sentinel = np.full(lv.pad, 7.25, dtype=e.np_dtype)
        got = e.download(name, 0, out=sentinel)
        inner = np.zeros(lv.pad, dtype=bool)
        inner[lv.interior] = True
        assert np.array_equal(got[inner], src[inner]), name
        assert np.all(got[~inner] == 7.25), name  # halo untouched
        # the device copy holds exactly the shape points
        assert e.norm(name, 0) == float(np.max(np.abs(src[lv.interior].astype(np.float64))))
    e.close()

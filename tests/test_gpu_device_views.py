"""GPU: external coupling on the device.  A caller writes the right-hand side and the boundary
data straight into the solver's device buffers (mgp_field_device / mgp_face_device, the role
the reference's DeviceArray::devptr plays for include/poisson_helpers.h) instead of staging
them through host arrays, and gets the same solve bit for bit; reads through the same views
see what mgp_download_field returns."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS, LEVELS, H = (33, 17, 17), 3, 1.0 / 32
BC = (1, 1, 1, 1, 0, 0)  # Neumann on x and y, Dirichlet on z


def _solver(mgp):
    return mgp.Solver(DIMS, LEVELS, H, BC, mgp.FULLWEIGHTING, mgp.JACOBI, mgp.F64, 4, 4, 0.0)


def test_device_written_data_solve_like_uploaded(mgp_mod, gpu_ready):
    import torch

    rng = np.random.default_rng(5)
    a, b = _solver(mgp_mod), _solver(mgp_mod)
    lv = a.level[0]
    f = a.empty_field(0)
    f[lv.interior] = rng.uniform(-1.0, 1.0, size=lv.shape)
    faces = [rng.uniform(-1.0, 1.0, size=lv.face_shape[fc]) for fc in range(6)]
    # host path
    a.upload("f", f, 0)
    for fc in range(6):
        a.upload_face(fc, faces[fc], 0)
    # device path: the caller's own device writes (here torch copies) into the views
    b.synchronize()
    tf = torch.as_tensor(b.device_field("f", 0), device="cuda")
    assert tuple(tf.shape) == lv.shape
    tf.copy_(torch.from_numpy(np.ascontiguousarray(f[lv.interior])).cuda())
    for fc in range(6):
        torch.as_tensor(b.device_face(fc, 0), device="cuda").copy_(torch.from_numpy(faces[fc]).cuda())
    torch.cuda.synchronize()
    for s in (a, b):
        s.write_bc(0)
        s.solve("Vcycle", 2)
    for name in ("u", "uprev", "r", "f"):
        assert np.array_equal(a.download(name, 0), b.download(name, 0)), name
    for fc in range(6):
        assert np.array_equal(a.download_face(fc, 0), b.download_face(fc, 0)), fc
    a.close()
    b.close()


def test_device_views_read_current_buffers(mgp_mod, gpu_ready):
    """After sweeps swap the Jacobi pair, asking again names the buffer that holds u now."""
    import torch

    rng = np.random.default_rng(9)
    s = _solver(mgp_mod)
    lv = s.level[0]
    f = s.empty_field(0)
    f[lv.interior] = rng.uniform(-1.0, 1.0, size=lv.shape)
    s.upload("f", f, 0)
    for steps in (1, 2, 3):
        s.relax(0, -1.0, steps)
        s.synchronize()
        for name in ("u", "uprev", "f", "r"):
            dev = torch.as_tensor(s.device_field(name, 0), device="cuda").cpu().numpy()
            host = s.download(name, 0)[lv.interior]
            assert np.array_equal(dev, host), (steps, name)
    s.close()

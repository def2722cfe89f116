"""GPU: the continuous-batching server.  Every request's result is the same served alone
and served in the mix (requests joining and leaving the batch between steps), and each
reaches its tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_stream(mgp, n=10, seed=7):
    from mgp import serve

    return serve.make_stream(n, rate=2000.0, seed=seed, kmin=4, kmax=6, tol=1e-8)


@pytest.mark.parametrize("inner", ["F32", "F64"])
def test_served_results_equal_alone_and_in_mix(mgp_mod, gpu_ready, inner):
    from mgp import serve

    dt = getattr(mgp_mod, inner)
    reqs = small_stream(mgp_mod)
    srv = serve.Server(inner=dt, max_batch=6, keep_solutions=True)
    stats = srv.run(reqs)
    srv.close()
    assert stats["converged"] == len(reqs)
    assert stats["max_batch_seen"] > 1  # the requests really overlapped on the device
    for r in reqs:
        assert r.rel_res < r.tol
        alone = serve.make_stream(len(reqs), rate=2000.0, seed=7, kmin=4, kmax=6, tol=1e-8)[r.rid]
        s1 = serve.Server(inner=dt, max_batch=1, keep_solutions=True, pool_bytes=0)
        s1.run([alone])
        s1.close()
        assert alone.iterations == r.iterations
        # same operations in the same order: identical bits (tolerance stated: exact)
        assert np.array_equal(alone.solution, r.solution), r.rid


def test_admission_respects_device_memory(mgp_mod, gpu_ready):
    """With a reserve that leaves room for about one request at a time, requests are admitted
    one after another and all still complete."""
    from mgp import serve

    reqs = small_stream(mgp_mod, n=4, seed=3)
    free, _ = mgp_mod.mem_info(0)
    probe = serve.Server(inner=mgp_mod.F32, max_batch=8)
    need = max(probe.batch.problem_bytes(r.dims, r.levels, r.h, r.bc) for r in reqs)
    probe.close()
    srv = serve.Server(inner=mgp_mod.F32, max_batch=8, reserve_bytes=free - int(1.5 * need))
    stats = srv.run(reqs)
    srv.close()
    assert stats["converged"] == len(reqs)
    assert stats["max_batch_seen"] <= 2


def test_sine_mode_rhs_matches_its_formula(mgp_mod, gpu_ready):
    """The device-side right-hand side of a served request is the sum of its sine modes."""
    from mgp import serve

    req = serve.make_request(3, 0.0, seed=11, kmin=4, kmax=6)
    s = mgp_mod.Solver(req.dims, req.levels, req.h, req.bc, mgp_mod.FULLWEIGHTING, mgp_mod.GAUSSSEIDEL, mgp_mod.F64)
    s.fill_sine_modes(req.amp, req.kx, req.ky, req.kz, req.lengths)
    f = s.download("f", 0)[s.level[0].interior]
    s.close()
    x, y, z = (np.arange(n) * req.h for n in req.dims)
    L = req.lengths
    want = np.zeros(req.dims)
    for a, kx, ky, kz in zip(req.amp, req.kx, req.ky, req.kz):
        want += a * np.sin(kx * np.pi / L[0] * x)[:, None, None] * np.sin(ky * np.pi / L[1] * y)[None, :, None] * \
            np.sin(kz * np.pi / L[2] * z)[None, None, :]
    # tolerance: libm and CUDA sin may differ in the last bit
    assert np.allclose(f, want, rtol=1e-12, atol=1e-13)

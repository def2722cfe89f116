"""CPU: the serving loop's host logic (mgp/serve.py) over a fake batch -- admission by the
server's own free-memory count and the slot limit, retirement at the tolerance or the step
limit, the reused landing buffer's halo, and the latency summary.  No device is touched."""
from types import SimpleNamespace

import numpy as np
import pytest

import mgp.serve as serve


class FakeLevel:
    def __init__(self, dims):
        self.shape = tuple(dims)
        self.halo = {"east": 1, "west": 1, "north": 1, "south": 1, "top": 1, "bottom": 1}
        self.pad = tuple(n + 2 for n in dims)
        self.size = int(np.prod(self.pad))

    @property
    def interior(self):
        nx, ny, nz = self.shape
        return (slice(1, 1 + nx), slice(1, 1 + ny), slice(1, 1 + nz))


class FakeSolver:
    np_dtype = np.float64

    def __init__(self, pid, dims):
        self.pid = pid
        self.level = [FakeLevel(dims)]
        self.filled = False

    def fill_sine_modes(self, amp, kx, ky, kz, lengths):
        self.filled = True

    def download(self, name, level, out):
        # the engine writes the shape points only
        out[self.level[0].interior] = float(self.pid + 1)


class FakeBatch:
    """Problem i converges (rel_res 1e-12) after `need` steps; bytes per problem = points * 8."""

    free = 10_000_000
    instances = []

    def __init__(self, *a, max_problems=64, device=0, **kw):
        self.max = max_problems
        self.probs = {}
        self.next_pid = 0
        self.resident_bytes = 0
        self.peak_resident = 0
        self.peak_count = 0
        self.mem_calls = 0
        FakeBatch.instances.append(self)

    def mem_info(self):
        self.mem_calls += 1
        return FakeBatch.free - self.resident_bytes, FakeBatch.free

    def reserve(self, nbytes):
        pass

    def problem_bytes(self, dims, levels, h, bc):
        return int(np.prod(dims)) * 8

    def add(self, dims, levels, h, bc):
        pid = self.next_pid
        self.next_pid += 1
        need = 2 + (dims[0] % 3)
        self.probs[pid] = SimpleNamespace(s=FakeSolver(pid, dims), steps=0, need=need,
                                          bytes=self.problem_bytes(dims, levels, h, bc))
        self.resident_bytes += self.probs[pid].bytes
        self.peak_resident = max(self.peak_resident, self.resident_bytes)
        self.peak_count = max(self.peak_count, len(self.probs))
        return pid

    def problem(self, pid):
        return self.probs[pid].s

    def remove(self, pid):
        self.resident_bytes -= self.probs[pid].bytes
        del self.probs[pid]

    def step(self):
        for p in self.probs.values():
            p.steps += 1
        return len(self.probs)

    def status(self, pid):
        p = self.probs[pid]
        return SimpleNamespace(iterations=p.steps, rel_res=1e-12 if p.steps >= p.need else 1.0)

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.instances = []
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    monkeypatch.setattr(serve, "host_array", lambda shape, dtype, pinned=False: np.full(shape, 7.0, dtype))
    return FakeBatch


def test_requests_are_deterministic_and_well_formed():
    a = serve.make_stream(20, 100.0, seed=3)
    b = serve.make_stream(20, 100.0, seed=3)
    assert [(r.dims, r.bc, r.kind, r.arrival) for r in a] == [(r.dims, r.bc, r.kind, r.arrival) for r in b]
    assert all(np.array_equal(x.amp, y.amp) for x, y in zip(a, b))
    arrivals = [r.arrival for r in a]
    assert arrivals == sorted(arrivals) and arrivals[0] > 0
    for r in a:
        assert all(((n - 1) & (n - 2)) == 0 and n >= 33 for n in r.dims)  # 2^k + 1, k >= 5
        assert r.levels == int(np.log2(min(r.dims) - 1)) - 1
        if r.kind == "dirichlet":
            assert r.bc == (0,) * 6
        elif r.kind == "neumann":
            assert r.bc == (1, 1, 1, 1, 0, 0)
        else:  # north with south, top with bottom
            assert r.bc[0] == r.bc[1] and r.bc[4] == r.bc[5]


def test_server_admits_by_memory_and_slots_and_retires_everything(fake):
    reqs = serve.make_stream(40, 1e6, seed=1, kmin=5, kmax=6)
    fake.free = 12 * 65 ** 3 * 8  # a handful of the largest requests at a time
    srv = serve.Server(max_batch=8, reserve_bytes=65 ** 3 * 8, pool_bytes=0, keep_solutions=True)
    stats = srv.run(reqs, time_scale=0.0)
    b = fake.instances[-1]
    assert stats["requests"] == 40 and stats["converged"] == 40
    assert b.peak_count <= 8
    assert b.peak_resident <= fake.free - srv.reserve
    assert not b.probs and b.resident_bytes == 0
    assert srv._free is not None and not srv._need
    for r in reqs:
        assert r.iterations == 2 + (r.dims[0] % 3)
        assert r.finished >= r.admitted >= r.arrival * 0.0
        # the shape points carry the download, the reused landing buffer's halo is zero
        u = r.solution
        assert u.shape == tuple(n + 2 for n in r.dims)
        inner = u[1:-1, 1:-1, 1:-1]
        assert np.all(inner == inner.flat[0]) and inner.flat[0] > 0
        halo = u.copy()
        halo[1:-1, 1:-1, 1:-1] = 0
        assert not halo.any()
    assert stats["p99_ms"] >= stats["p50_ms"] >= 0.0
    assert stats["max_batch_seen"] <= 8 and stats["steps"] == len(srv.batch_sizes)


def test_server_asks_the_device_only_when_its_count_refuses(fake):
    reqs = serve.make_stream(30, 1e6, seed=2, kmin=5, kmax=5)
    fake.free = 1 << 40  # never short of memory
    srv = serve.Server(max_batch=4, reserve_bytes=0, pool_bytes=0)
    srv.run(reqs, time_scale=0.0)
    # one query when the count is first needed (the constructor's own query excluded)
    assert fake.instances[-1].mem_calls <= 2


def test_request_larger_than_the_device_is_an_error(fake):
    reqs = serve.make_stream(1, 1e6, seed=4, kmin=6, kmax=6)
    fake.free = 1000
    srv = serve.Server(max_batch=4, reserve_bytes=0, pool_bytes=0)
    with pytest.raises(RuntimeError, match="does not fit"):
        srv.run(reqs, time_scale=0.0)


def test_step_limit_retires_unconverged_requests(fake):
    reqs = serve.make_stream(5, 1e6, seed=5, kmin=5, kmax=5)
    fake.free = 1 << 40
    srv = serve.Server(max_batch=8, reserve_bytes=0, pool_bytes=0, max_steps=1)
    stats = srv.run(reqs, time_scale=0.0)
    assert stats["converged"] == 0
    assert all(r.iterations == 1 for r in reqs)

"""CPU: domain decomposition along x (mgp/decomp.py).  The planner's slabs nest over the levels
and cover every plane once; the decomposed solve -- each slab an oracle hierarchy over its
planes, halo planes exchanged after every operation (after every half-sweep with red-black
smoothing, each slab sweeping the colour that is the one-domain colour in its own layout) --
reproduces the one-domain oracle solve bit for bit at every owned plane, with Jacobi and with
red-black Gauss-Seidel, the slabs in one process and as two gloo ranks."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mgp import decomp
from oracle.oracle import Oracle

RST = {"inj": 0, "fw": 1}
RLX = {"jacobi": 0, "gs": 1}


class OracleSlab:
    """Executor over one slab: the oracle on the slab's planes (the global requested kinds,
    Dirichlet at the cuts), loaded from the global oracle's level-0 state."""

    comm_device = torch.device("cpu")

    def __init__(self, slab, g: Oracle, bc, levels, h, rst, rlx="jacobi"):
        self.slab = slab
        nx, ny, nz = g.meta[0].shape
        self.o = Oracle((slab.nx, ny, nz), levels, h, decomp.slab_bc(slab, bc), RST[rst], RLX[rlx], False)
        m, gm = self.o.meta[0], g.meta[0]
        self.hw = m.halo["west"]
        off = slab.lo + gm.halo["west"] - self.hw  # global padded x index of local padded 0
        for name in fields_of(rlx):
            self.o.field(name, 0)[...] = g.field(name, 0)[off:off + m.pad[0]]
        for fc in range(6):
            gf, lf = g.face(fc, 0), self.o.face(fc, 0)
            if fc in (0, 1, 4, 5):  # north/south/top/bottom: the slab's x range
                lf[...] = gf[slab.lo:slab.hi + 1]
            elif fc == decomp.WEST:
                lf[...] = gf if slab.rank == 0 else g.shape_view("u", 0)[slab.lo][None]
            else:
                lf[...] = gf if slab.rank == slab.parts - 1 else g.shape_view("u", 0)[slab.hi][None]

    def plane(self, field, level, i):
        return self.o.field(field, level)[i + self.o.meta[level].halo["west"]]

    def plane_tensor(self, field, level, i):
        return torch.from_numpy(np.ascontiguousarray(self.plane(field, level, i)))

    def empty_plane(self, field, level):
        return torch.empty(self.plane(field, level, 0).shape, dtype=torch.float64)

    def set_plane(self, field, level, i, values):
        self.o.field(field, level)[i + self.o.meta[level].halo["west"]] = np.asarray(values)

    def relax(self, l, omega, ns):
        self.o.relax(l, omega, ns)

    def relax_colour(self, l, omega, colour):
        self.o.relax_colour(l, omega, colour)

    def layout(self, l):
        m = self.o.meta[l]
        return m.halo["west"], m.pad[1] * m.pad[2]

    def residual(self, l):
        self.o.residual(l)

    def restrict(self, l):
        self.o.restrict(l)

    def restrict_bc(self, l):
        self.o.restrict_bc(l)

    def zero_u(self, l):
        self.o.zero_u(l)

    def prolong_add(self, l):
        self.o.prolong(l)
        self.o.add(l)

    def owned_norm(self, field, slab):
        _, _, olo, ohi = slab.at(0)
        v = self.o.shape_view(field, 0)[slab.local(0, olo):slab.local(0, ohi)]
        return float(np.max(np.abs(v))) if v.size else 0.0

    def owned(self, field):
        _, _, olo, ohi = self.slab.at(0)
        return self.o.shape_view(field, 0)[self.slab.local(0, olo):self.slab.local(0, ohi)].copy()


CASES = [
    # dims, levels, requested bc (N S E W T B), restriction, cycle, nsmooth, parts, relaxation
    ((65, 17, 17), 3, (1, 1, 1, 1, 0, 0), "fw", "Vcycle", 2, 2, "jacobi"),
    ((97, 17, 9), 3, (0, 0, 1, 0, 1, 0), "inj", "Fcycle", 3, 3, "jacobi"),
    ((129, 9, 17), 4, (1, 0, 0, 1, 0, 1), "fw", "Fcycle", 2, 4, "jacobi"),
    ((33, 9, 9), 1, (0, 0, 0, 1, 0, 0), "fw", "Vcycle", 4, 3, "jacobi"),  # one level: relaxation only, H = 1
    # red-black: padded y*z extent odd (N/S alike, T/B alike, odd ny, nz), so slabs whose offset
    # (+ the global west halo) is odd sweep the other local colour
    ((65, 17, 17), 3, (1, 1, 1, 1, 0, 0), "fw", "Vcycle", 2, 2, "gs"),  # Neumann west: every cut slab flips
    ((97, 17, 9), 3, (0, 0, 1, 0, 1, 1), "inj", "Fcycle", 3, 3, "gs"),  # flips on the coarsest level only
    ((129, 17, 17), 4, (1, 1, 0, 1, 0, 0), "fw", "Fcycle", 2, 4, "gs"),
    ((129, 17, 17), 4, (0, 0, 0, 0, 0, 0), "inj", "Vcycle", 3, 3, "gs"),  # all Dirichlet
]
FLIPPING = (4, 5, 6)  # red-black cases where some slab sweeps the other local colour


def fields_of(rlx):
    return ("u", "uprev", "f", "r") if rlx == "jacobi" else ("u", "f", "r")


def global_state(dims, levels, bc, rst, seed, rlx="jacobi"):
    h = 1.0 / (dims[0] - 1)
    g = Oracle(dims, levels, h, bc, RST[rst], RLX[rlx], False)
    rng = np.random.default_rng(seed)
    for name in fields_of(rlx):
        g.field(name, 0)[...] = rng.uniform(-1, 1, size=g.meta[0].pad)
    for fc in range(6):
        g.face(fc, 0)[...] = rng.uniform(-1, 1, size=g.face(fc, 0).shape)
    g.write_bc(0)
    return g, h


def test_plan_slabs_nest_and_cover():
    for nx, levels, parts in ((513, 6, 2), (513, 6, 8), (65, 3, 5), (33, 1, 7), (129, 4, 3)):
        slabs = decomp.plan_slabs(nx, levels, parts)
        H = 1 << (levels - 1)
        for l in range(levels):
            n_l = (nx - 1) // (1 << l) + 1
            owned = []
            for s in slabs:
                lo, hi, olo, ohi = s.at(l)
                assert (s.hi - s.lo) % H == 0
                # the exchanged planes olo-1 and ohi lie inside the slab, off its Dirichlet ends
                # (the west end may be olo-1 itself: it is then never relaxed and only exchanged)
                assert lo <= olo - (1 if s.rank else 0)
                if s.rank < parts - 1:
                    assert ohi <= hi - 1
                else:
                    assert ohi == hi + 1
                owned += list(range(olo, ohi))
            assert owned == list(range(n_l)), (nx, levels, parts, l)
    with pytest.raises(ValueError):
        decomp.plan_slabs(64, 3, 2)
    with pytest.raises(ValueError):
        decomp.plan_slabs(17, 3, 5)


def run_slabs_local(dims, levels, bc, rst, cycle, ns, parts, rlx, seed):
    g, h = global_state(dims, levels, bc, rst, seed, rlx)
    slabs = decomp.plan_slabs(dims[0], levels, parts)
    ex = {s.rank: OracleSlab(s, g, bc, levels, h, rst, rlx) for s in slabs}
    omega = g.default_omega()
    solver = decomp.SlabSolver(slabs, decomp.LocalExchange(ex), levels, omega, maxiter=3, relaxation=rlx,
                               west_halo=g.meta[0].halo["west"])
    rel, it, hist = solver.solve(cycle, ns)
    rr, it_g, _, hist_g = g.solve(cycle, ns, omega, 3, 1, 0.0)
    return g, slabs, ex, solver, (rel, it, hist), (rr, it_g, hist_g)


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_slabs_in_one_process_match_global_solve(ci):
    dims, levels, bc, rst, cycle, ns, parts, rlx = CASES[ci]
    g, slabs, ex, solver, (rel, it, hist), (rr, it_g, hist_g) = run_slabs_local(dims, levels, bc, rst, cycle, ns,
                                                                                parts, rlx, 100 + ci)
    assert rel == rr and it == it_g
    assert hist[1:] == list(hist_g)  # the oracle's history starts after the initial residual
    for name in ("u", "r"):
        whole = g.shape_view(name, 0)
        for s in slabs:
            _, _, olo, ohi = s.at(0)
            assert np.array_equal(ex[s.rank].owned(name), whole[olo:ohi]), (name, s.rank)
    if ci in FLIPPING:
        assert any(solver.colour_flip(s.rank, l) for s in slabs for l in range(levels))


def test_red_black_layout_without_x_alternation_is_refused():
    """P_y even (one Neumann, one Dirichlet face in y): the colour does not depend on i."""
    dims, levels, bc, rst = (65, 17, 17), 3, (1, 0, 1, 1, 0, 0), "fw"
    g, h = global_state(dims, levels, bc, rst, 7, "gs")
    slabs = decomp.plan_slabs(dims[0], levels, 2)
    ex = {s.rank: OracleSlab(s, g, bc, levels, h, rst, "gs") for s in slabs}
    with pytest.raises(ValueError):
        decomp.SlabSolver(slabs, decomp.LocalExchange(ex), levels, 1.0, maxiter=1, relaxation="gs",
                          west_halo=g.meta[0].halo["west"])


def test_global_west_halo_matches_the_one_domain_layout():
    import mgp

    for dims, levels, bc, rst, _, _, _, rlx in CASES:
        g, h = global_state(dims, levels, bc, rst, 0, rlx)
        got = decomp.global_west_halo(mgp, dims, levels, h, bc, RST[rst], RLX[rlx])
        assert got == g.meta[0].halo["west"], (dims, bc)


def test_red_black_needs_the_global_west_halo():
    slabs = decomp.plan_slabs(65, 3, 2)
    with pytest.raises(ValueError):
        decomp.SlabSolver(slabs, None, 3, 1.0, maxiter=1, relaxation="gs")


def _gloo_rank(rank, world, port, case, seed, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims, levels, bc, rst, cycle, ns, parts, rlx = case
        g, h = global_state(dims, levels, bc, rst, seed, rlx)
        slabs = decomp.plan_slabs(dims[0], levels, world)
        e = OracleSlab(slabs[rank], g, bc, levels, h, rst, rlx)
        solver = decomp.SlabSolver(slabs, decomp.DistExchange(e, rank, world), levels, g.default_omega(), maxiter=3,
                                   relaxation=rlx, west_halo=g.meta[0].halo["west"])
        rel, it, hist = solver.solve(cycle, ns)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), u=e.owned("u"), r=e.owned("r"), rel=rel, it=it,
                 hist=np.array(hist))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ci", [0, 2, 4, 6])
def test_slabs_as_two_gloo_ranks_match_global_solve(ci):
    case = CASES[ci][:6] + (2, CASES[ci][7])
    dims, levels, bc, rst, cycle, ns, _, rlx = case
    port = 29500 + (os.getpid() % 1000) + ci
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_rank, args=(2, port, case, 300 + ci, d), nprocs=2, join=True, start_method="spawn")
        res = [np.load(os.path.join(d, f"rank{r}.npz")) for r in range(2)]
        g, h = global_state(dims, levels, bc, rst, 300 + ci, rlx)
        rr, it_g, _, hist_g = g.solve(cycle, ns, g.default_omega(), 3, 1, 0.0)
        slabs = decomp.plan_slabs(dims[0], levels, 2)
        for r, s in enumerate(slabs):
            assert float(res[r]["rel"]) == rr and int(res[r]["it"]) == it_g
            assert list(res[r]["hist"])[1:] == list(hist_g)
            _, _, olo, ohi = s.at(0)
            for name in ("u", "r"):
                assert np.array_equal(res[r][name], g.shape_view(name, 0)[olo:ohi]), (name, r)


class _LayoutOnly:
    """Executor stand-in that only reports a slab's layout (its own oracle metadata)."""

    def __init__(self, o):
        self.o = o

    def layout(self, l):
        m = self.o.meta[l]
        return m.halo["west"], m.pad[1] * m.pad[2]


def test_colour_flip_is_the_padded_index_parity_difference():
    """For random geometries, every slab and level: the colour a slab sweeps differs from the
    one-domain colour exactly where the padded linear indices of the same point differ in
    parity (the reference's colour rule, include/gaussseidel.h:56,81)."""
    rng = np.random.default_rng(5)
    checked = 0
    for _ in range(40):
        levels = int(rng.integers(1, 5))
        H = 1 << (levels - 1)
        nx = H * int(rng.integers(4, 12)) + 1
        ny = (1 << (levels - 1)) * int(rng.integers(1, 4)) + 1
        nz = (1 << (levels - 1)) * int(rng.integers(1, 4)) + 1
        bc = tuple(int(x) for x in rng.integers(0, 2, size=6))
        parts = int(rng.integers(2, 5))
        try:
            slabs = decomp.plan_slabs(nx, levels, parts)
        except ValueError:
            continue
        h = 1.0 / (nx - 1)
        g = Oracle((nx, ny, nz), levels, h, bc, 1, 1, False)
        ex = {s.rank: _LayoutOnly(Oracle((s.nx, ny, nz), levels, h, decomp.slab_bc(s, bc), 1, 1, False))
              for s in slabs}

        class _Comm:
            def __init__(self, ex):
                self.ex = ex

            def ranks(self):
                return sorted(self.ex)

        solver = decomp.SlabSolver.__new__(decomp.SlabSolver)
        solver.slabs, solver.comm, solver.west_halo = slabs, _Comm(ex), g.meta[0].halo["west"]
        for s in slabs:
            for l in range(levels):
                gm, lm = g.meta[l], ex[s.rank].o.meta[l]
                lo = s.at(l)[0]
                for il in (0, 1, s.at(l)[1] - lo):  # a few planes of the slab
                    for j, k in ((0, 0), (1, 0), (0, 1), (gm.shape[1] - 1, gm.shape[2] - 1)):
                        def idx(m, i):
                            return (((i + m.halo["west"]) * m.pad[1] + j + m.halo["south"]) * m.pad[2] + k
                                    + m.halo["bottom"])

                        diff = (idx(gm, il + lo) - idx(lm, il)) & 1
                        assert diff == solver.colour_flip(s.rank, l), (nx, ny, nz, bc, levels, parts, s.rank, l)
                        checked += 1
    assert checked > 100

"""Domain decomposition of one solve along x: slabs of i-planes, one per GPU.

The reference divides its domain over devices with internal boundaries (include/ompboundary.h,
PoissonSolver(dev_shape, ...) in include/libpoisson.h); its exchanged values are relaxed copies
of the neighbour's planes, so its multi-device result is not the one-device result.  Here the
split is chosen so that the decomposed solve performs exactly the operations of the one-GPU
solve, point for point:

* Level l of rank r is an ordinary level hierarchy (a plain engine solver) over the global
  planes [a_r, b_r] / 2^l.  a_r and b_r are multiples of H = 2^(levels-1), so the coarse slabs
  are the fine slabs halved at every level.  Rank r owns the planes [s_r, s_{r+1}) (the last
  rank also s_{parts}); a_r = s_r - H and b_r = s_{r+1} + H around them (the global ends where
  there is no neighbour).
* The end planes a_r and b_r are Dirichlet faces of the local grid: never relaxed.  The other
  planes outside the owned range are computed by the local kernels from stale neighbours and
  then overwritten: after every operation that changes a field, the plane next to each side of
  the owned range is copied from the neighbour that owns it.  Every value an owned point reads
  is then the one-GPU value: sweeps and residuals read one plane across, FullWeighting reads
  fine plane 2I-1, and the prolongation reads coarse plane I+1.
* Norms run over owned planes only and combine as a max (an all-reduce MAX between processes).

Relaxation: weighted Jacobi (one sweep at a time, exchanged in between), or red-black
Gauss-Seidel as ordered half-sweeps of one colour each, exchanged in between (a point of one
colour reads only the other colour).  The colour of a point is the parity of the reference's
padded linear index in the ONE-domain layout (include/gaussseidel.h:56,81).  A slab's own
layout has the same padded y/z extents P_y, P_z but its own west halo w_s (0 at a cut, which is
Dirichlet) and starts at global plane lo, so its padded index differs from the global one by
(lo + w_g - w_s) * P_y * P_z: where that is odd, the slab sweeps the other local colour.  With
P_y * P_z even the colour does not depend on i at all (x-neighbours share a colour and the
one-domain sweep runs column by column in i order); such layouts are refused.

Exchange: ranks in one process copy planes directly; ranks in different processes send them
with torch.distributed point-to-point operations (NCCL between GPUs, gloo on the host).  Each
plane is one contiguous block (x is the slowest axis in both the engine's and the reference's
layout).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

WEST, EAST = 3, 2  # mgp_face order: north, south, east, west, top, bottom
DIRICHLET = 0


@dataclass
class Slab:
    rank: int
    parts: int
    lo: int      # first local plane a_r (global index, finest level)
    hi: int      # last local plane b_r
    own_lo: int  # first owned plane s_r
    own_hi: int  # one past the last owned plane

    def at(self, level: int):
        """(lo, hi, own_lo, own_hi) at `level`, global plane indices of that level."""
        d = 1 << level
        return self.lo // d, self.hi // d, self.own_lo // d, (self.own_hi - 1) // d + 1 if self.own_hi else 0

    def local(self, level: int, plane: int) -> int:
        return plane - self.lo // (1 << level)

    @property
    def nx(self) -> int:
        return self.hi - self.lo + 1


def plan_slabs(nx: int, levels: int, parts: int, weights=None) -> list:
    """Split planes 0..nx-1 into `parts` slabs (see the module comment).  Split points are
    multiples of H = 2^(levels-1), balanced by plane count (or by `weights`)."""
    H = 1 << (levels - 1)
    if levels < 1 or (nx - 1) % H:
        raise ValueError(f"nx={nx} is not coarsenable over {levels} levels")
    units = (nx - 1) // H
    if parts < 1 or parts > units:
        raise ValueError(f"{parts} slabs need at least {parts} coarse intervals; nx={nx} has {units}")
    w = np.ones(parts) if weights is None else np.asarray(weights, dtype=float)
    cum = np.concatenate([[0.0], np.cumsum(w) / np.sum(w)])
    cuts = [0]
    for r in range(1, parts):
        c = int(round(cum[r] * units))
        c = min(max(c, cuts[-1] + 1), units - (parts - r))
        cuts.append(c)
    cuts.append(units)
    s = [c * H for c in cuts]
    out = []
    for r in range(parts):
        own_lo = s[r]
        own_hi = s[r + 1] if r < parts - 1 else nx
        lo = 0 if r == 0 else s[r] - H
        hi = nx - 1 if r == parts - 1 else s[r + 1] + H
        out.append(Slab(r, parts, lo, hi, own_lo, own_hi))
    return out


def slab_bc(slab: Slab, bc_requested) -> tuple:
    """Requested face kinds of a slab's local grid: the global request, Dirichlet where a
    neighbour slab lies.  With the global strict flag the local grid resolves them as the
    global one does (the reference's resolution and halo widths go face by face), so every
    slab has the global layout in y and z."""
    bc = list(bc_requested)
    if slab.rank > 0:
        bc[WEST] = DIRICHLET
    if slab.rank < slab.parts - 1:
        bc[EAST] = DIRICHLET
    return tuple(bc)


# ---- exchanges ------------------------------------------------------------------------------
class LocalExchange:
    """All slabs in this process: planes are copied between executors directly."""

    def __init__(self, executors: dict):
        self.ex = executors  # rank -> executor

    def ranks(self):
        return sorted(self.ex)

    def exchange(self, slabs: list, field: str, level: int) -> None:
        for r in self.ranks():
            s = slabs[r]
            lo, hi, olo, ohi = s.at(level)
            if r > 0:  # my plane olo-1 <- left neighbour's owned plane olo-1
                left = slabs[r - 1]
                self.ex[r].set_plane(field, level, s.local(level, olo - 1),
                                     self.ex[r - 1].plane(field, level, left.local(level, olo - 1)))
            if r < s.parts - 1:  # my plane ohi <- right neighbour's owned plane ohi
                right = slabs[r + 1]
                self.ex[r].set_plane(field, level, s.local(level, ohi),
                                     self.ex[r + 1].plane(field, level, right.local(level, ohi)))

    def allreduce_max(self, values: dict) -> float:
        return max(values.values())


class DistExchange:
    """One slab per process, planes sent with torch.distributed (batched isend/irecv); every
    rank issues the same exchanges in the same order."""

    def __init__(self, executor, rank: int, world: int, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.ex = {rank: executor}
        self.rank, self.world, self.group = rank, world, group

    def ranks(self):
        return [self.rank]

    def exchange(self, slabs: list, field: str, level: int) -> None:
        dist = self.dist
        r = self.rank
        s = slabs[r]
        lo, hi, olo, ohi = s.at(level)
        ex = self.ex[r]
        ops, recvs = [], []
        if r > 0:
            ops.append(dist.P2POp(dist.isend, ex.plane_tensor(field, level, s.local(level, olo)), r - 1, self.group))
            buf = ex.empty_plane(field, level)
            ops.append(dist.P2POp(dist.irecv, buf, r - 1, self.group))
            recvs.append((s.local(level, olo - 1), buf))
        if r < self.world - 1:
            ops.append(dist.P2POp(dist.isend, ex.plane_tensor(field, level, s.local(level, ohi - 1)), r + 1,
                                  self.group))
            buf = ex.empty_plane(field, level)
            ops.append(dist.P2POp(dist.irecv, buf, r + 1, self.group))
            recvs.append((s.local(level, ohi), buf))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for plane, buf in recvs:
            ex.set_plane(field, level, plane, buf)

    def allreduce_max(self, values: dict) -> float:
        import torch

        t = torch.tensor([values[self.rank]], dtype=torch.float64, device=self.ex[self.rank].comm_device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(t.item())


# ---- the decomposed solve -------------------------------------------------------------------
class SlabSolver:
    """The reference's solve loop and V/F-cycles (include/libpoisson.h:237-357,
    include/vcycle.h:14-98, include/fcycle.h:13-97) over slabs, one operation at a time with the
    halo exchanges between them.  Executors provide the level operations of one slab (relax,
    relax_colour, residual, restrict, restrict_bc, zero_u, prolong_add, the max-norm over owned
    planes), plane access and, for red-black smoothing, layout(level) = (west halo, P_y * P_z)
    of their own padded layout.

    relaxation: "jacobi" or "gs"; west_halo: the west halo width of the one-domain layout
    (global_west_halo), which fixes the red-black colours."""

    def __init__(self, slabs: list, comm, levels: int, omega: float, maxiter: int, miniter: int = 1, tol: float = 0.0,
                 relaxation: str = "jacobi", west_halo: int | None = None):
        self.slabs, self.comm, self.levels = slabs, comm, levels
        self.omega, self.maxiter, self.miniter, self.tol = omega, maxiter, miniter, tol
        self.gs = relaxation.lower() in ("gs", "gaussseidel", "gauss-seidel")
        if self.gs and west_halo is None:
            raise ValueError("red-black smoothing needs the one-domain west halo width (global_west_halo)")
        self.west_halo = west_halo
        self.alternate = True  # GaussSeidel::alternate (include/gaussseidel.h:18): colour 0 first
        if self.gs:
            # with P_y * P_z even the colour does not depend on i: x-neighbours share a colour, the
            # one-domain half-sweep runs in i order (column-ordered) and does not split into slabs
            for r in comm.ranks():
                for l in range(levels):
                    if comm.ex[r].layout(l)[1] % 2 == 0:
                        raise ValueError("red-black layout with an even padded y*z extent: the colours do not "
                                         "alternate along x, so the sweep cannot be split into x-slabs")

    def colour_flip(self, rank: int, l: int) -> int:
        """1 where the slab's padded index parity differs from the one-domain layout's."""
        lo = self.slabs[rank].at(l)[0]
        w_s, pyz = self.comm.ex[rank].layout(l)
        return ((lo + self.west_halo - w_s) * pyz) & 1

    # level operations on every local slab, each followed by the exchange it needs
    def _each(self, fn):
        for r in self.comm.ranks():
            fn(self.comm.ex[r])

    def relax(self, l: int, ns: int) -> None:
        if not self.gs:
            for _ in range(ns):  # Jacobi: one sweep at a time, exchanged in between
                self._each(lambda e: e.relax(l, self.omega, 1))
                self.comm.exchange(self.slabs, "u", l)
            return
        for _ in range(2 * ns):  # red-black: one colour at a time (relaxation.h:19-94)
            colour = 0 if self.alternate else 1
            for r in self.comm.ranks():
                self.comm.ex[r].relax_colour(l, self.omega, colour ^ self.colour_flip(r, l))
            self.comm.exchange(self.slabs, "u", l)
            self.alternate = not self.alternate

    def setup(self, l: int) -> None:
        self._each(lambda e: e.residual(l))
        self.comm.exchange(self.slabs, "r", l)
        self._each(lambda e: e.restrict_bc(l))
        self._each(lambda e: e.restrict(l))
        self._each(lambda e: e.zero_u(l + 1))

    def prolong(self, l: int) -> None:
        self._each(lambda e: e.prolong_add(l))
        self.comm.exchange(self.slabs, "u", l)

    def vcycle(self, l: int, ns: int) -> None:
        self.relax(l, ns)
        if l >= self.levels - 1:
            return
        self.setup(l)
        self.vcycle(l + 1, ns)
        self.prolong(l)
        self.relax(l, ns)

    def fcycle(self, l: int, ns: int) -> None:
        self.relax(l, ns)
        self.setup(l)
        if l < self.levels - 2:
            self.fcycle(l + 1, ns)
        self.vcycle(l + 1, ns)
        self.prolong(l)
        if l == 0:
            self.vcycle(0, ns)

    def norm(self, field: str) -> float:
        vals = {r: self.comm.ex[r].owned_norm(field, self.slabs[r]) for r in self.comm.ranks()}
        return self.comm.allreduce_max(vals)

    def residual_norm(self) -> float:
        self._each(lambda e: e.residual(0))
        self.comm.exchange(self.slabs, "r", 0)
        return self.norm("r")

    def solve(self, cycle: str, ns: int):
        """Returns (relative residual, reported iterations, history), as the reference's loop
        computes them (the stop rule of include/libpoisson.h:306-355)."""
        fnorm = self.norm("f")
        rel = self.residual_norm() / fnorm
        hist = [rel]
        it = 0
        for it in range(self.maxiter):
            (self.vcycle if cycle.lower() == "vcycle" else self.fcycle)(0, ns)
            norm = self.residual_norm() / fnorm
            hist.append(norm)
            if it >= self.miniter:
                if norm > 2.0 * rel:
                    rel = norm
                    break
                if abs(norm - rel) < self.tol:
                    rel = norm
                    break
            rel = norm
        else:
            it = self.maxiter
        return rel, it, hist


def global_west_halo(mgp, dims, levels, h, bc_requested, restriction, relaxation, strict_bc=False) -> int:
    """West halo width of the one-domain layout (the reference's Domain halo for the resolved
    west face kind), planned from the descriptor alone (mgp_plan_level, no device needed)."""
    import ctypes

    d = mgp.make_desc(dims, levels, h, bc_requested, restriction, relaxation, mgp.F64, 1, 1, 0.0, (0.0, 0.0, 0.0), 0,
                      strict_bc, 0)
    li = mgp.LevelInfo()
    mgp._check(mgp.lib().mgp_plan_level(ctypes.byref(d), 0, ctypes.byref(li)))
    return int(li.halo[1])  # halo order: east, west, north, south, top, bottom


# ---- the engine executor (one CUDA solver per slab) ----------------------------------------
class EngineSlab:
    """One slab on one GPU: a plain engine solver over the slab's planes (the global requested
    boundary kinds and strict flag, Dirichlet at the cuts), driven one level operation at a
    time."""

    def __init__(self, mgp, slab: Slab, dims, levels, h, bc_requested, restriction, strict_bc=False, device=0,
                 relaxation=None):
        import torch

        self.mgp, self.slab, self.torch = mgp, slab, torch
        rlx = mgp.JACOBI if relaxation is None else relaxation
        self.solver = mgp.Solver((slab.nx, dims[1], dims[2]), levels, h, slab_bc(slab, bc_requested), restriction,
                                 rlx, mgp.F64, 1, 1, 0.0, device=device, strict_bc=strict_bc)
        self.comm_device = torch.device("cuda", device)

    def layout(self, l):
        lv = self.solver.level[l]
        return lv.halo["west"], lv.pad[1] * lv.pad[2]

    def relax_colour(self, l, omega, colour):
        self.solver.relax_colour(l, omega, colour)

    def _planes(self, field: str, level: int):
        """The field's buffer as (nx, plane pitch) -- looked up each time: Jacobi sweeps swap
        the u pair."""
        v = self.solver.device_field(field, level)
        sx = v.strides[0] // 8
        flat = self.mgp.DeviceView(v.ptr, (v.shape[0], sx), (sx * 8, 8), np.float64, self.solver)
        return self.torch.as_tensor(flat, device=self.comm_device), v

    def plane(self, field, level, i):
        self.solver.synchronize()
        return self._planes(field, level)[0][i]

    plane_tensor = plane

    def empty_plane(self, field, level):
        return self.torch.empty_like(self._planes(field, level)[0][0])

    def set_plane(self, field, level, i, values):
        self.solver.synchronize()
        self._planes(field, level)[0][i].copy_(values)
        self.torch.cuda.synchronize(self.comm_device)

    def relax(self, l, omega, ns):
        self.solver.relax(l, omega, ns)

    def residual(self, l):
        self.solver.residual(l)

    def restrict(self, l):
        self.solver.restrict(l)

    def restrict_bc(self, l):
        self.solver.restrict_bc(l)

    def zero_u(self, l):
        self.solver.zero_u(l)

    def prolong_add(self, l):
        self.solver.prolong_add(l)

    def owned_norm(self, field, slab: Slab) -> float:
        self.solver.synchronize()
        t, v = self._planes(field, 0)
        _, _, olo, ohi = slab.at(0)
        a, b = slab.local(0, olo), slab.local(0, ohi)
        if b <= a:
            return 0.0
        sy = v.strides[1] // 8
        rows = t[a:b, : v.shape[1] * sy].reshape(b - a, v.shape[1], sy)[:, :, : v.shape[2]]
        return float(rows.abs().max().item())

    def close(self):
        self.solver.close()

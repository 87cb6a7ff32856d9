"""One single-level case split across ranks: slabs of the slowest direction, ghost-plane exchange per RK
stage, one maximum reduction of the wave speed per step.

This is the distributed form of the reference's single-level advance (ThirdOrderSSPRK with FillPatch,
source/Class_Compressible_PhaseField.cpp:3937-4107; the ghost exchange that AMReX's FillBoundary does
inside FillPatch, source/COMPAS.cpp:1645-1732; ComputeDt's ReduceRealMin over the ranks,
source/COMPAS.cpp:2249-2303). The box is cut along its slowest direction (z in 3D, y in 2D) into one slab
per rank. In the SoA layout of a padded box every component's run of consecutive planes is one
contiguous block, so a rank sends its NGROW boundary planes of each component as they lie (no packing)
and receives its neighbours' planes straight into its ghost planes. A plane travels whole, with the
sender's ghost cells of the faster directions filled by the sender's own boundary fill, which gives
them the values a single-box fill gives.

Per RK stage each slab fills its physical ghosts (compas_b200_fill_boundary on the slab's geometry; at
the cut faces the fill writes only the slab's ghost planes, which the exchange overwrites), the planes across every cut
face (and across the periodic wrap of the cut direction) are exchanged, and the fused stage kernel runs
on the slab (compas_b200_rk3_stage), accumulating the slab's wave-speed maximum. Per step the ranks take
the maximum of those maxima (exact in any order) and compute the step size on the host with the
level's own expression (cfl dx / c_max, the 1.1x change limiter, the stop-time clamp), so every rank
takes the same step and the result is the single-box level's, bit for bit: each cell's stage
arithmetic sees the same stencil values.

The ranks talk through a communicator object: DistComm (torch.distributed point-to-point and
all-reduce: NCCL between GPUs, gloo between CPU processes) or LocalComm (all slabs in one process,
planes copied between them, for a single GPU). The per-slab work goes through a backend object; the
default, DeviceBackend, is the CUDA library's C ABI on torch CUDA tensors.
"""
from __future__ import annotations

import numpy as np

DBL_MAX = float(np.finfo(np.float64).max)


def split(n: int, world: int) -> list:
    """(start, count) of each rank's slab of n cells: counts differ by at most one, the larger first."""
    if world < 1 or n < world:
        raise ValueError(f"cannot split {n} cells among {world} ranks")
    base, extra = divmod(n, world)
    out, s = [], 0
    for r in range(world):
        c = base + (1 if r < extra else 0)
        out.append((s, c))
        s += c
    return out


def _dmin(a: float, b: float) -> float:
    return b if b < a else a


def next_dt(t: float, dt_prev: float, cmax: float, stop_time: float, cfl: float, dx, dim: int, limiter: bool):
    """The step size of the level advance from the previous step's wave-speed maximum (ComputeDt,
    source/COMPAS.cpp:2249-2303, as the level's device step control computes it): (dt, dt_prev after
    the step), or (None, why) when the run stops (stop time reached, or a step size that is not positive
    and finite)."""
    if not (t < stop_time):
        return None, "stop"
    with np.errstate(divide="ignore", invalid="ignore"):
        dt_est = DBL_MAX
        c = np.float64(cmax)
        for d in range(dim):
            dt_est = _dmin(dt_est, float(np.float64(cfl) * np.float64(dx[d]) / c))
    if t == 0.0:
        dt_prev = dt_est
    if limiter and dt_prev > 0.0:
        dt_est = _dmin(dt_est, 1.1 * dt_prev)
    dt0 = dt_est
    eps = 1.0e-3 * dt0
    if t + dt0 > stop_time - eps:
        dt0 = stop_time - t
    if not (dt0 > 0.0) or not (dt0 <= DBL_MAX):
        return None, "cfl"
    return dt0, dt0


class Slab:
    """Rank `rank`'s slab of the global box: its geometry and its place along the cut direction."""

    def __init__(self, p, g, rank: int, world: int):
        from . import make_geom

        self.dim = int(p.dim)
        self.cut = self.dim - 1  # slowest direction
        self.ng = int(g.ng)
        n = [int(g.n[d]) for d in range(3)]
        self.start, self.count = split(n[self.cut], world)[rank]
        if self.count < self.ng:
            raise ValueError(f"a slab needs at least {self.ng} cells along the cut direction, rank {rank} "
                             f"would get {self.count}")
        self.rank, self.world = rank, world
        self.periodic = (int(g.lo_bc[self.cut]) == 0)
        lo = [int(g.lo_bc[d]) for d in range(3)]
        hi = [int(g.hi_bc[d]) for d in range(3)]
        # cut faces: the slab's own fill writes only its ghost planes there, which the exchange then
        # overwrites; they keep the periodic code of a periodic direction (both faces are cut then) and
        # take the outflow code otherwise (a periodic code needs both faces)
        if world > 1:
            cut_code = 0 if self.periodic else 2
            if rank > 0 or self.periodic:
                lo[self.cut] = cut_code
            if rank < world - 1 or self.periodic:
                hi[self.cut] = cut_code
        n[self.cut] = self.count
        self.geom = make_geom(n[:self.dim] + [1] * (3 - self.dim), [float(g.dx[d]) for d in range(3)], self.ng,
                              lo, hi)
        self.lo_peer = rank - 1 if rank > 0 else (world - 1 if self.periodic and world > 1 else None)
        self.hi_peer = rank + 1 if rank < world - 1 else (0 if self.periodic and world > 1 else None)
        # the cut direction's axis of a padded array viewed as (N, PZ, PY, PX)
        self.axis = 1 if self.dim == 3 else 2

    def planes(self, a, first: int, count: int) -> list:
        """Per component, the contiguous block of `count` padded planes of the cut direction starting at
        padded index `first` (views of a, which has the padded shape (N, PZ, PY, PX))."""
        if self.axis == 1:
            return [a[c, first:first + count] for c in range(a.shape[0])]
        return [a[c, 0, first:first + count] for c in range(a.shape[0])]

    def send_low(self, a):   # the first NGROW valid planes, for the lower neighbour's high ghosts
        return self.planes(a, self.ng, self.ng)

    def send_high(self, a):  # the last NGROW valid planes, for the upper neighbour's low ghosts
        return self.planes(a, self.count, self.ng)

    def ghost_low(self, a):
        return self.planes(a, 0, self.ng)

    def ghost_high(self, a):
        return self.planes(a, self.ng + self.count, self.ng)

    def global_slice(self, g):
        """Index of this slab's valid cells in the global valid array (N, nz, ny, nx)."""
        s = slice(self.start, self.start + self.count)
        return (slice(None), s) if self.dim == 3 else (slice(None), slice(None), s)


class LocalComm:
    """All slabs in one process (one GPU): planes are copied between the slabs' arrays; the maximum is
    taken over the slabs."""

    def __init__(self, world: int):
        self.world = world
        self.ranks = list(range(world))

    def exchange(self, slabs, arrays) -> None:
        # upward (each slab's high valid planes into its upper neighbour's low ghosts), then downward
        for s, a in zip(slabs, arrays):
            if s.hi_peer is not None:
                for dst, src in zip(slabs[s.hi_peer].ghost_low(arrays[s.hi_peer]), s.send_high(a)):
                    dst.copy_(src)
        for s, a in zip(slabs, arrays):
            if s.lo_peer is not None:
                for dst, src in zip(slabs[s.lo_peer].ghost_high(arrays[s.lo_peer]), s.send_low(a)):
                    dst.copy_(src)

    def max(self, values) -> float:
        return max(float(v) for v in values)


class DistComm:
    """One slab per process over torch.distributed: point-to-point plane transfers (NCCL between GPUs,
    gloo on CPU) and an all-reduce for the maximum. Every rank posts its transfers in the same order
    (upward, then downward; components in order), so the messages between any two ranks match even
    when they are each other's lower and upper neighbour (two ranks on a periodic cut)."""

    def __init__(self, dist, device="cpu"):
        self.dist = dist
        self.world = dist.get_world_size()
        self.ranks = [dist.get_rank()]
        self.device = device

    def exchange(self, slabs, arrays) -> None:
        dist = self.dist
        (s,), (a,) = slabs, arrays
        for phase in ("up", "down"):
            ops = []
            if phase == "up":
                if s.hi_peer is not None:
                    ops += [dist.P2POp(dist.isend, t, s.hi_peer) for t in s.send_high(a)]
                if s.lo_peer is not None:
                    ops += [dist.P2POp(dist.irecv, t, s.lo_peer) for t in s.ghost_low(a)]
            else:
                if s.lo_peer is not None:
                    ops += [dist.P2POp(dist.isend, t, s.lo_peer) for t in s.send_low(a)]
                if s.hi_peer is not None:
                    ops += [dist.P2POp(dist.irecv, t, s.hi_peer) for t in s.ghost_high(a)]
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()

    def max(self, values) -> float:
        import torch

        (v,) = values
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


class DeviceBackend:
    """The per-slab work on the GPU through the C ABI (torch CUDA tensors, the current stream)."""

    def __init__(self, p):
        import torch

        self.p = p
        self.torch = torch

    def alloc(self, shape):
        return self.torch.zeros(shape, dtype=self.torch.float64, device="cuda")

    def scalar(self):
        return self.torch.zeros(1, dtype=self.torch.float64, device="cuda")

    def fill(self, g, U) -> None:
        from . import FillPatch

        FillPatch(self.p, g, U)

    def cmax_pass(self, g, U, cm, scratch) -> None:
        from . import compute_dUdt_FV

        compute_dUdt_FV(self.p, g, U, scratch, cmax=cm, err=self.err)

    def stage(self, g, s: int, Us, Uold, Unew, dt_dev, cm) -> None:
        from . import ThirdOrderSSPRK_stage

        ThirdOrderSSPRK_stage(self.p, g, s, Us, Uold, Unew, dt_dev, cmax=cm, err=self.err)

    def set_scalar(self, x, v: float) -> None:
        x.fill_(float(v))

    def read(self, x) -> float:
        return float(x.item())

    def status(self) -> int:
        return int(self.err.item())

    def new_status(self):
        self.err = self.torch.zeros(1, dtype=self.torch.int32, device="cuda")


class ShardedLevel:
    """A single-level case advanced by `comm.world` ranks, each holding the slabs `comm.ranks`.

    upload(U) takes the global padded state (host numpy or any array indexable like it) and keeps the
    local slabs; advance(nsteps) runs whole TVD-RK3 steps; download() returns the local slabs' valid
    cells with their global index ranges."""

    def __init__(self, p, g, comm, backend=None):
        from . import padded_shape

        if int(p.phase_field) or int(p.id_bound):
            raise ValueError("the sharded level runs the hyperbolic step (no Phase-Field step, no ID_Bound = 1)")
        self.p, self.g, self.comm = p, g, comm
        self.backend = backend if backend is not None else DeviceBackend(p)
        self.slabs = [Slab(p, g, r, comm.world) for r in comm.ranks]
        b = self.backend
        self.U, self.U1, self.U2, self.cm, self.scratch = [], [], [], [], []
        for s in self.slabs:
            shape = padded_shape(p, s.geom)
            self.U.append(b.alloc(shape))
            self.U1.append(b.alloc(shape))
            self.U2.append(b.alloc(shape))
            self.scratch.append(b.alloc(shape))
            self.cm.append(b.scalar())
        self.dt_dev = b.scalar()
        self.t, self.dt_prev, self.steps, self.cmax = 0.0, 1.0e100, 0, 0.0
        self.dts = []
        self.stopped = None
        b.new_status()

    def _fill(self, arrays) -> None:
        for s, a in zip(self.slabs, arrays):
            self.backend.fill(s.geom, a)
        self.comm.exchange(self.slabs, arrays)

    def upload(self, U, t0: float = 0.0) -> None:
        """Local slabs of the global padded state U (host numpy or a torch tensor; its valid cells, ghosts
        are filled here), then the
        initial wave-speed maximum (CalculateInitialcmax, source/Class_Compressible_PhaseField.cpp:4501-4605)."""
        import torch

        from . import valid_view

        for s, a in zip(self.slabs, self.U):
            src = valid_view(U, self.p, self.g)[s.global_slice(self.g)]
            if isinstance(src, np.ndarray):
                src = torch.from_numpy(np.ascontiguousarray(src))
            valid_view(a, self.p, s.geom).copy_(src)
        self.t, self.dt_prev, self.steps, self.dts, self.stopped = float(t0), 1.0e100, 0, [], None
        self._fill(self.U)
        for s, a, c, w in zip(self.slabs, self.U, self.cm, self.scratch):
            self.backend.set_scalar(c, 0.0)
            self.backend.cmax_pass(s.geom, a, c, w)
        self.cmax = self.comm.max([self.backend.read(c) for c in self.cm])

    def advance(self, nsteps: int, stop_time: float = 1.0e300) -> int:
        """Up to nsteps steps (fewer at the stop time); returns the number taken."""
        p, b = self.p, self.backend
        dx = [float(self.g.dx[d]) for d in range(3)]
        taken = 0
        for _ in range(nsteps):
            dt, nxt = next_dt(self.t, self.dt_prev, self.cmax, stop_time, float(p.cfl), dx, int(p.dim),
                              bool(p.change_limiter))
            if dt is None:
                self.stopped = nxt
                break
            self.dt_prev = nxt
            b.set_scalar(self.dt_dev, dt)
            for c in self.cm:
                b.set_scalar(c, 0.0)
            ins, outs = (self.U, self.U1, self.U2), (self.U1, self.U2, self.U)
            for st in range(3):
                self._fill(ins[st])
                for i, s in enumerate(self.slabs):
                    b.stage(s.geom, st, ins[st][i], self.U[i], outs[st][i], self.dt_dev, self.cm[i])
            self.cmax = self.comm.max([b.read(c) for c in self.cm])
            self.t += dt
            self.steps += 1
            self.dts.append(dt)
            taken += 1
        return taken

    def status(self) -> int:
        return self.backend.status()

    def download(self) -> list:
        """[(global valid-cell index, valid cells of the slab)] of the local slabs."""
        from . import valid_view

        return [(s.global_slice(self.g), valid_view(a, self.p, s.geom)) for s, a in zip(self.slabs, self.U)]

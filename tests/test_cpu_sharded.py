"""The sharded single-level advance (compas_b200.sharded) on CPU: slab split, step-size control, ghost-plane
exchange and the stage sequence, with the per-slab work done by the CPU oracle (a test backend) so that
the decomposition can be checked without a GPU. The slabs together must give the single-box oracle's
advance to the bit (state and every step size): in one process (LocalComm, 1-3 slabs; a periodic cut
direction exchanges across the wrap) and as two gloo processes (DistComm, the transport bench.py's
NCCL ranks use)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import compas_b200 as cb
from compas_b200 import cases, sharded
from oracle.oracle import Oracle
from tests.helpers import oracle_kind


class OracleBackend:
    """Per-slab work through the oracle on torch CPU tensors: the boundary fill, the right-hand side with
    its wave-speed maximum, the stage combination as the fused stage kernel forms it, and the SIXEQS
    pressure relaxation after every stage."""

    def __init__(self, p, kind):
        self.p, self.kind, self._o = p, kind, {}
        self.relax = (int(p.physics) == cb.SIXEQS and int(p.relaxation) != 0)

    def _oracle(self, g):
        key = (tuple(g.n), tuple(g.lo_bc), tuple(g.hi_bc))
        if key not in self._o:
            self._o[key] = Oracle(self.kind, self.p, g)
        return self._o[key]

    def alloc(self, shape):
        return torch.zeros(shape, dtype=torch.float64)

    def scalar(self):
        return torch.zeros(1, dtype=torch.float64)

    def fill(self, g, U):
        self._oracle(g).fill_ghosts(U.numpy())

    def cmax_pass(self, g, U, cm, scratch):
        _, c = self._oracle(g).compute_dudt(U.numpy())
        cm[0] = max(float(cm[0]), c)

    def stage(self, g, s, Us, Uold, Unew, dt_dev, cm):
        o = self._oracle(g)
        L, c = o.compute_dudt(Us.numpy())
        cm[0] = max(float(cm[0]), c)
        dt = float(dt_dev[0])
        ca, cb_, cd = [(1.0, 0.0, 1.0), (0.25, 0.75, 0.25), (2.0 / 3.0, 1.0 / 3.0, 2.0 / 3.0)][s]
        us, u0 = Us.numpy(), Uold.numpy()
        v = 1.0 * us if s == 0 else ca * us + cb_ * u0
        out = v + (cd * dt) * L
        vv = cb.valid_view(out, self.p, g)
        cb.valid_view(Unew.numpy(), self.p, g)[...] = vv
        if self.relax:
            o.relax(Unew.numpy())

    def set_scalar(self, x, v):
        x[0] = float(v)

    def read(self, x):
        return float(x[0])

    def status(self):
        return 0

    def new_status(self):
        pass


def _assemble(p, g, parts):
    out = np.zeros(cb.valid_view(np.zeros(cb.padded_shape(p, g)), p, g).shape)
    for idx, v in parts:
        out[idx] = np.asarray(v)
    return out


def _disc():
    phys, dim, inputs, geom, U = cases.advected_disc(n=24)
    return cb.make_parm(phys, dim, inputs), cb.make_geom(**geom), U


def _droplet():
    phys, dim, inputs, geom, U = cases.shock_droplet(n=12)
    return cb.make_parm(phys, dim, inputs), cb.make_geom(**geom), U


def test_split_and_slab_geometry():
    assert sharded.split(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert sharded.split(9, 3) == [(0, 3), (3, 3), (6, 3)]
    with pytest.raises(ValueError):
        sharded.split(2, 3)
    p, g, _ = _droplet()
    s0, s1 = sharded.Slab(p, g, 0, 2), sharded.Slab(p, g, 1, 2)
    assert (s0.start, s0.count, s1.start, s1.count) == (0, 6, 6, 6)
    # outflow cut direction: the physical faces keep their code, the cut faces (exchanged) take the
    # outflow code, which the boundary fill accepts on one side alone
    assert (s0.geom.lo_bc[2], s0.geom.hi_bc[2], s1.geom.lo_bc[2], s1.geom.hi_bc[2]) == (2, 2, 2, 2)
    assert (s0.lo_peer, s0.hi_peer, s1.lo_peer, s1.hi_peer) == (None, 1, 0, None)
    with pytest.raises(ValueError):
        sharded.Slab(p, g, 4, 5)  # 12 / 5 -> the last slabs have 2 cells < NGROW 3
    pd, gd, _ = _disc()
    r0, r1 = sharded.Slab(pd, gd, 0, 2), sharded.Slab(pd, gd, 1, 2)
    assert (r0.lo_peer, r0.hi_peer, r1.lo_peer, r1.hi_peer) == (1, 1, 0, 0)  # periodic: a ring
    assert (r0.geom.lo_bc[1], r0.geom.hi_bc[1]) == (0, 0)
    # a slab's geometry passes the library's boundary-code check (no GPU needed for it)
    for s in (s0, s1, r0, r1):
        lo = [s.geom.lo_bc[d] for d in range(s.dim)]
        hi = [s.geom.hi_bc[d] for d in range(s.dim)]
        assert all((a == 0) == (b == 0) for a, b in zip(lo, hi))


def test_next_dt_matches_level_rules():
    dx = [0.1, 0.05, 1.0]
    dt, prev = sharded.next_dt(0.0, 1e100, 2.0, 1e300, 0.5, dx, 2, True)
    assert dt == 0.5 * 0.05 / 2.0 and prev == dt
    # the change limiter: at most 1.1x the previous step
    dt2, _ = sharded.next_dt(1.0, 0.001, 1e-9, 1e300, 0.5, dx, 2, True)
    assert dt2 == 1.1 * 0.001
    # the stop-time clamp within 1e-3 dt of the stop time
    dt3, _ = sharded.next_dt(1.0, 1.0, 2.0, 1.0 + 0.5 * 0.05 / 2.0 * 0.9995, 0.5, dx, 2, True)
    assert dt3 == (1.0 + 0.5 * 0.05 / 2.0 * 0.9995) - 1.0
    assert sharded.next_dt(2.0, 1.0, 2.0, 1.0, 0.5, dx, 2, True) == (None, "stop")
    # no wave speed: the step runs to the stop time, as the level's device step control does
    assert sharded.next_dt(0.0, 1e100, 0.0, 1e300, 0.5, dx, 2, True) == (1e300, 1e300)
    assert sharded.next_dt(0.0, 1e100, -1.0, 1e300, 0.5, dx, 2, True) == (None, "cfl")


@pytest.mark.parametrize("case,world,steps", [(_disc, 1, 4), (_disc, 2, 4), (_disc, 3, 4),
                                               (_droplet, 2, 3), (_droplet, 3, 3)])
def test_local_slabs_match_single_box_oracle(case, world, steps):
    p, g, U = case()
    kind = oracle_kind(int(p.physics), int(p.dim))
    ref = np.ascontiguousarray(U.copy())
    t_ref, dts_ref = Oracle(kind, p, g).advance(ref, steps)
    lv = sharded.ShardedLevel(p, g, sharded.LocalComm(world), OracleBackend(p, kind))
    lv.upload(U)
    assert lv.advance(steps) == steps
    got = _assemble(p, g, lv.download())
    np.testing.assert_array_equal(np.array(lv.dts), dts_ref)
    assert lv.t == t_ref
    np.testing.assert_array_equal(got, cb.valid_view(ref, p, g))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, case_name, steps, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p, g, U = {"disc": _disc, "droplet": _droplet}[case_name]()
        kind = oracle_kind(int(p.physics), int(p.dim))
        lv = sharded.ShardedLevel(p, g, sharded.DistComm(dist), OracleBackend(p, kind))
        lv.upload(U)
        lv.advance(steps)
        (idx, v), = lv.download()
        out.put((rank, idx, np.array(v), list(lv.dts)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case_name,steps", [("disc", 3), ("droplet", 2)])
def test_two_gloo_ranks_match_single_box_oracle(case_name, steps):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, case_name, steps, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted((out.get(timeout=180) for _ in range(world)), key=lambda x: x[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p, g, U = {"disc": _disc, "droplet": _droplet}[case_name]()
    ref = np.ascontiguousarray(U.copy())
    _, dts_ref = Oracle(oracle_kind(int(p.physics), int(p.dim)), p, g).advance(ref, steps)
    got = _assemble(p, g, [(idx, v) for _, idx, v, _ in res])
    for _, _, _, dts in res:
        np.testing.assert_array_equal(np.array(dts), dts_ref)
    np.testing.assert_array_equal(got, cb.valid_view(ref, p, g))

"""Continuous-batching request loop for shock-interface solves.

Requests arrive over time (Poisson arrivals), each a case of some type, size and step count. The loop
keeps every admitted case resident in HBM inside a per-model `Batch` (one persistent launch per RK
stage advances all of a model's cases together), admits waiting requests as soon as their memory fits
the budget - while others are running - and retires cases when their step count is reached. It
reports time-to-solution (arrival to completion) percentiles and the aggregate cell-update rate, and
can replay the same requests one at a time on a single-case level for comparison.

Request types:
  bubble2d   2D FIVEEQS shock-bubble (WENO5B), side^2 cells
  droplet3d  3D SIXEQS shock-droplet (WENO5B, relaxation), side^3 cells: the bounded scheme, because
             with WENO5 the droplet's volume fraction leaves [0, 1] and the run stops on a NaN after
             about 700 steps at 112^3 in both precision forms, inside the requests' 100-2000 steps
  triple2d   2D FIVEEQS_NPHASE (NPHASE = 3) triple point on [0,7] x [0,3] (WENO5), 7 side x 3 side cells
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import FIVEEQS, FIVEEQS_NPHASE, SIXEQS, Batch, Level, make_geom, make_parm, padded_shape, valid_view
from . import cases as _cases

# kind: (physics, dim, FiniteVolume.Scheme id, NPHASE)
KINDS = {"bubble2d": (FIVEEQS, 2, 6, 2), "droplet3d": (SIXEQS, 3, 6, 2), "triple2d": (FIVEEQS_NPHASE, 2, 5, 3)}


@dataclass
class Request:
    rid: int
    kind: str
    side: int
    steps: int
    arrival: float
    params: dict = field(default_factory=dict)
    admitted: float = -1.0
    finished: float = -1.0
    case_id: int = -1
    cells: int = 0
    bytes: int = 0
    result: object = None


def make_case(req: Request, precision: str, device="cuda", xp=None):
    """(parm, geom, initial padded state on the device) of a request."""
    import torch

    xp = torch if xp is None else xp
    if req.kind == "bubble2d":
        phys, dim, inputs, geom, U = _cases.shock_bubble(nx=req.side, ny=req.side, length=1.0,
                                                         center=(0.55, 0.5), radius=0.2,
                                                         Ma=req.params.get("Ma", 1.5),
                                                         rho_b=req.params.get("ratio", 0.138),
                                                         xp=xp, device=device)
    elif req.kind == "triple2d":
        phys, dim, inputs, geom, U = _cases.triple_point(m=req.side, xp=xp, device=device)
    else:
        phys, dim, inputs, geom, U = _cases.shock_droplet(n=req.side, xp=xp, device=device)
        inputs = dict(inputs, **{"FiniteVolume.Scheme": "WENO5B"})
    inputs = dict(inputs, **{"compas_b200.precision": precision})
    return make_parm(phys, dim, inputs), make_geom(**geom), U


def poisson_requests(n, rate, seed=0, kinds=("bubble2d", "droplet3d", "triple2d"), sides2d=(128, 1024),
                     sides3d=(64, 192), sides_triple=(32, 128), steps=(100, 2000)):
    """n requests with exponential inter-arrival times of mean 1/rate (seeded). The side of a request
    is a multiple of 16 in the kind's range (the triple point's side m gives 7m x 3m cells)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        kind = kinds[int(rng.integers(len(kinds)))]
        lo, hi = {"bubble2d": sides2d, "droplet3d": sides3d, "triple2d": sides_triple}[kind]
        side = int(rng.integers(lo // 16, hi // 16 + 1)) * 16
        st = int(rng.integers(steps[0], steps[1] + 1))
        params = {"Ma": float(rng.uniform(1.1, 3.0)), "ratio": float(np.exp(rng.uniform(np.log(0.01), np.log(1000))))}
        out.append(Request(i, kind, side, st, t, params))
    return out


def _cells(req):
    if req.kind == "triple2d":
        return 21 * req.side * req.side
    return req.side ** (2 if req.kind == "bubble2d" else 3)


class Server:
    """Admission against a byte budget, continuous batching, retirement at the step count."""

    def __init__(self, budget_bytes: float = 150e9, precision: str = "mixed", capacity: int = 4096,
                 steps_per_iter: int = 1, keep_results: bool = False):
        self.budget = float(budget_bytes)
        self.precision = precision
        prec = 1 if precision == "mixed" else 0
        self.batches = {k: Batch(ph, d, id_limiter=lim, precision=prec, capacity=capacity, nphase=nph)
                        for k, (ph, d, lim, nph) in KINDS.items()}
        self.steps_per_iter = steps_per_iter
        self.keep_results = keep_results
        self.in_use = 0

    def close(self):
        for b in self.batches.values():
            b.close()

    def prepare(self, requests):
        """Build every request's initial state on the device ahead of time (kept on the request), so
        that run() measures admission, the solves and retirement, not the initial-condition
        construction."""
        for r in requests:
            if getattr(r, "_case", None) is None:
                r._case = make_case(r, self.precision)

    def run(self, requests, clock=None):
        import torch

        clock = clock or time.perf_counter
        pending = sorted(requests, key=lambda r: r.arrival)
        active = {k: {} for k in self.batches}
        done = []
        t0 = clock()
        qi = 0
        while qi < len(pending) or any(active[k] for k in active):
            now = clock() - t0
            # admit every arrived request that fits the budget, in arrival order
            while qi < len(pending) and pending[qi].arrival <= now:
                r = pending[qi]
                prebuilt = getattr(r, "_case", None)
                p, g, U = prebuilt if prebuilt is not None else make_case(r, self.precision)
                r.cells = _cells(r)
                r.bytes = 3 * U.numel() * 8
                if self.in_use + r.bytes > self.budget and any(active[k] for k in active):
                    del U
                    break  # wait for memory to free up (FIFO)
                r.case_id = self.batches[r.kind].add(p, g, U, max_steps=r.steps)
                r.admitted = clock() - t0
                r._pg = (p, g)
                r._case = None  # the batch holds its own copy
                self.in_use += r.bytes
                active[r.kind][r.case_id] = r
                qi += 1
                del U
            if not any(active[k] for k in active):
                # idle until the next arrival
                if qi < len(pending):
                    wait = pending[qi].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            for k, b in self.batches.items():
                if active[k]:
                    b.advance(self.steps_per_iter)
            for k, b in self.batches.items():
                if not active[k]:
                    continue
                for info in b.poll():
                    r = active[k].get(info.id)
                    if r is None or not (info.done or info.steps >= r.steps):
                        continue
                    if info.status:
                        raise RuntimeError(f"request {r.rid}: status word {info.status}")
                    r.finished = clock() - t0
                    if self.keep_results:
                        r.result = b.download(r.case_id)
                    b.remove(r.case_id)
                    self.in_use -= r.bytes
                    del active[k][info.id]
                    done.append(r)
        torch.cuda.synchronize()
        return done


def summarize(done, wall_s):
    tts = np.array([r.finished - r.arrival for r in done])
    work = sum(r.cells * 3 * r.steps for r in done)
    return {"requests": len(done), "p50_tts_s": float(np.percentile(tts, 50)), "p99_tts_s": float(np.percentile(tts, 99)),
            "mean_tts_s": float(tts.mean()), "cell_updates_per_s_per_stage": work / wall_s, "wall_s": wall_s}


def sequential_service(requests, precision="fp64", sample_steps=None):
    """Service time of each request alone on a single-case level (device work, after one warm-up
    step on a separate level), keyed by request id. With sample_steps, a request of more steps is
    timed over its first sample_steps steps and the time scaled by steps / sample_steps (the cost of a
    step of a fixed box does not depend on the step)."""
    import torch

    service = {}
    for r in requests:
        p, g, U = make_case(r, precision)
        lv = Level(p, g)
        lv.upload(U)
        lv.advance(1)
        torch.cuda.synchronize()
        lv2 = Level(p, g)
        lv2.upload(U)
        k = r.steps if not sample_steps else min(r.steps, int(sample_steps))
        t0 = time.perf_counter()
        lv2.advance(k)
        lv2.sync()
        service[r.rid] = (time.perf_counter() - t0) * (r.steps / k)
        lv.close()
        lv2.close()
    return service


def sequential_tts(requests, service) -> list:
    """Time-to-solution of each request served one at a time in arrival order (FIFO, no overlap) with
    the given service times."""
    t = 0.0
    tts = []
    for r in sorted(requests, key=lambda x: x.arrival):
        start = max(t, r.arrival)
        t = start + service[r.rid]
        tts.append(t - r.arrival)
    return tts


def sequential_baseline(requests, precision="fp64", service=None):
    """The same requests one at a time on a single-case level (FIFO, no overlap): per-request service
    times measured on the GPU (or given), time-to-solution from the arrival times."""
    if service is None:
        service = sequential_service(requests, precision)
    t = 0.0
    tts = []
    for r in sorted(requests, key=lambda x: x.arrival):
        start = max(t, r.arrival)
        t = start + service[r.rid]
        tts.append(t - r.arrival)
    tts = np.array(tts)
    work = sum(_cells(r) * 3 * r.steps for r in requests)
    busy = sum(service.values())
    return {"p50_tts_s": float(np.percentile(tts, 50)), "p99_tts_s": float(np.percentile(tts, 99)),
            "cell_updates_per_s_per_stage": work / busy, "busy_s": busy}

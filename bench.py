#!/usr/bin/env python
"""Benchmark of the fused WENO5 + HLLC + TVD-RK3 level advance on one or more B200s.

Workload (one rank): the 3D six-equation shock-droplet, 256^3 cells (16.8 M), water droplet of radius
0.1 in air, Mach 2.4 shock, WENO5 + HLLC + TVD-RK3 with the pressure relaxation after every stage,
plain FP64. A step is one coarse time step (ComputeDt + three RK stages) of the whole box; the
metric is cell-updates per second per RK stage (cells x 3 x steps / time). Inputs are larger than L2
(3 state arrays of 144 MB each), so no L2 flush is needed between steps.

  value   device time (CUDA events on the launching stream), state resident in HBM, max over ranks
  e2e     the same metric through the C ABI with host buffers: every step copies the state in from
          pinned host memory, advances one step, and copies the result back
  roofline  the stage kernel alone, timed live with CUDA events: algorithmic bytes per launch
          ((8/3) N 8 B per cell on average over the three stages) / mean launch time, against the
          measured HBM copy bandwidth
  cpu_baseline  the reference's own hot-path arithmetic (the reference headers compiled for the CPU,
          OpenMP over the host cores) on a bounded sample of the same case

Multi-GPU: every rank runs its own independent case (weak scaling, no data-path collective).
`--impl reference` times the reference CPU build alone (rank 0) on the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK stage"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="cells per direction of the cube")
    ap.add_argument("--cpu-n", type=int, default=128, help="cube side of the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=6)
    ap.add_argument("--error-steps", type=int, default=200,
                    help="steps after which the mixed form's error against the FP64 form is measured")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=10)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-phase-field", action="store_true")
    ap.add_argument("--no-phase-field-sixeq", action="store_true", help="only the 2D CAC Phase-Field line")
    ap.add_argument("--no-amr", action="store_true")
    ap.add_argument("--amr-steps", type=int, default=5)
    ap.add_argument("--pf-steps", type=int, default=10)
    ap.add_argument("--force-kernel", default=None,
                    help="shape,order of the stage kernel instead of the autotuner's pick (profiling)")
    ap.add_argument("--e2e-slabs", type=int, default=32, help="slabs of the host-buffer step (e2e)")
    ap.add_argument("--no-tma", action="store_true", help="stage the halo slabs with ordinary loads (profiling)")
    ap.add_argument("--shard", action="store_true",
                    help="one 256^3 case cut into slabs across the ranks (strong scaling) instead of replicas")
    ap.add_argument("--shard-slabs", type=int, default=1, help="with --shard on one GPU: slabs held in the process")
    ap.add_argument("--no-sixn", action="store_true")
    ap.add_argument("--sixn-n", type=int, default=512, help="SIXEQS_IE_NPHASE shock-bubble: 2n x n cells")
    ap.add_argument("--sixn-steps", type=int, default=20)
    ap.add_argument("--no-triple", action="store_true")
    ap.add_argument("--triple-m", type=int, default=256, help="triple point side: 7m x 3m cells")
    ap.add_argument("--triple-steps", type=int, default=20)
    ap.add_argument("--serve-requests", type=int, default=12)
    ap.add_argument("--serve-rate", type=float, default=16.0, help="headline arrival rate (one of --serve-rates)")
    ap.add_argument("--serve-rates", default="4,16", help="arrival rates swept (requests/s)")
    ap.add_argument("--serve-sizes", default="config", choices=["bench", "config"],
                    help="request sizes: 'config' (the serving configuration: 128-1024^2, 64-192^3, triple point "
                         "224x96-896x384, 100-2000 steps) or 'bench' (reduced: 128-512^2, 64-96^3, 100-300 steps)")
    ap.add_argument("--serve-seq-sample", type=int, default=50,
                    help="time the one-at-a-time baselines over this many steps per request and scale (0: all)")
    return ap.parse_args()


def workload_config(n, extra=None):
    cfg = {"workload": f"3D SIXEQS shock-droplet {n}^3, WENO5+HLLC+TVD-RK3, pressure relaxation every stage",
           "cells": n ** 3, "nstate": 8,
           "l2": f"inputs larger than L2 (three state arrays of {(n + 6) ** 3 * 64 / 1e9:.2f} GB), no flush",
           "parallelism": "replicas"}
    if extra:
        cfg.update(extra)
    return cfg


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the mixed stage kernel, from
# one ncu capture of the 128^3 shock-droplet (three launches, one per RK stage, averaged) scaled by the
# 8x cells of a 256^3 launch; a measured constant, not recomputed by this run.
STAGE_TRAFFIC_BYTES = 2.99e9
STAGE_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, mixed stage kernel (TMA form, NT 288), "
                        "128^3 shock-droplet, mean of the three RK stages (373.7 MB), x8 for 256^3")


def _reference_oracle(n):
    """The CPU oracle of the n^3 shock-droplet and its initial state. The case (EOS coefficients,
    scheme ids) comes from the oracle's own reading of the inputs keys and the initial state from the
    package's numpy case builder, so this loads no CUDA library: the reference build
    (oracle/_ref, the reference's own headers) where it exists, else the C restatement."""
    from compas_b200 import cases
    from oracle.oracle import SIXEQS, Oracle, have_ref
    from oracle.parm import reference_case

    phys, dim, inputs, geom, U = cases.shock_droplet(n=n)
    kind = "reference" if have_ref(SIXEQS, 3) else "port"
    return Oracle(kind, reference_case(phys, dim, inputs, geom), None), U


def cpu_baseline(n, steps):
    """The reference-header CPU build (or the C restatement) on an n^3 sample of the same case."""
    o, U = _reference_oracle(n)
    kind = o.kind
    _, dts = o.advance(U, 1)  # untimed: the first step (with the t = 0 wave-speed pass)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.rk3_step(U, float(dts[0]))
    el = time.perf_counter() - t0
    val = n ** 3 * 3 * steps / el
    return {"value": val, "unit": UNIT, "cores": o.threads(), "kind": kind,
            "sample": f"{n}^3 cells of the same shock-droplet case, {steps} coarse steps (3 RK stages each) "
                      f"after one untimed step, OpenMP over {o.threads()} host threads, {el:.1f} s"}


# Algorithmic floating-point operations per cell and RK stage of the 256^3 shock-droplet (SIXEQS 3D,
# WENO5 + HLLC + relaxation), a static count of the formulas with each +, -, *, / and sqrt counted as
# one operation (the per-function table is in DESIGN.md): per face 16 WENO5 calls (79 each), two
# primitive-to-conservative conversions (30), the HLLC flux with its conversions, fluxes and sound
# speeds (437); per cell three faces, one cell conversion (30), the divergence (88), the
# non-conservative terms (14), the stage combination (32 on average) and the closed-form relaxation
# (118). The mixed form does the WENO5 reconstruction, the wave speeds and the star ratios in FP32 and
# the conversions, the upwind-side flux assembly, the divergence, the stage and the relaxation in FP64.
STAGE_FLOPS = {"mixed": {"fp32": 4044, "fp64": 564}, "fp64": {"fp32": 0, "fp64": 5385}}
STAGE_FLOPS_SOURCE = ("static count of the formulas per cell and RK stage, SIXEQS 3D WENO5+HLLC+relaxation, each "
                      "+ - * / sqrt = 1 operation")
# Executed floating-point operations per cell and RK stage, from ncu's SASS operation counters
# (smsp__sass_thread_inst_executed_op_{f,d}{add,mul,fma}_pred_on.sum, FMA = 2) of the 128^3 capture of
# each form's stage kernel, mean of the three RK stages. They exceed the static counts by the
# instruction sequences of the divisions and square roots (reciprocal refinement, range checks).
STAGE_FLOPS_EXECUTED = {"mixed": {"fp32": 3502, "fp64": 1104}, "fp64": {"fp32": 955, "fp64": 17342}}
STAGE_FLOPS_EXECUTED_SOURCE = ("ncu SASS operation counters (add, mul, fma x2) of the 128^3 stage-kernel capture, "
                               "mean of the three RK stages")


def stage_kernel_times(cb, torch, p, g, lv, stream, cells, N):
    """Mean CUDA-event duration of the stage kernel of one form over two steps' stages (launched alone,
    after a warm-up step), with its algorithmic bytes per launch and the boundary-fill time."""
    shape = cb.padded_shape(p, g)
    Us = torch.empty(shape, dtype=torch.float64, device="cuda")
    lv.download(out=Us, stream=stream)
    cb.FillPatch(p, g, Us, stream=stream)
    U0 = Us.clone()
    Un = torch.empty_like(Us)
    dt_dev = torch.tensor([1e-9], dtype=torch.float64, device="cuda")
    cmax = torch.zeros(1, dtype=torch.float64, device="cuda")
    errw = torch.zeros(1, dtype=torch.int32, device="cuda")
    for s in range(3):
        cb.ThirdOrderSSPRK_stage(p, g, s, Us, U0, Un, dt_dev, cmax, errw, stream=stream)
    torch.cuda.synchronize()
    durs, algo = [], []
    for _ in range(2):
        for s in range(3):
            ea = torch.cuda.Event(enable_timing=True)
            eb = torch.cuda.Event(enable_timing=True)
            ea.record(stream)
            cb.ThirdOrderSSPRK_stage(p, g, s, Us, U0, Un, dt_dev, cmax, errw, stream=stream)
            eb.record(stream)
            eb.synchronize()
            durs.append(ea.elapsed_time(eb) / 1e3)
            algo.append(cells * N * 8 * (2 if s == 0 else 3))
    fa = torch.cuda.Event(enable_timing=True)
    fb = torch.cuda.Event(enable_timing=True)
    fa.record(stream)
    cb.FillPatch(p, g, Us, stream=stream)
    fb.record(stream)
    fb.synchronize()
    return {"mean_s": sum(durs) / len(durs), "bytes": sum(algo) / len(algo), "fill_ms": fa.elapsed_time(fb)}


def compute_roofline(name, mean_s, cells, fma_peaks):
    """FP32 and FP64 pipe fractions of one form's stage kernel: executed FLOPs per launch (the frozen
    per-cell counts) / the launch's mean duration, against the measured FMA throughputs."""
    fl = STAGE_FLOPS.get(name)
    out = {"peak_tflops": {k: v / 1e12 for k, v in fma_peaks.items()},
           "peak_source": "compas_b200_fma_peak: sustained FMA rate of each pipe, measured in this run"}
    if fl is None:
        out["note"] = "FLOPs per cell-stage " + STAGE_FLOPS_SOURCE
        return out
    ex = STAGE_FLOPS_EXECUTED.get(name, {})
    for k in ("fp32", "fp64"):
        if not fl[k] and not ex.get(k):
            continue
        ach = fl[k] * cells / mean_s
        out[k] = {"flops_per_cell_stage": fl[k], "achieved_tflops": ach / 1e12, "frac": ach / fma_peaks[k]}
        if ex.get(k):
            ache = ex[k] * cells / mean_s
            out[k].update({"executed_flops_per_cell_stage": ex[k], "executed_tflops": ache / 1e12,
                           "executed_frac": ache / fma_peaks[k]})
    out["flops_source"] = STAGE_FLOPS_SOURCE
    out["executed_source"] = STAGE_FLOPS_EXECUTED_SOURCE
    return out


def run_batched(args):
    """48 independent 2D FIVEEQS shock-bubble cases (seeded, uneven sizes) in one persistent box-list
    launch per RK stage (mixed precision, WENO5B, CUDA-graph steps), against the same cases run one
    after the other on single-case levels."""
    import torch

    import compas_b200 as cb
    from compas_b200 import cases

    stream = torch.cuda.current_stream()
    cs = cases.batch_shock_bubbles(count=48, seed=0, xp=torch, device="cuda")
    cells = sum(c[3]["n"][0] * c[3]["n"][1] for c in cs)
    K, W = args.batch_steps, 2
    out = {"workload": "48 independent 2D FIVEEQS shock-bubble cases, numpy PCG64 seed 0: side U{64..768}, "
                       "aspect U[1,2], Mach U[1.1,3], density ratio logU[0.01,1000], radius U[0.1,0.3]; WENO5B+HLLC",
           "cases": len(cs), "cells": cells, "steps": K}
    for prec in ("mixed", "fp64"):
        b = cb.Batch(cb.FIVEEQS, 2, id_limiter=6, precision=1 if prec == "mixed" else 0)
        for phys, dim, inputs, geom, U, _ in cs:
            b.add(cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec})), cb.make_geom(**geom), U)
        b.advance(W, stream=stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.advance(K, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        assert all(i.status == 0 for i in b.poll())
        out[f"batched_{prec}"] = cells * 3 * K / (ms / 1e3)
        b.close()
        # the same cases one after the other
        tot = 0.0
        for phys, dim, inputs, geom, U, _ in cs:
            lv = cb.Level(cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec})),
                          cb.make_geom(**geom))
            lv.upload(U, stream=stream)
            lv.advance(W, stream=stream)
            e0.record(stream)
            lv.advance(K, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
            lv.close()
        out[f"sequential_{prec}"] = cells * 3 * K / (tot / 1e3)
    out["unit"] = UNIT + " per RK stage (aggregate over the cases)"
    out["batched_mixed_vs_sequential_fp64"] = out["batched_mixed"] / out["sequential_fp64"]
    return out


def run_phase_field(args):
    """2D shock-helium-bubble with the CAC Phase-Field regularisation (the reference's configuration:
    2048 x 1024 cells on [0,2]x[0,1], WENO5B + HLLC, CAC-Adv with the implicit regularisation
    potential, eta = dx): hyperbolic step + Phase-Field step per coarse step, both precisions, against
    the same steps without the Phase-Field step. Timed with CUDA events around whole steps (the
    Phase-Field host loop reads dt, max|u| and max|grad Q| each step, as the reference's does)."""
    import torch

    import compas_b200 as cb
    from compas_b200 import cases

    phys, dim, inputs, geom, U = cases.shock_bubble(nx=2048, ny=1024, xp=torch, device="cuda")
    workload = ("2D FIVEEQS shock-helium-bubble 2048x1024, WENO5B+HLLC+TVD-RK3, CAC-Adv Phase-Field "
                "(implicit regularisation potential, Eta_Multiplier 1), reflective top/bottom, outflow left/right")
    return _phase_field_line(args.pf_steps, phys, dim, inputs, geom, U, workload,
                             {"PhaseField.phase_field": "1", "PhaseField.Mechanism": "CAC-Adv"})


def run_phase_field_sixeq(args):
    """3D six-equation shock-droplet 128^3 with the explicit ACDI Phase-Field step of the reference's
    shock-droplet example (Eta_Multiplier 0.5, PhaseField.cfl 0.3, the phasic formulation of the
    six-equation Parm.H), relaxation after every stage; timed as run_phase_field."""
    import torch

    from compas_b200 import cases

    phys, dim, inputs, geom, U = cases.shock_droplet(n=128, xp=torch, device="cuda")
    workload = ("3D SIXEQS shock-droplet 128^3, WENO5+HLLC+TVD-RK3 with relaxation, ACDI Phase-Field (explicit, "
                "Eta_Multiplier 0.5, cfl 0.3, phasic formulation), outflow on every side")
    return _phase_field_line(max(2, args.pf_steps // 2), phys, dim, inputs, geom, U, workload,
                             {"PhaseField.phase_field": "1", "PhaseField.Mechanism": "ACDI",
                              "PhaseField.ID_ExplicitRC": "1", "PhaseField.Eta_Multiplier": "0.5",
                              "PhaseField.cfl": "0.3"})


def _phase_field_line(K, phys, dim, inputs, geom, U, workload, pf_keys):
    import torch

    import compas_b200 as cb

    stream = torch.cuda.current_stream()
    g = cb.make_geom(**geom)
    cells = geom["n"][0] * geom["n"][1] * (geom["n"][2] if dim == 3 else 1)
    W = 2
    out = {"workload": workload, "cells": cells, "steps": K,
           "unit": UNIT + " per hyperbolic RK stage (Phase-Field step included)"}
    for prec in ("mixed", "fp64"):
        for pf_on in (True, False):
            extra = {"compas_b200.precision": prec}
            if pf_on:
                extra.update(pf_keys)
            p = cb.make_parm(phys, dim, dict(inputs, **extra))
            lv = cb.Level(p, g)
            lv.upload(U, stream=stream)
            lv.advance(W, stream=stream)
            torch.cuda.synchronize()
            sub0 = lv.pf_substeps()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lv.advance(K, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            info = lv.sync()
            assert info.status == 0
            key = f"{prec}_{'with_phase_field' if pf_on else 'hyperbolic_only'}"
            out[key] = cells * 3 * K / (ms / 1e3)
            if pf_on:
                out[f"{prec}_pf_substeps_per_step"] = (lv.pf_substeps() - sub0) / K
                out[f"{prec}_ms_per_step"] = ms / K
            lv.close()
    out["mixed_vs_fp64_with_phase_field"] = out["mixed_with_phase_field"] / out["fp64_with_phase_field"]
    return out


def run_amr(args):
    """3-level AMR shock-helium-bubble (refinement ratio 2, max_grid_size drawn with numpy PCG64 seed 0
    from {32, 64, 128}): level 0 512 x 256 on [0,2]x[0,1], level 1 around the shock and the bubble,
    level 2 around the bubble; every level's boxes advance through the persistent box-list stage
    kernel, one launch per RK stage, subcycled, with refluxing and average-down. Rate: composite
    cell-updates per RK stage (each level's cells x its substeps x 3) per second."""
    import numpy as np
    import torch

    import compas_b200 as cb
    from compas_b200 import amr, cases

    rng = np.random.Generator(np.random.PCG64(0))
    mgs = int(rng.choice([32, 64, 128]))
    kw = dict(nx=512, ny=256, scheme="WENO5B")
    phys, dim, inputs, geom, _ = cases.shock_bubble(**kw, quadrature=False)
    regions = [((64, 96, 0), (895, 415, 0)), ((512, 256, 0), (1407, 767, 0))]
    boxes = amr.hierarchy((512, 256), dim, regions, mgs)
    states = amr.box_states(cases.shock_bubble, kw, (512, 256), dim, boxes, xp=torch, device="cuda")
    cells = [0, 0, 0]
    for lev, lo, hi in boxes:
        cells[lev] += (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1)
    per_step = sum(c * (1 << lev) for lev, c in enumerate(cells)) * 3
    out = {"workload": f"3-level AMR 2D FIVEEQS shock-helium-bubble, level 0 512x256, max_grid_size {mgs} (seed 0), "
                       f"WENO5B+HLLC, subcycled TVD-RK3 with refluxing", "boxes": len(boxes),
           "cells_per_level": cells, "steps": args.amr_steps,
           "unit": UNIT + " per RK stage (composite: each level's cells x substeps)"}
    stream = torch.cuda.current_stream()
    for prec in ("mixed", "fp64"):
        p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec}))
        A = cb.Amr(p, cb.make_geom(**geom), boxes)
        for b, U in enumerate(states):
            A.upload(b, U, stream=stream)
        A.advance(2, stream=stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = A.launches()
        e0.record(stream)
        A.advance(args.amr_steps, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        assert A.sync().status == 0
        out[prec] = per_step * args.amr_steps / (ms / 1e3)
        out[f"{prec}_ms_per_coarse_step"] = ms / args.amr_steps
        out[f"{prec}_launches_per_coarse_step"] = (A.launches() - l0) / args.amr_steps
        A.close()
    out["mixed_vs_fp64"] = out["mixed"] / out["fp64"]
    return out


def run_triple_point(args):
    """2D FIVEEQS_NPHASE (NPHASE = 3) triple point on [0,7]x[0,3] at 1792 x 768 cells (sharp
    interfaces, reflecting walls, WENO5 with the consistent limiter + HLLC + TVD-RK3, cfl 0.4), both
    precisions, single-box level advance timed with CUDA events."""
    import torch

    import compas_b200 as cb
    from compas_b200 import cases

    stream = torch.cuda.current_stream()
    m = args.triple_m
    phys, dim, inputs, geom, U = cases.triple_point(m=m, xp=torch, device="cuda")
    g = cb.make_geom(**geom)
    cells = geom["n"][0] * geom["n"][1]
    K, W = args.triple_steps, 3
    bytes_cs = cases.algorithmic_bytes_per_cell_stage(phys, dim, 3)
    peak = measured_peaks()[0]
    out = {"workload": f"2D FIVEEQS_NPHASE (NPHASE 3) triple point {7 * m}x{3 * m} on [0,7]x[0,3], WENO5 "
                       "(consistent limiter)+HLLC+TVD-RK3, reflecting walls", "cells": cells, "steps": K,
           "unit": UNIT, "algorithmic_bytes_per_cell_stage": bytes_cs}
    for prec in ("mixed", "fp64"):
        p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": prec}))
        lv = cb.Level(p, g)
        lv.upload(U, stream=stream)
        lv.advance(W, stream=stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lv.advance(K, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        info = lv.sync()
        assert info.status == 0
        rate = cells * 3 * K / (ms / 1e3)
        out[prec] = rate
        out[f"{prec}_ms_per_step"] = ms / K
        out[f"{prec}_hbm_frac_of_measured"] = rate * bytes_cs / 1e9 / peak if peak else None
        lv.close()
    out["mixed_vs_fp64"] = out["mixed"] / out["fp64"]
    return out


def run_sixn(args):
    """2D SIXEQS_IE_NPHASE shock-bubble interaction (a Mach 1.1 water shock on an air bubble, with a
    helium bubble for NPHASE 3) at 2n x n cells, MUSCL (consistent limiter) + HLLC + TVD-RK3 with the
    Newton pressure relaxation after every stage, plain FP64 (bit-identical to the reference), phases
    started out of pressure equilibrium; single-box level advance timed with CUDA events. Beside it the
    reference-header CPU build on the same case for three steps (OpenMP over the host threads)."""
    import torch

    import compas_b200 as cb
    from compas_b200 import cases
    from oracle.oracle import Oracle, case_from, have_ref

    stream = torch.cuda.current_stream()
    n, K, W = args.sixn_n, args.sixn_steps, 3
    peak = measured_peaks()[0]
    out = {}
    for npk in (2, 3):
        phys, dim, inputs, geom, U = cases.sixn_shock_bubbles(n=n, nphase=npk, dp=0.05, xp=torch, device="cuda")
        p = cb.make_parm(phys, dim, inputs)
        g = cb.make_geom(**geom)
        cells = geom["n"][0] * geom["n"][1]
        bytes_cs = cases.algorithmic_bytes_per_cell_stage(phys, dim, npk)
        lv = cb.Level(p, g)
        lv.upload(U, stream=stream)
        lv.advance(W, stream=stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lv.advance(K, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        info = lv.sync()
        assert info.status == 0
        lv.close()
        rate = cells * 3 * K / (ms / 1e3)
        res = {"workload": f"2D SIXEQS_IE_NPHASE (NPHASE {npk}) shock-bubble {2 * n}x{n}, MUSCL (consistent "
                           "limiter)+HLLC+TVD-RK3, Newton pressure relaxation after every stage, FP64",
               "cells": cells, "steps": K, "value": rate, "unit": UNIT, "ms_per_step": ms / K,
               "algorithmic_bytes_per_cell_stage": bytes_cs,
               "hbm_frac_of_measured": rate * bytes_cs / 1e9 / peak if peak else None}
        if not args.no_cpu and have_ref(phys, dim, npk):
            m = n
            _, _, _, geom_s, Us = cases.sixn_shock_bubbles(n=m, nphase=npk, dp=0.05)
            o = Oracle("reference", case_from(p, cb.make_geom(**geom_s)), None)
            _, dts = o.advance(Us, 1)
            steps = 3
            t0 = time.perf_counter()
            for _ in range(steps):
                o.rk3_step(Us, float(dts[0]))
            el = time.perf_counter() - t0
            cpu = 2 * m * m * 3 * steps / el
            res["cpu_reference"] = {"value": cpu, "unit": UNIT, "cores": o.threads(), "kind": "reference",
                                    "sample": f"{2 * m}x{m} cells of the same case, {steps} steps after one untimed "
                                              f"step, OpenMP over {o.threads()} host threads, {el:.1f} s"}
            res["speedup_vs_cpu_reference"] = rate / cpu
        out[f"nphase{npk}"] = res
    return out


def run_serving(args, rank=0, world=1, dist=None):
    """Poisson arrivals of mixed 2D shock-bubble / 3D shock-droplet / 2D three-material triple-point
    solves under an HBM budget, continuous batching, at several arrival rates, against the same
    requests one at a time on the plain FP64 path. The request set (kinds, sizes, steps) is the same at
    every rate (the seeded draws do not depend on the rate); only the arrival times scale. With several
    GPUs every rank serves the requests dealt to it (round-robin; no collective on the data path) and
    rank 0 merges the ranks' time-to-solution records; the sequential baseline is each GPU serving its
    share one request at a time."""
    import numpy as np

    from compas_b200 import replicas, serving

    if args.serve_sizes == "config":
        sizes = dict(sides2d=(128, 1024), sides3d=(64, 192), sides_triple=(32, 128), steps=(100, 2000))
        sizes_txt = ("2D FIVEEQS shock-bubble 128^2-1024^2, 3D SIXEQS shock-droplet 64^3-192^3 and 2D FIVEEQS_NPHASE "
                     "(NPHASE 3) triple point 224x96-896x384, 100-2000 steps each")
    else:
        sizes = dict(sides2d=(128, 512), sides3d=(64, 96), sides_triple=(32, 96), steps=(100, 300))
        sizes_txt = ("2D FIVEEQS shock-bubble 128^2-512^2, 3D SIXEQS shock-droplet 64^3-96^3 and 2D FIVEEQS_NPHASE "
                     "(NPHASE 3) triple point 224x96-672x288, 100-300 steps each (reduced sizes)")

    def reqs_at(rate):
        return serving.poisson_requests(args.serve_requests, rate, seed=0, **sizes)

    rates = [float(x) for x in args.serve_rates.split(",")]
    base = reqs_at(rates[0])
    mine_base = replicas.deal_requests(base, rank, world)
    sample = args.serve_seq_sample or None
    service = serving.sequential_service(mine_base, precision="fp64", sample_steps=sample)
    service_mixed = serving.sequential_service(mine_base, precision="mixed", sample_steps=sample)
    kinds = {k: sum(1 for r in base if r.kind == k) for k in serving.KINDS}
    out = {"workload": f"{len(base)} requests {kinds}, Poisson arrivals at each rate (seed 0): {sizes_txt}; budget "
                       "150 GB per GPU; continuous batching in the mixed form vs the same requests one at a time in "
                       "the mixed form and on the plain FP64 path; initial states built before the clock starts"
                       + (f"; one-at-a-time service timed over {sample} steps per request and scaled" if sample else "")
                       + (f"; requests dealt round-robin to {world} GPUs" if world > 1 else ""),
           "rates": {}}
    for rate in rates:
        reqs = replicas.deal_requests(reqs_at(rate), rank, world)
        srv = serving.Server(budget_bytes=150e9, precision="mixed", steps_per_iter=4)
        srv.prepare(reqs)
        t0 = time.perf_counter()
        done = srv.run(reqs)
        wall = time.perf_counter() - t0
        srv.close()
        mine = {"tts": [r.finished - r.arrival for r in done], "work": sum(r.cells * 3 * r.steps for r in done),
                "wall": wall, "seq_tts": serving.sequential_tts(reqs, service),
                "seq_busy": sum(service[r.rid] for r in reqs),
                "seqm_tts": serving.sequential_tts(reqs, service_mixed),
                "seqm_busy": sum(service_mixed[r.rid] for r in reqs)}
        allr = replicas.gather(mine, dist)
        if rank != 0:
            continue
        tts = np.concatenate([np.asarray(x["tts"]) for x in allr])
        seq_tts = np.concatenate([np.asarray(x["seq_tts"]) for x in allr])
        work = sum(x["work"] for x in allr)
        wall_max = max(x["wall"] for x in allr)
        busy_max = max(x["seq_busy"] for x in allr)
        summ = {"requests": int(tts.size), "p50_tts_s": float(np.percentile(tts, 50)),
                "p99_tts_s": float(np.percentile(tts, 99)), "mean_tts_s": float(tts.mean()),
                "cell_updates_per_s_per_stage": work / wall_max, "wall_s": wall_max}
        seq = {"p50_tts_s": float(np.percentile(seq_tts, 50)), "p99_tts_s": float(np.percentile(seq_tts, 99)),
               "cell_updates_per_s_per_stage": work / busy_max, "busy_s": busy_max}
        seqm_tts = np.concatenate([np.asarray(x["seqm_tts"]) for x in allr])
        busym_max = max(x["seqm_busy"] for x in allr)
        seqm = {"p50_tts_s": float(np.percentile(seqm_tts, 50)), "p99_tts_s": float(np.percentile(seqm_tts, 99)),
                "cell_updates_per_s_per_stage": work / busym_max, "busy_s": busym_max}
        out["rates"][f"{rate:g}/s"] = {
            "continuous_batching_mixed": summ, "sequential_mixed": seqm, "sequential_fp64": seq,
            # batching gain (same precision) and the precision gain, separately
            "batching_gain_vs_sequential_mixed": summ["cell_updates_per_s_per_stage"] / seqm["cell_updates_per_s_per_stage"],
            "precision_gain_sequential": seqm["cell_updates_per_s_per_stage"] / seq["cell_updates_per_s_per_stage"],
            "throughput_ratio": summ["cell_updates_per_s_per_stage"] / seq["cell_updates_per_s_per_stage"]}
    if rank != 0:
        return None
    head = out["rates"][f"{args.serve_rate:g}/s"] if f"{args.serve_rate:g}/s" in out["rates"] else \
        next(iter(out["rates"].values()))
    out.update(head)  # the headline rate's figures at the top level
    return out


def run_reference(args, rank):
    if rank != 0:
        return None
    n = args.cpu_n
    o, U = _reference_oracle(n)
    kind = o.kind
    _, dts = o.advance(U, 1)
    for _ in range(args.warmup):
        o.rk3_step(U, float(dts[0]))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.rk3_step(U, float(dts[0]))
    el = time.perf_counter() - t0
    val = n ** 3 * 3 * args.steps / el
    sample = (f"each step one coarse step (3 RK stages) of the same shock-droplet case on a {n}^3 box "
              f"(a bounded sample of the {args.n}^3 workload), OpenMP over {o.threads()} host threads")
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args.n, {"parallelism": "CPU, rank 0 only"}),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": o.threads(), "kind": kind, "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_ours(args, rank, world, dist):
    import numpy as np
    import torch

    import compas_b200 as cb
    from compas_b200 import cases

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    n = args.n
    phys, dim, inputs, geom, U = cases.shock_droplet(n=n, xp=torch, device="cuda")
    g = cb.make_geom(**geom)
    cells = n ** 3
    if args.no_tma:
        inputs = dict(inputs, **{"compas_b200.tma": "0"})
    forms = {"mixed": cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"})),
             "fp64": cb.make_parm(phys, dim, inputs)}
    if args.precision != "both":
        forms = {args.precision: forms[args.precision]}

    from compas_b200 import replicas

    def barrier():
        replicas.barrier(dist, torch.cuda.synchronize)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, device="cuda")

    levels, ms, clks, tuned = {}, {}, [], {}
    for name, p in forms.items():
        lv = cb.Level(p, g)
        if args.force_kernel:
            lv.set_kernel(*(int(x) for x in args.force_kernel.split(",")))
        lv.upload(U, stream=stream)
        # warm-up (includes the t = 0 wave-speed pass and the CUDA-graph capture)
        lv.advance(args.warmup, use_graph=True, stream=stream)
        torch.cuda.synchronize()
        info0 = lv.sync()
        clocks = Clocks(local)
        barrier()
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lv.advance(args.steps, use_graph=True, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t_ms = e0.elapsed_time(e1)
        clks.append(clocks.stop())
        barrier()
        info = lv.sync()
        assert info.steps == info0.steps + args.steps, (info0, info)
        ms[name] = max_over_ranks(t_ms)
        levels[name] = lv
        tuned[name] = lv.kernel() + (lv.tma(),)
    head = "mixed" if "mixed" in forms else "fp64"
    p = forms[head]
    value = replicas.whole_job_rate(cells, 3, args.steps, ms[head] / 1e3, world)

    # error of the mixed form against the FP64 form after the configuration's step count (both levels
    # continue, untimed, from the warm-up + timed steps to --error-steps)
    err = None
    if len(levels) == 2:
        done = args.warmup + args.steps
        if args.error_steps > done:
            for lvx in levels.values():
                lvx.advance(args.error_steps - done, use_graph=True, stream=stream)
            torch.cuda.synchronize()
            for lvx in levels.values():
                assert lvx.sync().status == 0
        done = max(done, args.error_steps)
        shape = cb.padded_shape(p, g)
        a = torch.empty(shape, dtype=torch.float64, device="cuda")
        b = torch.empty(shape, dtype=torch.float64, device="cuda")
        levels["mixed"].download(out=a, stream=stream)
        levels["fp64"].download(out=b, stream=stream)
        torch.cuda.synchronize()
        va, vb = cb.valid_view(a, p, g), cb.valid_view(b, p, g)
        names = ["a1rho1", "a2rho2", "rho_u", "rho_v", "rho_w", "a1rho1E1", "a2rho2E2", "alpha1"]
        err = {"norm": "relative L1 (sum|mixed - fp64| / sum|fp64|) per field after "
                       f"{done} steps of the {n}^3 workload",
               "fields": {nm: float((va[c] - vb[c]).abs().sum() / vb[c].abs().sum()) for c, nm in enumerate(names)},
               "bound": "<= 1e-5 in a1rho1, a2rho2, alpha1"}
        del a, b

    # ---- roofline: each form's stage kernel alone, CUDA events around each launch ----
    N = cb.nstate(p.physics, p.dim)
    shape = cb.padded_shape(p, g)
    kern = {name: stage_kernel_times(cb, torch, forms[name], g, levels[name], stream, cells, N) for name in forms}
    mean_dur, bytes_per_launch, fill_ms = kern[head]["mean_s"], kern[head]["bytes"], kern[head]["fill_ms"]
    achieved = bytes_per_launch / mean_dur / 1e9
    peak, peak_kind = measured_peaks()
    fma_peaks = {"fp32": cb.fma_peak(False, stream=stream), "fp64": cb.fma_peak(True, stream=stream)}

    # ---- e2e: host state in, one step, result out, every step (headline form) ----
    lv = levels[head]
    host_in = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    host_out = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    lv.download(out=host_in, stream=stream)
    torch.cuda.synchronize()
    lv.step_host(host_in, host_out, slabs=args.e2e_slabs, stream=stream)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lv.step_host(host_in, host_out, slabs=args.e2e_slabs, stream=stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = replicas.whole_job_rate(cells, 3, args.steps, e2e_s, world)
    lv.sync()
    nbytes = int(lv.nbytes)
    for l in levels.values():
        l.close()

    clk = None
    good = [c for c in clks if c]
    if good:
        clk = {"sm_mhz": statistics.median([c["sm_mhz"] for c in good]), "sm_max_mhz": good[0]["sm_max_mhz"],
               "reasons": sorted(set(r for c in good for r in c["reasons"])),
               "samples": sum(c["samples"] for c in good)}
    line = None
    # serving runs on every rank (each serves its dealt requests); the rest of the extras on rank 0
    serving_res = None if args.no_serving else run_serving(args, rank, world, dist)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_baseline(args.cpu_n, args.cpu_steps)
        batched = None if args.no_batched else run_batched(args)
        pf_res = None if args.no_phase_field else run_phase_field(args)
        pf6_res = None if (args.no_phase_field or args.no_phase_field_sixeq) else run_phase_field_sixeq(args)
        amr_res = None if args.no_amr else run_amr(args)
        triple_res = None if args.no_triple else run_triple_point(args)
        sixn_res = None if args.no_sixn else run_sixn(args)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms[head] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 reconstruction, f64 state/EOS/Riemann/relaxation" if head == "mixed" else "f64",
            "data": "synthetic",
            "config": workload_config(n, {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                          "precision": head,
                                          "stage_kernel_autotuned": {
                                              k: {"launch_shape": v[0], "tile_order": ("x fastest", "bricks")[v[1]],
                                                  "tma_halo_staging": v[2]}
                                              for k, v in tuned.items()}}),
            "fp64_plain": ({"value": replicas.whole_job_rate(cells, 3, args.steps, ms["fp64"] / 1e3, world),
                            "ms_per_step": ms["fp64"] / args.steps,
                            "note": "bit-identical to the reference CPU arithmetic"} if "fp64" in ms else None),
            "mixed_error_vs_fp64": err,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "path": f"C-ABI compas_b200_level_step_host: pinned host state in, one step, pinned host state "
                            f"out, {args.e2e_slabs} z-slabs with the copies in both directions overlapping the stages"},
            "gpu_launches": 8 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": STAGE_TRAFFIC_BYTES if head == "mixed" else None,
                         "traffic_source": STAGE_TRAFFIC_SOURCE if head == "mixed" else None,
                         "kernel": f"stage_kernel<SixEq<3>, WENO5, {head}> (fused WENO5+HLLC+divergence+RK3+relaxation)",
                         "bytes_per_launch": bytes_per_launch, "mean_launch_ms": mean_dur * 1e3,
                         "peak_source": f"{peak_kind} HBM copy bandwidth (MEASURED_PEAKS.json)",
                         "compute": compute_roofline(head, mean_dur, cells, fma_peaks),
                         # the plain FP64 form's kernel (bit-identical to the reference arithmetic)
                         "fp64_form": ({"mean_launch_ms": kern["fp64"]["mean_s"] * 1e3,
                                        "achieved": kern["fp64"]["bytes"] / kern["fp64"]["mean_s"] / 1e9,
                                        "frac": kern["fp64"]["bytes"] / kern["fp64"]["mean_s"] / 1e9 / peak,
                                        "compute": compute_roofline("fp64", kern["fp64"]["mean_s"], cells, fma_peaks),
                                        "cell_updates_per_s_per_stage": cells / kern["fp64"]["mean_s"]}
                                       if "fp64" in kern and head != "fp64" else None)},
            "fill_boundary_ms": fill_ms,
            "clocks": clk,
            "cpu_baseline": cpu,
            "batched": batched,
            "serving": serving_res,
            "phase_field": pf_res,
            "phase_field_sixeq": pf6_res,
            "amr": amr_res,
            "triple_point": triple_res,
            "sixeqs_ie_nphase": sixn_res,
        }
        if cpu:
            # device-resident speed-up over the reference CPU arithmetic, per precision form; "fp64" is the
            # same-precision figure (the plain path is bit-identical to the reference's arithmetic)
            line["speedup_vs_cpu_baseline"] = {head: value / cpu["value"]}
            if line["fp64_plain"]:
                line["speedup_vs_cpu_baseline"]["fp64"] = line["fp64_plain"]["value"] / cpu["value"]
    return line


def run_sharded(args, rank, world, dist):
    """The 3D SIXEQS shock-droplet (mixed form) as ONE case cut along z into slabs across the ranks
    (compas_b200.sharded: NCCL ghost-plane exchange per RK stage, wave-speed maximum per step; on one
    GPU --shard-slabs slabs held in the process). Strong scaling: value = the case's cell-updates per
    RK stage / the slowest rank's time."""
    import torch

    import compas_b200 as cb
    from compas_b200 import cases, replicas, sharded

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.n
    phys, dim, inputs, geom, U = cases.shock_droplet(n=n, xp=torch, device="cuda")
    p = cb.make_parm(phys, dim, dict(inputs, **{"compas_b200.precision": "mixed"}))
    g = cb.make_geom(**geom)
    comm = sharded.DistComm(dist, device="cuda") if world > 1 else sharded.LocalComm(args.shard_slabs)
    lv = sharded.ShardedLevel(p, g, comm)
    lv.upload(U)
    del U
    lv.advance(args.warmup)
    replicas.barrier(dist, torch.cuda.synchronize)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    lv.advance(args.steps)
    e1.record()
    replicas.barrier(dist, torch.cuda.synchronize)
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
    assert lv.status() == 0
    if rank != 0:
        return None
    slabs = world if world > 1 else args.shard_slabs
    return {"metric": METRIC, "value": n ** 3 * 3 * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32 reconstruction, f64 state/EOS/Riemann/relaxation",
            "data": "synthetic (analytic initial condition)",
            "config": {"workload": f"3D SIXEQS shock-droplet {n}^3, WENO5+HLLC+TVD-RK3 with relaxation, one case "
                                   f"in {slabs} z-slabs", "parallelism": f"sharded x{slabs}",
                       "l2": "inputs larger than L2"},
            "gpu_launches": 6 * slabs * args.steps // max(world, 1),
            "e2e": None, "note": "host-driven steps (dt on the host, a fill and a stage launch per slab and stage); "
                                 "the headline line is the single-box level"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        line = run_sharded(args, rank, world, dist) if args.shard else run_ours(args, rank, world, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

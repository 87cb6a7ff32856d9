"""Plot files and checkpoints of levels and multi-level hierarchies.

Plot files follow AMReX's plotfile layout, as COMPAS writes them with WriteMultiLevelPlotfile
(source/COMPAS.cpp:2483-2511): a directory holding a `Header` (HyperCLaw-V1.1: variable names,
dimension, time, finest level, domain corners, refinement ratios, each level's domain box, step and
cell size, then per level its boxes in physical coordinates) and per level `Level_<l>/Cell_H` (the
box list, one FabOnDisk entry per box, per-box minima and maxima) with the data in
`Level_<l>/Cell_D_00000` (per box a FAB header line naming little-endian IEEE doubles and the box,
then the components one after the other, x fastest). The plot variables are computed on the device
(compas_b200_derive: the reference's compute_derived_var, state or derived names).

Checkpoints keep what a restart needs to continue the run to the bit: the `Header` in the layout of
COMPAS's WriteCheckpointFile (title line, finest level, step, dt and time per level, each level's box
array), an engine line with the last step's largest face wave speed (the next step's ComputeDt input)
as an exact hexadecimal float, and the padded state of every box (ghost cells included, little-endian
doubles) in `Level_<l>/Cell_D`. A level restarts through set_state + set_control.
"""
from __future__ import annotations

import os

import numpy as np

from . import _DERIVED_NAMES, Level, derive, padded_shape

_FAB_REAL = "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))"


def _box_str(lo, hi, dim):
    f = lambda v: "(" + ",".join(str(int(x)) for x in v[:dim]) + ")"  # noqa: E731
    return f"({f(lo)} {f(hi)} {f([0, 0, 0])})"


def write_plotfile(path, levels, names, time, steps, prob_lo, prob_hi, dx0, dim):
    """levels[l] = list of (lo, hi, data) with data (len(names), nz, ny, nx) float64 of the box's
    valid cells; level l has cell size dx0 / 2^l and refinement ratio 2 to the next."""
    nlev = len(levels)
    os.makedirs(path, exist_ok=True)
    dom_lo = [0, 0, 0]
    doms = []
    for l in range(nlev):
        ncell = [int(round((prob_hi[d] - prob_lo[d]) / dx0[d])) << l for d in range(dim)]
        doms.append((dom_lo, [n - 1 for n in ncell]))
    with open(os.path.join(path, "Header"), "w") as h:
        h.write("HyperCLaw-V1.1\n")
        h.write(f"{len(names)}\n")
        for nm in names:
            h.write(nm + "\n")
        h.write(f"{dim}\n")
        h.write(f"{time:.17g}\n")
        h.write(f"{nlev - 1}\n")
        h.write(" ".join(f"{prob_lo[d]:.17g}" for d in range(dim)) + "\n")
        h.write(" ".join(f"{prob_hi[d]:.17g}" for d in range(dim)) + "\n")
        h.write(" ".join("2" for _ in range(nlev - 1)) + "\n")
        h.write(" ".join(_box_str(lo, hi, dim) for lo, hi in doms) + "\n")
        h.write(" ".join(str(int(steps)) for _ in range(nlev)) + "\n")
        for l in range(nlev):
            h.write(" ".join(f"{dx0[d] / (1 << l):.17g}" for d in range(dim)) + "\n")
        h.write("0\n0\n")
        for l, boxes in enumerate(levels):
            h.write(f"{l} {len(boxes)} {time:.17g}\n{int(steps)}\n")
            dxl = [dx0[d] / (1 << l) for d in range(dim)]
            for lo, hi, _ in boxes:
                for d in range(dim):
                    h.write(f"{prob_lo[d] + lo[d] * dxl[d]:.17g} {prob_lo[d] + (hi[d] + 1) * dxl[d]:.17g}\n")
            h.write(f"Level_{l}/Cell\n")
    for l, boxes in enumerate(levels):
        ldir = os.path.join(path, f"Level_{l}")
        os.makedirs(ldir, exist_ok=True)
        offsets = []
        with open(os.path.join(ldir, "Cell_D_00000"), "wb") as f:
            for lo, hi, data in boxes:
                offsets.append(f.tell())
                f.write(f"{_FAB_REAL}{_box_str(lo, hi, dim)} {len(names)}\n".encode())
                f.write(np.ascontiguousarray(data, dtype="<f8").tobytes())
        with open(os.path.join(ldir, "Cell_H"), "w") as c:
            c.write(f"1\n0\n{len(names)}\n0\n({len(boxes)} 0\n")
            for lo, hi, _ in boxes:
                c.write(_box_str(lo, hi, dim) + "\n")
            c.write(")\n")
            c.write(f"{len(boxes)}\n")
            for off in offsets:
                c.write(f"FabOnDisk: Cell_D_00000 {off}\n")
            c.write("\n")
            for fn in (np.min, np.max):
                c.write(f"{len(boxes)},{len(names)}\n")
                for _, _, data in boxes:
                    vals = fn(np.asarray(data).reshape(len(names), -1), axis=1)
                    c.write("".join(f"{v:.17g}," for v in vals) + "\n")


def _parse_box(s):
    parts = s.strip().strip("()").split(") (")
    lo = [int(x) for x in parts[0].strip("(").split(",")]
    hi = [int(x) for x in parts[1].split(",")]
    return lo, hi


def read_plotfile(path):
    """(names, time, levels) of a plot file written by write_plotfile; levels[l] = [(lo, hi, data)]."""
    with open(os.path.join(path, "Header")) as h:
        lines = h.read().split("\n")
    assert lines[0] == "HyperCLaw-V1.1"
    nv = int(lines[1])
    names = lines[2:2 + nv]
    dim = int(lines[2 + nv])
    time = float(lines[3 + nv])
    finest = int(lines[4 + nv])
    levels = []
    for l in range(finest + 1):
        ldir = os.path.join(path, f"Level_{l}")
        with open(os.path.join(ldir, "Cell_H")) as c:
            cl = c.read().split("\n")
        nb = int(cl[4].strip("(").split()[0])
        boxes = [_parse_box(cl[5 + b]) for b in range(nb)]
        offs = [int(x.split()[-1]) for x in cl if x.startswith("FabOnDisk:")]
        raw = open(os.path.join(ldir, "Cell_D_00000"), "rb").read()
        out = []
        for (lo, hi), off in zip(boxes, offs):
            end = raw.index(b"\n", off)
            head = raw[off:end].decode()
            assert head.startswith(_FAB_REAL)
            n = [hi[d] - lo[d] + 1 for d in range(dim)] + [1] * (3 - dim)
            cnt = nv * n[0] * n[1] * n[2]
            data = np.frombuffer(raw, dtype="<f8", count=cnt, offset=end + 1).reshape(nv, n[2], n[1], n[0])
            lo3 = list(lo) + [0] * (3 - dim)
            hi3 = list(hi) + [0] * (3 - dim)
            out.append((tuple(lo3), tuple(hi3), data.copy()))
        levels.append(out)
    return names, time, levels


def level_plotfile(path, lv: Level, names=None, prob_lo=(0.0, 0.0, 0.0), stream=None):
    """Plot file of a single-box level: the plot variables (default: every derived name of the model)
    computed on the device from the level's current state."""
    import torch

    p, g = lv.p, lv.g
    dim = p.dim
    names = list(names or _DERIVED_NAMES[p.physics])
    U = torch.empty(padded_shape(p, g), dtype=torch.float64, device="cuda")
    lv.download(out=U, stream=stream)
    from . import FillPatch

    FillPatch(p, g, U, stream=stream)
    nz = g.n[2] if dim == 3 else 1
    out = torch.empty((len(names), nz, g.n[1], g.n[0]), dtype=torch.float64, device="cuda")
    derive(p, g, U, names, out, stream=stream)
    info = lv.get_control()
    lo = (0, 0, 0)
    hi = (g.n[0] - 1, g.n[1] - 1, (g.n[2] - 1) if dim == 3 else 0)
    prob_hi = [prob_lo[d] + g.n[d] * g.dx[d] for d in range(3)]
    write_plotfile(path, [[(lo, hi, out.cpu().numpy())]], names, info["t"], info["steps"], prob_lo, prob_hi,
                   [g.dx[d] for d in range(3)], dim)


def amr_plotfile(path, A, names=None, prob_lo=(0.0, 0.0, 0.0), stream=None):
    """Plot file of a multi-level hierarchy (compas_b200.Amr): every level's ghost cells filled at its
    current time, the plot variables computed on the device box by box."""
    import torch

    from . import make_geom, parm_nstate

    p, g0 = A.p, A.g0
    dim = p.dim
    names = list(names or _DERIVED_NAMES[p.physics])
    nlev = 1 + max(b[0] for b in A.boxes)
    levels = [[] for _ in range(nlev)]
    for lev in range(nlev):
        A.fill(lev, stream=stream)
    for b, (lev, lo, hi) in enumerate(A.boxes):
        n = [hi[d] - lo[d] + 1 for d in range(3)]
        gb = make_geom(n, [g0.dx[d] / (1 << lev) if d < dim else 1.0 for d in range(3)], g0.ng)
        ng = g0.ng
        shape = (parm_nstate(p), (n[2] + 2 * ng) if dim == 3 else 1, n[1] + 2 * ng, n[0] + 2 * ng)
        U = torch.empty(shape, dtype=torch.float64, device="cuda")
        A.download(b, out=U, stream=stream)
        out = torch.empty((len(names), n[2] if dim == 3 else 1, n[1], n[0]), dtype=torch.float64, device="cuda")
        derive(p, gb, U, names, out, stream=stream)
        levels[lev].append((tuple(lo), tuple(hi), out.cpu().numpy()))
    info = A.sync()
    prob_hi = [prob_lo[d] + g0.n[d] * g0.dx[d] for d in range(3)]
    write_plotfile(path, levels, names, info.t, info.steps, prob_lo, prob_hi, [g0.dx[d] for d in range(3)], dim)


def write_checkpoint(path, lv: Level):
    """Checkpoint of a single-box level (the layout of COMPAS's WriteCheckpointFile for the header)."""
    info = lv.get_control()
    dim = lv.p.dim
    g = lv.g
    os.makedirs(os.path.join(path, "Level_0"), exist_ok=True)
    lo = (0, 0, 0)
    hi = (g.n[0] - 1, g.n[1] - 1, (g.n[2] - 1) if dim == 3 else 0)
    with open(os.path.join(path, "Header"), "w") as h:
        h.write("Checkpoint file for COMPAS\n0\n")
        h.write(f"{info['steps']} \n{info['dt_prev']:.17g} \n{info['t']:.17g} \n")
        h.write(f"(1 0\n{_box_str(lo, hi, dim)}\n)\n")
        h.write(f"compas_b200 cmax {float(info['cmax']).hex()} dt_prev {float(info['dt_prev']).hex()} "
                f"t {float(info['t']).hex()} ng {g.ng}\n")
    U = lv.download()
    with open(os.path.join(path, "Level_0", "Cell_D"), "wb") as f:
        f.write(np.ascontiguousarray(U, dtype="<f8").tobytes())


def read_checkpoint(path, lv: Level, stream=None):
    """Restart a level (of the checkpoint's parameters and geometry) from a checkpoint."""
    with open(os.path.join(path, "Header")) as h:
        lines = h.read().split("\n")
    assert lines[0] == "Checkpoint file for COMPAS"
    steps = int(lines[2].split()[0])
    eng = [x for x in lines if x.startswith("compas_b200 ")][0].split()
    kv = {eng[i]: eng[i + 1] for i in range(1, len(eng) - 1, 2)}
    U = np.fromfile(os.path.join(path, "Level_0", "Cell_D"), dtype="<f8").reshape(lv.shape)
    lv.set_state(U, stream=stream)
    lv.set_control(float.fromhex(kv["t"]), float.fromhex(kv["dt_prev"]), float.fromhex(kv["cmax"]), steps,
                   stream=stream)


__all__ = ["write_plotfile", "read_plotfile", "level_plotfile", "amr_plotfile", "write_checkpoint",
           "read_checkpoint"]

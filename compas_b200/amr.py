"""Fixed AMR hierarchies (refinement ratio 2) for the multi-level advance: box lists per level and the
initial data of every box.

A hierarchy is a list of boxes (level, lo, hi) with inclusive corners in the level's index space.
Level 0 tiles the domain; every finer level tiles a rectangle that lies inside the refinement of
the level below, at least `nest` coarse cells away from that level's region boundary (inside the
domain), so that its ghost cells and their interpolation stencil reach valid coarse cells, as
AMReX's proper nesting guarantees. Boxes are chopped to at most `max_grid_size` cells per side
(amr.max_grid_size of the reference, source/COMPAS.cpp:1276-1314).
"""
from __future__ import annotations

import numpy as np

from . import nstate


def chop(lo, hi, mgs, dim):
    """Boxes of at most mgs cells per side tiling [lo, hi] (inclusive)."""
    ranges = []
    for d in range(dim):
        edges = list(range(lo[d], hi[d] + 1, mgs))
        ranges.append([(e, min(e + mgs - 1, hi[d])) for e in edges])
    out = []
    if dim == 2:
        for (y0, y1) in ranges[1]:
            for (x0, x1) in ranges[0]:
                out.append(((x0, y0, 0), (x1, y1, 0)))
    else:
        for (z0, z1) in ranges[2]:
            for (y0, y1) in ranges[1]:
                for (x0, x1) in ranges[0]:
                    out.append(((x0, y0, z0), (x1, y1, z1)))
    return out


def nested_regions(domain, dim, regions, nest=4):
    """Check and return the refined rectangles: regions[l] (l >= 1) in level-l index space must lie in
    the refinement of regions[l-1] shrunk by `nest` coarse cells (except along the domain boundary)."""
    out = [((0, 0, 0), tuple(domain[d] - 1 if d < dim else 0 for d in range(3)))]
    for lev, (lo, hi) in enumerate(regions, start=1):
        plo, phi = out[-1]
        ndom = [domain[d] << (lev - 1) for d in range(dim)]
        for d in range(dim):
            if lo[d] % 2 or (hi[d] + 1) % 2:
                raise ValueError("refined regions must be aligned to the refinement ratio")
            clo, chi = lo[d] // 2, (hi[d] + 1) // 2 - 1
            need_lo = plo[d] + (nest if plo[d] > 0 else 0)
            need_hi = phi[d] - (nest if phi[d] < ndom[d] - 1 else 0)
            if clo < need_lo or chi > need_hi:
                raise ValueError(f"level {lev} region {lo}-{hi} is not properly nested in level {lev - 1}")
        out.append((tuple(lo), tuple(hi)))
    return out


def hierarchy(domain, dim, regions, max_grid_size, nest=4):
    """Box list [(lev, lo, hi), ...]: level 0 tiles the domain, level l >= 1 tiles regions[l-1]."""
    regs = nested_regions(domain, dim, regions, nest)
    boxes = []
    for lev, (lo, hi) in enumerate(regs):
        for blo, bhi in chop(lo, hi, max_grid_size, dim):
            boxes.append((lev, blo, bhi))
    return boxes


def box_states(case_fn, kw, domain, dim, boxes, ng=3, xp=None, device=None):
    """Initial padded state of every box: the case's cell averages at the box's level resolution
    (the reference's InitData on each level, include/InitData.H:19-290)."""
    nlev = 1 + max(b[0] for b in boxes)
    full = {}
    for lev in range(nlev):
        scale = 1 << lev
        kw_l = dict(kw)
        if dim == 2 and "nx" in kw:
            kw_l.update(nx=kw["nx"] * scale, ny=kw["ny"] * scale)
        elif "m" in kw:  # the triple point: 7m x 3m cells
            kw_l.update(m=kw["m"] * scale)
        else:
            kw_l.update(n=kw["n"] * scale)
        phys, d, inputs, geom, U = case_fn(ng=ng, xp=xp, device=device, **kw_l)
        full[lev] = (U, geom)
    out = []
    for lev, lo, hi in boxes:
        U = full[lev][0]
        gz = ng if dim == 3 else 0
        sl = [slice(None)]
        if dim == 3:
            sl.append(slice(lo[2] - ng + gz, hi[2] + ng + 1 + gz))
        else:
            sl.append(slice(0, 1))
        sl.append(slice(lo[1] - ng + ng, hi[1] + ng + 1 + ng))
        sl.append(slice(lo[0] - ng + ng, hi[0] + ng + 1 + ng))
        part = U[tuple(sl)]
        out.append(part.copy() if xp is None or xp is np else part.contiguous())
    return out


def level0_geom(case_fn, kw, ng=3):
    """(physics, dim, inputs, geom) of level 0 of the case."""
    phys, dim, inputs, geom, _ = case_fn(ng=ng, quadrature=False, **kw)
    return phys, dim, inputs, geom


def composite_sum(states, boxes, dim, ng, comp, covered_by_finer):
    """Sum of component comp over the composite grid (uncovered cells of every level) times the cell
    volume of its level (relative to level 0)."""
    total = 0.0
    for (lev, lo, hi), U in zip(boxes, states):
        v = np.asarray(U)[comp]
        gz = ng if dim == 3 else 0
        if dim == 2:
            inner = v[0, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1]
        else:
            inner = v[gz:gz + hi[2] - lo[2] + 1, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1]
        mask = covered_by_finer(lev, lo, hi)
        vol = 1.0 / (1 << (dim * lev))
        total += float(inner[~mask].sum()) * vol
    return total


def covered_mask_fn(boxes, dim):
    """covered(lev, lo, hi) -> boolean mask of the box's valid cells covered by level lev + 1."""
    fine = {}
    for lev, lo, hi in boxes:
        fine.setdefault(lev, []).append((lo, hi))

    def covered(lev, lo, hi):
        shape = tuple(hi[d] - lo[d] + 1 for d in reversed(range(dim)))
        m = np.zeros(shape, dtype=bool)
        for flo, fhi in fine.get(lev + 1, []):
            clo = [max(flo[d] // 2, lo[d]) for d in range(dim)]
            chi = [min(fhi[d] // 2, hi[d]) for d in range(dim)]
            if any(clo[d] > chi[d] for d in range(dim)):
                continue
            if dim == 2:
                m[clo[1] - lo[1]:chi[1] - lo[1] + 1, clo[0] - lo[0]:chi[0] - lo[0] + 1] = True
            else:
                m[clo[2] - lo[2]:chi[2] - lo[2] + 1, clo[1] - lo[1]:chi[1] - lo[1] + 1,
                  clo[0] - lo[0]:chi[0] - lo[0] + 1] = True
        return m

    return covered


__all__ = ["chop", "hierarchy", "box_states", "level0_geom", "composite_sum", "covered_mask_fn", "nstate"]

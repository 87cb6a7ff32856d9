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


def _dilate(mask, r):
    """Cells within r cells (max norm) of a set cell."""
    if r <= 0:
        return mask.copy()
    out = mask.copy()
    for ax in range(mask.ndim):
        acc = out.copy()
        for s in range(1, r + 1):
            fwd = np.zeros_like(out)
            bwd = np.zeros_like(out)
            sl_a = [slice(None)] * out.ndim
            sl_b = [slice(None)] * out.ndim
            sl_a[ax], sl_b[ax] = slice(s, None), slice(None, -s)
            fwd[tuple(sl_a)] = out[tuple(sl_b)]
            bwd[tuple(sl_b)] = out[tuple(sl_a)]
            acc |= fwd | bwd
        out = acc
    return out


def _region_mask(boxes, lev, shape):
    """Cells of level lev (array (nz, ny, nx)) covered by the boxes of that level."""
    m = np.zeros(shape, dtype=bool)
    for l, lo, hi in boxes:
        if l == lev:
            m[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = True
    return m


def cluster_blocks(marked, bs, mgs):
    """Boxes (lo, hi) in level cells covering the marked blocks (array (nbz, nby, nbx) of blocks of bs
    cells): greedy, x runs first, then whole runs stacked along y and z, each box at most mgs cells
    per side."""
    nbz, nby, nbx = marked.shape
    lim = max(1, mgs // bs)
    free = marked.copy()
    out = []
    for bz in range(nbz):
        for by in range(nby):
            for bx in range(nbx):
                if not free[bz, by, bx]:
                    continue
                x1 = bx
                while x1 + 1 < nbx and free[bz, by, x1 + 1] and x1 + 1 - bx < lim:
                    x1 += 1
                y1 = by
                while y1 + 1 < nby and y1 + 1 - by < lim and free[bz, y1 + 1, bx:x1 + 1].all():
                    y1 += 1
                z1 = bz
                while z1 + 1 < nbz and z1 + 1 - bz < lim and free[z1 + 1, by:y1 + 1, bx:x1 + 1].all():
                    z1 += 1
                free[bz:z1 + 1, by:y1 + 1, bx:x1 + 1] = False
                out.append(((bx * bs, by * bs, bz * bs), ((x1 + 1) * bs - 1, (y1 + 1) * bs - 1, (z1 + 1) * bs - 1)))
    return out


def regrid_boxes(tags_by_level, boxes, domain, dim, n_error_buf=1, blocking_factor=8, max_grid_size=32, nest=4):
    """New box list from the refinement tags of every level but the finest (the regrid after ErrorEst):
    tags_by_level[l] holds, for each box of level l (in the order of `boxes`), its (nz, ny, nx) tag
    array. Per level l, the tags are buffered by n_error_buf cells; blocks of blocking_factor / 2 level-l
    cells (blocking_factor fine cells) holding a tag are marked; only blocks inside the region of the new
    level l (the old level 0, or the boxes just made for it) shrunk by `nest` level-l cells away from
    that region's boundary inside the domain are kept (proper nesting); the marked blocks are clustered
    into boxes of at most max_grid_size fine cells per side. Level 0 is kept; a level whose tags give
    no block keeps one block at the centre of the nested region. This clustering is this engine's own:
    blocks aligned to the blocking factor, greedy x-then-y-then-z growth (AMReX clusters tags with
    Berger-Rigoutsos instead)."""
    nlev = 1 + max(b[0] for b in boxes)
    new = [b for b in boxes if b[0] == 0]
    if blocking_factor % 2 or blocking_factor < 2:
        raise ValueError("blocking_factor must be even")
    bs = blocking_factor // 2
    for l in range(nlev - 1):
        dom = [domain[d] << l if d < dim else 1 for d in range(3)]
        shape = (dom[2], dom[1], dom[0])
        if any(dom[d] % bs for d in range(dim)):
            raise ValueError("the level's domain must be a multiple of blocking_factor / 2 cells")
        tags = np.zeros(shape, dtype=bool)
        lb = [b for b in boxes if b[0] == l]
        for (lev, lo, hi), t in zip(lb, tags_by_level[l]):
            tags[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] |= np.asarray(t, dtype=bool).reshape(
                hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
        if dim == 2:
            tags = tags[:1]
        tags = _dilate(tags, n_error_buf) if dim == 3 else _dilate(tags[0], n_error_buf)[None]
        # nesting: inside the new level-l region, nest cells from its boundary (not from the domain's)
        region = _region_mask(new, l, shape)
        outside = ~region
        if dim == 2:
            outside_d = _dilate(outside[0], nest)[None]
        else:
            outside_d = _dilate(outside, nest)
        allowed = region & ~outside_d
        tags &= allowed
        nb = [dom[d] // bs if d < dim else 1 for d in range(3)]
        blk_t = tags.reshape(nb[2], 1 if dim == 2 else bs, nb[1], bs, nb[0], bs).any(axis=(1, 3, 5))
        blk_ok = allowed.reshape(nb[2], 1 if dim == 2 else bs, nb[1], bs, nb[0], bs).all(axis=(1, 3, 5))
        marked = blk_t & blk_ok
        if not marked.any():
            ok = np.argwhere(blk_ok)
            if ok.size == 0:
                raise ValueError(f"level {l} leaves no room for a properly nested level {l + 1}")
            c = ok[len(ok) // 2]
            marked[tuple(c)] = True
        mgs_l = max(bs, max_grid_size // 2)
        for lo, hi in cluster_blocks(marked, bs if dim == 3 else bs, mgs_l):
            flo = tuple(2 * lo[d] if d < dim else 0 for d in range(3))
            fhi = tuple(2 * hi[d] + 1 if d < dim else 0 for d in range(3))
            new.append((l + 1, flo, fhi))
    return new


__all__ = ["chop", "hierarchy", "box_states", "level0_geom", "composite_sum", "covered_mask_fn", "nstate",
           "regrid_boxes", "cluster_blocks"]

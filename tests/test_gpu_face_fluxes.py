"""Face fluxes of one box for the flux registers of a multi-level host (compas_b200_face_fluxes).

The reference's compute_dUdt_FV scales the face fluxes by the face areas and hands them to
FluxRegister::CrseInit(-dt_lev) / FineAdd(+dt_lev) (source/Class_Compressible_PhaseField.cpp:3433-3536).
The fused stage kernel keeps its fluxes in shared memory, so the per-box ABI recomputes them for the
registers. Checked here:
  * the raw fluxes are the ones the fused kernel used: their divergence, formed on the host in the
    kernel's order (x, then y, then z, divided by dx), reproduces compute_dUdt of the conservative
    components to the bit (plain FP64), and the mixed form's within round-off;
  * area scaling is the face area times the raw flux, bit for bit; the box-boundary mode writes the
    same boundary faces as the all-faces mode and nothing else;
  * a two-level step driven only through the per-box entry points (coarse and fine RK3 stages, the
    registers filled from these face fluxes with the RK3 stage weights, reflux, average-down) keeps
    the composite masses, momenta and total energy of a periodic domain to round-off, and fails to
    without the reflux.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import build_case

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _faces(torch, p, g, which=cb.FACES_ALL, area=True, U=None, fill=0.0):
    N, NC = cb.parm_nstate(p), cb.nc_terms(p)
    F = [torch.full(cb.face_shape(p, g, d, N), fill, dtype=torch.float64, device="cuda") for d in range(p.dim)]
    Fn = [torch.full(cb.face_shape(p, g, d, NC), fill, dtype=torch.float64, device="cuda") for d in range(p.dim)]
    cb.face_fluxes(p, g, U, F, Fn, which=which, area_scaled=area)
    torch.cuda.synchronize()
    return [f.cpu().numpy() for f in F], [f.cpu().numpy() for f in Fn]


def _divergence(F, p, g, mixed):
    """-(div F) in the fused kernel's order: (F_hi - F_lo)/dx_0, then + (F_hi - F_lo)/dx_1, ..."""
    acc = None
    for d in range(p.dim):
        f = F[d]
        if d == 0:
            df = f[:, :, :, 1:] - f[:, :, :, :-1]
        elif d == 1:
            df = f[:, :, 1:, :] - f[:, :, :-1, :]
        else:
            df = f[:, 1:, :, :] - f[:, :-1, :, :]
        t = df * (1.0 / g.dx[d]) if mixed else df / g.dx[d]
        acc = t if acc is None else acc + t
    return -acc


CASES = [
    ("bubble2d_weno5b", cases.shock_bubble, dict(nx=40, ny=24, scheme="WENO5B"), {}),
    ("droplet3d_six", cases.shock_droplet, dict(n=12), {}),
    ("triple_nphase_muscl", cases.triple_point, dict(m=6), {"FiniteVolume.Scheme": "MUSCL-MC"}),
    ("bubble2d_hll_weno3", cases.shock_bubble, dict(nx=40, ny=24, scheme="WENO3"), {"Physics.RiemannSolver": "HLL"}),
]


@pytest.mark.parametrize("name,fn,kw,extra", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_face_flux_divergence_is_the_fused_right_hand_side(name, fn, kw, extra, precision):
    import torch

    phys, dim, inputs, geom, U = fn(**kw)
    p = cb.make_parm(phys, dim, dict(inputs, **extra, **{"compas_b200.precision": precision}))
    g = cb.make_geom(**geom)
    Ud = _dev(torch, U)
    cb.FillPatch(p, g, Ud)
    dU = torch.zeros_like(Ud)
    cb.compute_dUdt_FV(p, g, Ud, dU)
    F, Fn = _faces(torch, p, g, area=False, U=Ud)
    mixed = precision == "mixed"
    div = _divergence(F, p, g, mixed)
    got = cb.valid_view(dU.cpu().numpy(), p, g)
    # conservative components: the partial densities and the momenta (every model), the total energy
    # (five-equation models); the others carry non-conservative terms as well
    if phys == cb.FIVEEQS:
        comps = list(range(2 + dim + 1))
    elif phys == cb.SIXEQS:
        comps = list(range(2 + dim))
    else:
        comps = list(range(p.nphase + dim + 1))
    for c in comps:
        if mixed:
            scale = max(float(np.abs(got[c]).max()), 1e-300)
            err = float(np.abs(div[c] - got[c]).max()) / scale
            assert err <= 1e-13, (c, err)
        else:
            np.testing.assert_array_equal(div[c], got[c], err_msg=f"component {c}")
    # area scaling: the face area times the raw flux, bit for bit
    Fa, Fna = _faces(torch, p, g, area=True, U=Ud)
    dx = list(g.dx)
    area = [dx[1] * (dx[2] if dim == 3 else 1.0), dx[0] * (dx[2] if dim == 3 else 1.0), dx[0] * dx[1]]
    for d in range(dim):
        np.testing.assert_array_equal(Fa[d], F[d] * area[d])
        np.testing.assert_array_equal(Fna[d], Fn[d] * area[d])


def test_boundary_mode_writes_the_boundary_faces_only():
    import torch

    p, g, U = build_case(cases.shock_droplet, n=10)
    Ud = _dev(torch, U)
    cb.FillPatch(p, g, Ud)
    F, Fn = _faces(torch, p, g, which=cb.FACES_ALL, U=Ud)
    B, Bn = _faces(torch, p, g, which=cb.FACES_BOUNDARY, U=Ud, fill=np.nan)
    for d in range(3):
        ax = 3 - d  # face arrays are (component, z, y, x)
        for arr_all, arr_b in ((F[d], B[d]), (Fn[d], Bn[d])):
            n = arr_all.shape[ax]
            for side in (0, n - 1):
                np.testing.assert_array_equal(np.take(arr_b, side, axis=ax), np.take(arr_all, side, axis=ax))
            inner = np.take(arr_b, list(range(1, n - 1)), axis=ax)
            assert np.isnan(inner).all()


def _inject(Uc_valid, lo, shape_f, ng):
    """Fine padded state (N, 1, ny+2ng, nx+2ng) by piecewise-constant injection from the coarse valid
    cells, the fine box's lower corner at coarse cell lo (2D)."""
    N = Uc_valid.shape[0]
    ny, nx = shape_f
    jf = np.arange(-ng, ny + ng)
    if_ = np.arange(-ng, nx + ng)
    jc = lo[1] + np.floor_divide(jf, 2)
    ic = lo[0] + np.floor_divide(if_, 2)
    out = np.empty((N, 1, ny + 2 * ng, nx + 2 * ng))
    out[:, 0] = Uc_valid[:, 0][:, jc][:, :, ic]
    return out


def _two_level_step(reflux, precision="fp64"):
    """One coarse step of a periodic 2D five-equation advected disc with a fine box (ratio 2) over its
    centre, the fine level subcycled twice, driven through the per-box entry points. Returns the
    relative change of the composite totals of the conservative components."""
    import torch

    n = 32
    phys, dim, inputs, geom, Uc = cases.advected_disc(n=n)
    inputs = dict(inputs, **{"compas_b200.precision": precision})
    p = cb.make_parm(phys, dim, inputs)
    gc = cb.make_geom(**geom)
    ng = gc.ng
    lo, nf = (8, 8), (16, 16)  # fine box: coarse cells [8, 24) x [8, 24) -> 32 x 32 fine cells
    gf = cb.make_geom((2 * nf[0], 2 * nf[1], 1), (gc.dx[0] / 2, gc.dx[1] / 2, 1.0), ng)
    N = cb.parm_nstate(p)
    Vc, Vf = gc.dx[0] * gc.dx[1], gf.dx[0] * gf.dx[1]
    cons = list(range(2 + dim + 1))  # masses, momenta, total energy
    Ucv = cb.valid_view(Uc, p, gc)
    Uf = _inject(Ucv, lo, (2 * nf[1], 2 * nf[0]), ng)
    cov = np.zeros((n, n), dtype=bool)
    cov[lo[1]:lo[1] + nf[1], lo[0]:lo[0] + nf[0]] = True

    def totals(Ucv_, Ufv_):
        return np.array([Ucv_[c, 0][~cov].sum() * Vc + Ufv_[c, 0].sum() * Vf for c in cons])

    t0 = totals(Ucv, cb.valid_view(Uf, p, gf))
    scale = np.array([np.abs(Ucv[c, 0]).sum() * Vc for c in cons])
    dt_c = 0.3 * gc.dx[0] / 1700.0
    W = (1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0)
    # registers on the coarse faces of the fine box boundary: x faces at i = 8 and 24 (rows 8..23),
    # y faces at j = 8 and 24 (columns 8..23)
    reg = {d: np.zeros((N, 2, nf[1 - d])) for d in range(2)}

    def rk3(pp, gg, Ud, dt, on_stage):
        dtd = torch.tensor([dt], dtype=torch.float64, device="cuda")
        U0 = Ud.clone()
        U1, U2 = torch.zeros_like(Ud), torch.zeros_like(Ud)
        ins, outs = (U0, U1, U2), (U1, U2, Ud)
        for s in range(3):
            on_stage(s, ins[s])
            cb.ThirdOrderSSPRK_stage(pp, gg, s, ins[s], U0, outs[s], dtd)
        torch.cuda.synchronize()

    # coarse level: periodic ghosts; CrseInit with -w dt_c on its faces at the fine box boundary
    Ucd = _dev(torch, Uc)

    def coarse_stage(s, Us):
        cb.FillPatch(p, gc, Us)
        F, _ = _faces(torch, p, gc, which=cb.FACES_ALL, U=Us)
        for side, i in enumerate((lo[0], lo[0] + nf[0])):
            reg[0][:, side] += -W[s] * dt_c * F[0][:, 0, lo[1]:lo[1] + nf[1], i]
        for side, j in enumerate((lo[1], lo[1] + nf[1])):
            reg[1][:, side] += -W[s] * dt_c * F[1][:, 0, j, lo[0]:lo[0] + nf[0]]

    rk3(p, gc, Ucd, dt_c, coarse_stage)
    # fine level: two substeps; ghosts by injection from the coarse start-of-step state (any ghost
    # values conserve the composite totals); FineAdd with +w dt_f, two fine faces per coarse face
    dt_f = dt_c / 2
    Ufd = _dev(torch, Uf)
    Uf_ghost_src = Uf.copy()

    def fine_stage(s, Us):
        a = Us.cpu().numpy()
        valid = cb.valid_view(a, p, gf).copy()
        a[:] = Uf_ghost_src
        cb.valid_view(a, p, gf)[:] = valid
        Us.copy_(torch.from_numpy(a).cuda())
        F, _ = _faces(torch, p, gf, which=cb.FACES_BOUNDARY, U=Us)
        for side, i in enumerate((0, 2 * nf[0])):
            f = F[0][:, 0, :, i]
            reg[0][:, side] += W[s] * dt_f * (f[:, 0::2] + f[:, 1::2])
        for side, j in enumerate((0, 2 * nf[1])):
            f = F[1][:, 0, j, :]
            reg[1][:, side] += W[s] * dt_f * (f[:, 0::2] + f[:, 1::2])

    for _ in range(2):
        rk3(p, gf, Ufd, dt_f, fine_stage)
    Ucv = cb.valid_view(Ucd.cpu().numpy(), p, gc).copy()
    Ufv = cb.valid_view(Ufd.cpu().numpy(), p, gf).copy()
    if reflux:
        # the cell on the low side of a face has it as its high face: -reg / V; high side: +reg / V
        for c in cons:
            Ucv[c, 0, lo[1]:lo[1] + nf[1], lo[0] - 1] -= reg[0][c, 0] / Vc
            Ucv[c, 0, lo[1]:lo[1] + nf[1], lo[0] + nf[0]] += reg[0][c, 1] / Vc
            Ucv[c, 0, lo[1] - 1, lo[0]:lo[0] + nf[0]] -= reg[1][c, 0] / Vc
            Ucv[c, 0, lo[1] + nf[1], lo[0]:lo[0] + nf[0]] += reg[1][c, 1] / Vc
    # average-down of the covered coarse cells
    avg = 0.25 * (Ufv[:, 0, 0::2, 0::2] + Ufv[:, 0, 1::2, 0::2] + Ufv[:, 0, 0::2, 1::2] + Ufv[:, 0, 1::2, 1::2])
    Ucv[:, 0, lo[1]:lo[1] + nf[1], lo[0]:lo[0] + nf[0]] = avg
    t1 = totals(Ucv, Ufv)
    return np.abs(t1 - t0) / scale


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_registers_from_face_fluxes_conserve_the_composite(precision):
    err = _two_level_step(True, precision)
    err_off = _two_level_step(False, precision)
    print(f"{precision}: composite conservation with reflux {err}, without {err_off}")
    assert np.all(err <= 1e-14), err
    # the test has teeth: skipping the reflux breaks conservation far above round-off
    assert np.max(err_off) > 1e3 * max(np.max(err), 1e-16), err_off


def test_rejects_thinc_and_bad_mode():
    import torch

    p, g, U = build_case(cases.advected_disc, n=16)
    Ud = _dev(torch, U)
    F = [torch.zeros(cb.face_shape(p, g, d, cb.parm_nstate(p)), dtype=torch.float64, device="cuda") for d in range(2)]
    with pytest.raises(cb.CompasError):
        cb.face_fluxes(p, g, Ud, F, which=7)
    pt = cb.make_parm(cb.FIVEEQS, 2, {"FiniteVolume.THINC": "1"})
    with pytest.raises(cb.CompasError):
        cb.face_fluxes(pt, g, Ud, F)

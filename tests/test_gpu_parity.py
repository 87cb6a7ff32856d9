"""Parity of the CUDA path (through the C ABI) with the CPU oracle on identical initial data.

The plain FP64 form evaluates the reference's formulas in the reference's order with FMA
contraction off, so the expected difference is zero; the asserted bound is the north star's
1e-11 relative L-infinity per field, and every test also reports the measured difference.
"""
import numpy as np
import pytest

import compas_b200 as cb
from compas_b200 import cases
from helpers import build_case, oracle_kind, rel_linf, run_gpu, run_oracle
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-11  # relative L-infinity per field (plain FP64 vs the reference CPU arithmetic)


def _cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _compare_steps(p, g, U, nsteps, use_graph=True):
    got, info, dts = run_gpu(p, g, U, nsteps, use_graph=use_graph)
    ref, t, dts_ref = run_oracle(p, g, U, nsteps)
    assert info.steps == len(dts_ref) == nsteps
    assert info.status == 0
    np.testing.assert_array_equal(dts, dts_ref)
    e = rel_linf(cb.valid_view(got, p, g), cb.valid_view(ref, p, g))
    print(f"{nsteps} steps, rel Linf per field vs {oracle_kind(p.physics, p.dim)} oracle: {e}")
    assert np.all(e <= TOL), e
    return e


def test_dudt_fiveeq_2d_matches_oracle():
    torch = _cuda()
    p, g, U = build_case(cases.advected_disc, n=64)
    o = Oracle(oracle_kind(p.physics, p.dim), p, g)
    Uf = U.copy()
    o.fill_ghosts(Uf)
    dU_ref, cmax_ref = o.compute_dudt(Uf)
    dev = torch.from_numpy(Uf).cuda()
    dU = torch.zeros_like(dev)
    cm = torch.zeros(1, dtype=torch.float64, device="cuda")
    cb.compute_dUdt_FV(p, g, dev, dU, cmax=cm)
    torch.cuda.synchronize()
    a = cb.valid_view(dU.cpu().numpy(), p, g)
    r = cb.valid_view(dU_ref, p, g)
    assert float(cm.item()) == cmax_ref
    e = rel_linf(a, r)
    print("dUdt rel Linf:", e, "bitwise equal:", np.array_equal(a, r))
    assert np.all(e <= TOL)


def test_fill_boundary_matches_oracle_all_codes():
    torch = _cuda()
    rng = np.random.default_rng(0)
    for dim, phys in ((2, cb.FIVEEQS), (3, cb.SIXEQS)):
        n = (11, 9, 7)[:dim] + ((1,) if dim == 2 else ())
        for lo, hi in (((2, 3, 4), (5, 2, 3)), ((0, 5, 2), (0, 4, 3)), ((4, 0, 5), (2, 0, 4))):
            p = cb.make_parm(phys, dim, {})
            g = cb.make_geom(n, (0.1, 0.1, 0.1), 3, lo, hi)
            U = rng.standard_normal(cb.padded_shape(p, g))
            ref = U.copy()
            Oracle(oracle_kind(phys, dim), p, g).fill_ghosts(ref)
            dev = torch.from_numpy(U).cuda()
            cb.FillPatch(p, g, dev)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(dev.cpu().numpy(), ref)


def test_advected_disc_64_20_steps():
    p, g, U = build_case(cases.advected_disc, n=64)
    _compare_steps(p, g, U, 20)


def test_advected_disc_128_200_steps_config():
    """The CPU-runnable configuration: 128x128, 200 steps, WENO5 + HLLC + TVD-RK3, cfl 0.5."""
    p, g, U = build_case(cases.advected_disc, n=128)
    got, info, dts = run_gpu(p, g, U, 200)
    ref, t, dts_ref = run_oracle(p, g, U, 200)
    a, r = cb.valid_view(got, p, g), cb.valid_view(ref, p, g)
    e = rel_linf(a, r)
    print("config advected disc 128^2 x 200 steps: rel Linf per field", e, "bitwise:", np.array_equal(a, r))
    assert np.all(e <= TOL)
    assert info.t == t
    # conservation of the masses, momenta and total energy (periodic box) to round-off
    V0 = cb.valid_view(U, p, g)
    for c in range(5):
        s0, s1 = float(V0[c].sum()), float(a[c].sum())
        assert abs(s1 - s0) <= 1e-12 * max(abs(s0), float(np.abs(V0[c]).sum())), (c, s0, s1)


def test_graph_and_stream_paths_identical():
    p, g, U = build_case(cases.advected_disc, n=48)
    a, ia, _ = run_gpu(p, g, U, 5, use_graph=True)
    b, ib, _ = run_gpu(p, g, U, 5, use_graph=False)
    np.testing.assert_array_equal(a, b)
    assert ia.t == ib.t


def test_odd_sizes_partial_tiles_2d():
    p, g, U = build_case(cases.shock_bubble, nx=37, ny=23, scheme="WENO5")
    _compare_steps(p, g, U, 6)


def test_sixeq_3d_shock_droplet_relaxation():
    p, g, U = build_case(cases.shock_droplet, n=24)
    _compare_steps(p, g, U, 4)


def test_sixeq_3d_odd_box():
    phys, dim, inputs, geom, U = cases.shock_droplet(n=12)
    p = cb.make_parm(phys, dim, inputs)
    # a non-cubic box with partial tiles in every direction, mixed wall codes
    geom["n"] = (13, 11, 9)
    geom["lo_bc"], geom["hi_bc"] = (2, 3, 5), (4, 2, 2)
    g = cb.make_geom(**geom)
    rng = np.random.default_rng(3)
    # a smooth perturbation of a uniform two-phase mixture
    Ug = np.zeros(cb.padded_shape(p, g))
    V = cb.valid_view(Ug, p, g)
    a1 = 0.3 + 0.2 * rng.random(V[0].shape)
    a2 = 1 - a1
    A1, A2, B2 = p.A1, p.A2, p.B2
    pres = 1e5 * (1 + 0.1 * rng.random(V[0].shape))
    V[0], V[1] = a1 * 1.2, a2 * 1000.0
    rho = V[0] + V[1]
    vel = [10 * rng.standard_normal(V[0].shape) for _ in range(3)]
    for d in range(3):
        V[2 + d] = rho * vel[d]
    ke = sum(v * v for v in vel)
    V[5] = a1 * (A1 * pres) + 0.5 * V[0] * ke
    V[6] = a2 * (A2 * pres + B2) + 0.5 * V[1] * ke
    V[7] = a1
    _compare_steps(p, g, Ug, 3)


def test_fiveeq_3d_and_sixeq_2d():
    phys, dim, inputs, geom, U = cases.shock_droplet(n=16)
    # the same droplet with the five-equation model in 3D
    inputs5 = dict(inputs)
    inputs5.pop("Physics.pressure_relaxation")
    p5 = cb.make_parm(cb.FIVEEQS, 3, inputs5)
    g5 = cb.make_geom(**geom)
    V6 = cb.valid_view(U, cb.make_parm(phys, dim, inputs), g5)
    U5 = np.zeros(cb.padded_shape(p5, g5))
    V5 = cb.valid_view(U5, p5, g5)
    V5[0:5] = V6[0:5]
    V5[5] = V6[5] + V6[6]
    V5[6] = V6[7]
    _compare_steps(p5, g5, U5, 3)
    p6, g6, U6 = build_case(cases.advected_disc, n=32)
    # six-equation 2D version of the advected disc
    p6 = cb.make_parm(cb.SIXEQS, 2, {"prob.EOS.gamma_1": 1.4, "prob.EOS.gamma_2": 4.4, "prob.EOS.pinf_2": 6e8,
                                     "Physics.pressure_relaxation": 1, "run.cfl": 0.5})
    Ux = np.zeros(cb.padded_shape(p6, g6))
    Vs = cb.valid_view(U6, cb.make_parm(cb.FIVEEQS, 2, {}), g6)
    Vx = cb.valid_view(Ux, p6, g6)
    a1 = Vs[5]
    Vx[0:4] = Vs[0:4]
    rho = Vs[0] + Vs[1]
    ke = 0.5 * (Vs[2] ** 2 + Vs[3] ** 2) / rho
    Vx[4] = a1 * (p6.A1 * 1e5) + ke * Vs[0] / rho
    Vx[5] = (1 - a1) * (p6.A2 * 1e5 + p6.B2) + ke * Vs[1] / rho
    Vx[6] = a1
    _compare_steps(p6, g6, Ux, 5)


def test_status_word_reports_nan_without_fault():
    p, g, U = build_case(cases.advected_disc, n=32)
    V = cb.valid_view(U, p, g)
    V[4, 0, 10, 10] = np.nan  # a NaN energy: the kernels must flag it and keep the context usable
    lv = cb.Level(p, g)
    lv.upload(U)
    lv.advance(1, use_graph=False)
    info = lv.sync(check=False)
    assert info.status != 0
    lv.close()
    # the context is still usable afterwards
    p2, g2, U2 = build_case(cases.advected_disc, n=32)
    got, info2, _ = run_gpu(p2, g2, U2, 1)
    assert info2.status == 0


def test_weno5b_fiveeq_2d_shock_bubble_walls_outflow():
    """WENO5B (bounded masses and volume fractions) on the shock-bubble with reflective top/bottom
    and outflow left/right, the configuration of the 2D shock-helium-bubble at reduced size."""
    p, g, U = build_case(cases.shock_bubble, nx=96, ny=48, scheme="WENO5B")
    _compare_steps(p, g, U, 10)


def test_weno5b_sixeq_3d():
    phys, dim, inputs, geom, U = cases.shock_droplet(n=20)
    inputs["FiniteVolume.Scheme"] = "WENO5B"
    p = cb.make_parm(phys, dim, inputs)
    g = cb.make_geom(**geom)
    _compare_steps(p, g, U, 3)

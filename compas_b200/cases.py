"""Initial data of the workloads: cell averages of the conserved state by 4-point Gauss-Legendre
quadrature per direction (include/InitData.H:19-290, run.QuadratureIC = 1), or cell-centre samples.

Every case returns (parm inputs, geometry kwargs, padded state) so that the CUDA path and the CPU
oracles start from the same bits. Arrays follow the padded Array4 layout (N, PZ, PY, PX) with zero
ghosts. `xp` may be numpy (default) or torch (then `device` places the arrays; FP64 throughout).
"""
from __future__ import annotations

import math

import numpy as np

from . import FIVEEQS, FIVEEQS_NPHASE, SIXEQS, SIXEQS_IE_NPHASE, nstate

# Gauss-Legendre nodes and weights on [-1, 1] (4 points, exact to degree 7)
_GL_X, _GL_W = np.polynomial.legendre.leggauss(4)


def eos_AB(gamma: float, pinf: float) -> tuple:
    """Stiffened-gas partial-form coefficients A = 1/(gamma-1), B = gamma pinf/(gamma-1) (source/Parm.cpp:126-130)."""
    return 1.0 / (gamma - 1.0), gamma * pinf / (gamma - 1.0)


def shock_state(Ma: float, u0: float, p0: float, rho0: float, gamma: float, pinf: float) -> tuple:
    """Post-shock (rho, u, p) behind a right-running normal shock of Mach Ma into a stiffened gas at
    rest state (rho0, u0, p0): the Rankine-Hugoniot relations written in the shifted pressure
    P = p + pinf, the same relations include/PhysicsFunctions.H:15-35 evaluates."""
    P0 = p0 + pinf
    c0 = math.sqrt(gamma * P0 / rho0)
    P1 = P0 * (1.0 + 2.0 * gamma / (gamma + 1.0) * (Ma * Ma - 1.0))
    r = P1 / P0
    mu = (gamma + 1.0) / (gamma - 1.0)
    rho1 = rho0 * (mu * r + 1.0) / (mu + r)
    # jump in velocity from mass conservation across the shock moving at u0 + Ma c0
    s = u0 + Ma * c0
    u1 = s - rho0 * (s - u0) / rho1
    return rho1, u1, P1 - pinf


def _xp_of(xp):
    if xp is None:
        return np
    return xp


def _zeros(xp, shape, device):
    if xp is np:
        return np.zeros(shape, dtype=np.float64)
    return xp.zeros(shape, dtype=xp.float64, device=device)


def _cons_from_prims(physics, dim, ar1, ar2, vel, p, alpha1, A, B, xp):
    """Conserved components from phase masses, velocity, a common pressure and alpha1 (stiffened gas)."""
    alpha2 = 1.0 - alpha1
    rho = ar1 + ar2
    ke = 0.0
    for v in vel:
        ke = ke + v * v
    out = [ar1, ar2] + [rho * v for v in vel]
    if physics == FIVEEQS:
        rho_e = alpha1 * (A[0] * p + B[0]) + alpha2 * (A[1] * p + B[1])
        out += [rho_e + 0.5 * rho * ke, alpha1]
    else:
        e1 = alpha1 * (A[0] * p + B[0]) + 0.5 * ar1 * ke
        e2 = alpha2 * (A[1] * p + B[1]) + 0.5 * ar2 * ke
        out += [e1, e2, alpha1]
    return out


def _average(physics, dim, n, dx, lo, pointwise, ng, quadrature, xp, device, nphase=2):
    """Padded state whose valid cells hold the cell averages of pointwise(x, y, z) -> list of N arrays."""
    N = nstate(physics, dim, nphase)
    gz = ng if dim == 3 else 0
    nz = n[2] if dim == 3 else 1
    shape = (N, nz + 2 * gz, n[1] + 2 * ng, n[0] + 2 * ng)
    U = _zeros(xp, shape, device)

    def ar(m, d):
        a = np.arange(m, dtype=np.float64) if xp is np else xp.arange(m, dtype=xp.float64, device=device)
        return lo[d] + (a + 0.5) * dx[d]

    xc = ar(n[0], 0)[None, None, :]
    yc = ar(n[1], 1)[None, :, None]
    zc = ar(nz, 2)[:, None, None] if dim == 3 else (xc * 0.0 + 0.0)
    if quadrature:
        nodes = list(zip(_GL_X, _GL_W))
        zn = nodes if dim == 3 else [(0.0, 2.0)]
        acc = None
        norm = 1.0 / (2 ** dim)
        for rz, wz in zn:
            for ry, wy in nodes:
                for rx, wx in nodes:
                    w = wx * wy * (wz if dim == 3 else 1.0)
                    vals = pointwise(xc + 0.5 * dx[0] * rx, yc + 0.5 * dx[1] * ry,
                                     zc + (0.5 * dx[2] * rz if dim == 3 else 0.0))
                    if acc is None:
                        acc = [w * v for v in vals]
                    else:
                        acc = [a + w * v for a, v in zip(acc, vals)]
        vals = [a * norm for a in acc]
    else:
        vals = pointwise(xc, yc, zc)
    for c in range(N):
        v = vals[c]
        if not hasattr(v, "shape") or v.shape != (nz, n[1], n[0]):
            v = v + 0.0 * xc * yc * (zc if dim == 3 else 1.0)
        U[c, gz:gz + nz, ng:ng + n[1], ng:ng + n[0]] = v
    return U


def _tanh(xp, x):
    return np.tanh(x) if xp is np else xp.tanh(x)


def _clip(xp, x, lo, hi):
    return np.clip(x, lo, hi) if xp is np else xp.clamp(x, lo, hi)


def _sqrt(xp, x):
    return np.sqrt(x) if xp is np else xp.sqrt(x)


def advected_disc(n=128, ng=3, quadrature=True, xp=None, device=None):
    """2D FIVEEQS advected interface on the periodic unit square: phase-2 disc of radius 0.25 at
    (0.5, 0.5), alpha2 = 0.5(1 + tanh((0.25 - r)/(2 dx))) clipped to [1e-6, 1 - 1e-6]; phase 1 ideal
    gas (gamma 1.4, rho 1), phase 2 stiffened gas (gamma 4.4, pinf 6e8, rho 1000); p = 1e5, u = v = 1.
    WENO5 + HLLC + TVD-RK3, cfl 0.5."""
    xp = _xp_of(xp)
    dim, physics = 2, FIVEEQS
    dx = (1.0 / n, 1.0 / n, 1.0)
    g1, g2, pinf2 = 1.4, 4.4, 6e8
    A = (1.0 / (g1 - 1.0), 1.0 / (g2 - 1.0))
    B = (0.0, g2 * pinf2 / (g2 - 1.0))

    def pw(x, y, z):
        r = _sqrt(xp, (x - 0.5) ** 2 + (y - 0.5) ** 2)
        a2 = _clip(xp, 0.5 * (1.0 + _tanh(xp, (0.25 - r) / (2.0 * dx[0]))), 1e-6, 1.0 - 1e-6)
        a1 = 1.0 - a2
        return _cons_from_prims(physics, dim, a1 * 1.0, a2 * 1000.0, [x * 0 + 1.0, y * 0 + 1.0], 1e5, a1, A, B, xp)

    inputs = {"FiniteVolume.Scheme": "WENO5", "Physics.RiemannSolver": "HLLC", "prob.EOS.EOS": 1,
              "prob.EOS.gamma_1": g1, "prob.EOS.gamma_2": g2, "prob.EOS.pinf_1": 0.0, "prob.EOS.pinf_2": pinf2,
              "run.cfl": 0.5}
    geom = dict(n=(n, n, 1), dx=dx, ng=ng, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    U = _average(physics, dim, (n, n, 1), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device)
    return physics, dim, inputs, geom, U


def advected_interface(n=32, dim=3, physics=SIXEQS, ng=3, quadrature=True, xp=None, device=None, relaxation=1):
    """The advected interface of advected_disc for either model in 2D or 3D: phase-2 disc / sphere of
    radius 0.25 at the centre of the periodic unit square / cube, the same phases, p = 1e5 and
    velocity 1 along every axis; for SIXEQS the pressure relaxation after every stage."""
    xp = _xp_of(xp)
    dx = (1.0 / n, 1.0 / n, 1.0 / n if dim == 3 else 1.0)
    g1, g2, pinf2 = 1.4, 4.4, 6e8
    A = (1.0 / (g1 - 1.0), 1.0 / (g2 - 1.0))
    B = (0.0, g2 * pinf2 / (g2 - 1.0))

    def pw(x, y, z):
        r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2 + ((z - 0.5) ** 2 if dim == 3 else 0.0)
        a2 = _clip(xp, 0.5 * (1.0 + _tanh(xp, (0.25 - _sqrt(xp, r2)) / (2.0 * dx[0]))), 1e-6, 1.0 - 1e-6)
        a1 = 1.0 - a2
        vel = [x * 0 + 1.0, y * 0 + 1.0] + ([z * 0 + 1.0] if dim == 3 else [])
        return _cons_from_prims(physics, dim, a1 * 1.0, a2 * 1000.0, vel, 1e5, a1, A, B, xp)

    inputs = {"FiniteVolume.Scheme": "WENO5", "Physics.RiemannSolver": "HLLC", "prob.EOS.EOS": 1,
              "prob.EOS.gamma_1": g1, "prob.EOS.gamma_2": g2, "prob.EOS.pinf_1": 0.0, "prob.EOS.pinf_2": pinf2,
              "run.cfl": 0.5}
    if physics == SIXEQS:
        inputs["Physics.pressure_relaxation"] = relaxation
    nz = n if dim == 3 else 1
    geom = dict(n=(n, n, nz), dx=dx, ng=ng, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    U = _average(physics, dim, (n, n, nz), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device)
    return physics, dim, inputs, geom, U


def shock_bubble(nx=2048, ny=1024, ng=3, quadrature=True, xp=None, device=None, Ma=1.22, rho_b=0.138,
                 gamma_b=1.648, radius=0.25, center=(0.6, 0.5), scheme="WENO5B", length=2.0):
    """2D FIVEEQS shock-helium-bubble on [0,length]x[0,1] (default [0,2]x[0,1]): air (phase 1, gamma
    1.4, rho 1, p 1), helium bubble (phase 2) with a tanh interface of width 2 dx, a Mach-Ma shock at
    x = 0.2 with the Rankine-Hugoniot post-shock state on its left; reflective top/bottom (code 4),
    outflow left/right (code 2)."""
    xp = _xp_of(xp)
    dim, physics = 2, FIVEEQS
    L = float(length)
    dx = (L / nx, 1.0 / ny, 1.0)
    g1, g2 = 1.4, gamma_b
    A = (1.0 / (g1 - 1.0), 1.0 / (g2 - 1.0))
    B = (0.0, 0.0)
    rs, us, ps = shock_state(Ma, 0.0, 1.0, 1.0, g1, 0.0)
    eps = 1e-6

    def pw(x, y, z):
        r = _sqrt(xp, (x - center[0]) ** 2 + (y - center[1]) ** 2)
        a2 = _clip(xp, 0.5 * (1.0 + _tanh(xp, (radius - r) / (2.0 * dx[0]))), eps, 1.0 - eps)
        a1 = 1.0 - a2
        post = (x < 0.2) * 1.0
        rho1 = 1.0 + post * (rs - 1.0)
        u = post * us
        p = 1.0 + post * (ps - 1.0)
        return _cons_from_prims(physics, dim, a1 * rho1, a2 * rho_b, [u, y * 0.0], p, a1, A, B, xp)

    inputs = {"FiniteVolume.Scheme": scheme, "Physics.RiemannSolver": "HLLC", "prob.EOS.EOS": 1,
              "prob.EOS.gamma_1": g1, "prob.EOS.gamma_2": g2, "run.cfl": 0.5}
    geom = dict(n=(nx, ny, 1), dx=dx, ng=ng, lo_bc=(2, 4, 0), hi_bc=(2, 4, 0))
    U = _average(physics, dim, (nx, ny, 1), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device)
    return physics, dim, inputs, geom, U


def _box_level_set_2d(xp, x, y, xmin, ymin, xmax, ymax):
    """Signed distance to the rectangle [xmin, xmax] x [ymin, ymax], negative inside (the triple-point
    problem's boxLevelSet2D, exec/TriplePoint-5Eq-N/prob/ProblemICBC.H:15-34)."""
    cx, cy = 0.5 * (xmin + xmax), 0.5 * (ymin + ymax)
    hx, hy = 0.5 * (xmax - xmin), 0.5 * (ymax - ymin)
    ax = xp.abs(x - cx) if xp is not np else np.abs(x - cx)
    ay = xp.abs(y - cy) if xp is not np else np.abs(y - cy)
    dx_, dy_ = ax - hx, ay - hy
    mx = (dx_ > 0.0) * dx_
    my = (dy_ > 0.0) * dy_
    outside = _sqrt(xp, mx * mx + my * my)
    big = xp.maximum(dx_, dy_) if xp is not np else np.maximum(dx_, dy_)
    inside = (big < 0.0) * big
    return outside + inside


# Triple-point material states (x < 1: driver; x > 1, y < 1.5: lower right; x > 1, y > 1.5: upper
# right), phase order of exec/TriplePoint-5Eq-N/prob/ProblemICBC.H (phase 1 lower right, phase 2
# driver, phase 3 upper right). TRIPLE_POINT_GAMMAS is the workload's gamma of each phase (driver and
# lower right 1.5, upper right 1.4); the reference example's inputs use (1.4, 1.5, 1.5).
TRIPLE_POINT_RHO = (1.0, 1.0, 0.125)
TRIPLE_POINT_P = (0.1, 1.0, 0.1)
TRIPLE_POINT_GAMMAS = (1.5, 1.5, 1.4)
TRIPLE_POINT_REFERENCE_GAMMAS = (1.4, 1.5, 1.5)


def triple_point(m=32, ng=3, quadrature=True, xp=None, device=None, gammas=TRIPLE_POINT_GAMMAS, eta=0.0,
                 scheme="WENO5"):
    """2D FIVEEQS_NPHASE (NPHASE = 3) triple point on [0,7] x [0,3] with 7m x 3m square cells, gases at
    rest, reflecting walls (code 4) on every side, HLLC, source term 0, cfl 0.4, no change limiter
    (the reference example's run keys). Volume fractions 0.5(1 + tanh(psi/(sqrt(2) eta))(1 - 1e-12))
    of the two rectangle level sets, material 3 the remainder, normalised; eta = 0 gives the sharp
    interfaces of the example (they lie on cell faces when m is a multiple of 2), pressure mixed by
    volume fraction; the reference's initial_condition (ProblemICBC.H:36-105)."""
    xp = _xp_of(xp)
    dim, physics, nphase = 2, FIVEEQS_NPHASE, 3
    nx, ny = 7 * m, 3 * m
    dx = (7.0 / nx, 3.0 / ny, 1.0)
    A = [1.0 / (g - 1.0) for g in gammas]
    eps = 1.0e-12

    def tanh_scaled(psi):
        if eta == 0.0:
            return (psi > 0.0) * 1.0 - (psi < 0.0) * 1.0
        return _tanh(xp, psi / (math.sqrt(2.0) * eta))

    def pw(x, y, z):
        psi0 = -_box_level_set_2d(xp, x, y, 1.0, -1.0, 8.0, 1.5)
        psi1 = -_box_level_set_2d(xp, x, y, -1.0, -1.0, 1.0, 4.0)
        a0 = 0.5 * (1.0 + tanh_scaled(psi0) * (1.0 - eps))
        a1 = 0.5 * (1.0 + tanh_scaled(psi1) * (1.0 - eps))
        a2 = 1 - a0 - a1
        ssum = (0.0 + a0) + a1
        ssum = ssum + a2
        al = [a0 / ssum, a1 / ssum, a2 / ssum]
        P = 0.0
        for k in range(nphase):
            P = P + al[k] * TRIPLE_POINT_P[k]
        ar = [al[k] * TRIPLE_POINT_RHO[k] for k in range(nphase)]
        rho = 0.0
        for k in range(nphase):
            rho = rho + ar[k]
        AP = 0.0
        for k in range(nphase):
            AP = AP + al[k] * A[k]
        rho_e = (AP * P + 0.0) + 0.0  # ideal gases: B_k = D_k = 0
        zero = x * 0.0 + y * 0.0
        return ar + [rho * zero, rho * zero, rho_e + (0.5 * rho) * (zero * zero + zero * zero)] + al

    inputs = {"FiniteVolume.Scheme": scheme, "Physics.RiemannSolver": "HLLC", "Physics.source_term": 0,
              "prob.EOS.EOS": 1, "prob.EOS.gamma": list(gammas), "prob.EOS.pinf": [0.0] * nphase,
              "run.cfl": 0.4, "run.timestep_change_limiter": 0}
    geom = dict(n=(nx, ny, 1), dx=dx, ng=ng, lo_bc=(4, 4, 0), hi_bc=(4, 4, 0))
    U = _average(physics, dim, (nx, ny, 1), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device, nphase=nphase)
    return physics, dim, inputs, geom, U


def nphase_bubbles(n=32, nphase=3, dim=2, ng=3, quadrature=True, xp=None, device=None, source_term=0,
                   eos=1, velocity=1.0):
    """FIVEEQS_NPHASE advected interfaces on the periodic unit square / cube: phase k < nphase - 1
    fills a disc (sphere) of radius 0.15 centred at (0.3 + 0.4 (k % 2), 0.3 + 0.4 (k // 2 % 2), 0.5)
    with a tanh profile of width 2 dx, the last phase takes the remainder; volume fractions clipped
    to [1e-6, 1] and normalised. Phases alternate between an ideal gas (gamma 1.4, rho 1) and a
    stiffened liquid (gamma 4.4, pinf 6e8, rho 1000; with eos = 3 also NASG covolume 1e-4 and q 0);
    uniform pressure 1e5 and velocity `velocity` along every axis. WENO5 + HLLC, cfl 0.5."""
    xp = _xp_of(xp)
    physics = FIVEEQS_NPHASE
    dx = (1.0 / n, 1.0 / n, 1.0 / n if dim == 3 else 1.0)
    gam = [1.4 if k % 2 == 0 else 4.4 for k in range(nphase)]
    pinf = [0.0 if k % 2 == 0 else 6e8 for k in range(nphase)]
    rho0 = [1.0 if k % 2 == 0 else 1000.0 for k in range(nphase)]
    bcov = [0.0 if k % 2 == 0 else 1e-4 for k in range(nphase)] if eos == 3 else [0.0] * nphase
    A = [1.0 / (g - 1.0) for g in gam]
    B = [gam[k] * pinf[k] / (gam[k] - 1.0) for k in range(nphase)]
    p0 = 1e5

    def pw(x, y, z):
        al = []
        rest = 1.0
        for k in range(nphase - 1):
            cx, cy = 0.3 + 0.4 * (k % 2), 0.3 + 0.4 * ((k // 2) % 2)
            r2 = (x - cx) ** 2 + (y - cy) ** 2 + ((z - 0.5) ** 2 if dim == 3 else 0.0)
            a = _clip(xp, 0.5 * (1.0 + _tanh(xp, (0.15 - _sqrt(xp, r2)) / (2.0 * dx[0]))), 1e-6, 1.0)
            al.append(a)
            rest = rest - a
        al.append(_clip(xp, rest, 1e-6, 1.0))
        ssum = 0.0
        for a in al:
            ssum = ssum + a
        al = [a / ssum for a in al]
        ar = [al[k] * rho0[k] for k in range(nphase)]
        rho = 0.0
        for v in ar:
            rho = rho + v
        rho_e = 0.0
        for k in range(nphase):
            phi = al[k] - bcov[k] * ar[k]
            rho_e = rho_e + phi * (A[k] * p0 + B[k])
        vel = [x * 0 + velocity, y * 0 + velocity] + ([z * 0 + velocity] if dim == 3 else [])
        ke = 0.0
        for v in vel:
            ke = ke + v * v
        return ar + [rho * v for v in vel] + [rho_e + 0.5 * rho * ke] + al

    inputs = {"FiniteVolume.Scheme": "WENO5", "Physics.RiemannSolver": "HLLC", "Physics.source_term": source_term,
              "prob.EOS.EOS": eos, "prob.EOS.gamma": gam, "prob.EOS.pinf": pinf, "run.cfl": 0.5}
    if eos == 3:
        inputs["prob.EOS.b"] = bcov
        inputs["prob.EOS.q"] = [0.0] * nphase
    nz = n if dim == 3 else 1
    geom = dict(n=(n, n, nz), dx=dx, ng=ng, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0))
    U = _average(physics, dim, (n, n, nz), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device, nphase=nphase)
    return physics, dim, inputs, geom, U


def sixn_shock_bubbles(n=32, nphase=2, dim=2, ng=3, quadrature=True, xp=None, device=None, eos=1,
                       relaxation=1, Ma=1.1, dp=0.0, scheme="MUSCL", riemann="HLLC", trace=0.0):
    """SIXEQS_IE_NPHASE shock-bubble interaction after exec/ShockBubble-WaterAir-6Eq-Nphase (water
    and air, pressures scaled by P0 = 101325 Pa and densities by 1000 kg/m^3), on [0, 2] x [0, 1]
    (x [0, 1] in 3D) with n cells per unit length: water (phase 0, gamma 4.4, pinf 6e8 / P0, rho 1)
    at p = 1 with a Mach-Ma water shock at x = 0.25 (Rankine-Hugoniot state behind it); an air bubble
    (phase 1, gamma 1.4, rho 0.001) of radius 0.2 at (0.7, 0.5[, 0.5]); with nphase = 3 a helium
    bubble (phase 2, gamma 1.667, rho 1.66e-4) of radius 0.15 at (1.3, 0.5[, 0.5]). Every phase
    keeps a volume fraction of at least 1e-6 (tanh interfaces of width 2 dx, normalised). dp > 0
    puts the phases out of pressure equilibrium (phase k at p (1 + dp k)), so that the relaxation
    after each stage has work. eos = 3 adds a NASG covolume (b = 1e-4 for water, q 0). Outflow in x,
    symmetry at y = 0, outflow at y = 1, periodic in z. Default MUSCL + HLLC with pressure
    relaxation, cfl 0.3 (the example's inputs)."""
    xp = _xp_of(xp)
    physics = SIXEQS_IE_NPHASE
    h = 1.0 / n
    dx = (h, h, h if dim == 3 else 1.0)
    P0 = 101325.0
    gam = [4.4, 1.4, 1.667][:nphase]
    pinf = [6.0e8 / P0, 0.0, 0.0][:nphase]
    rho0 = [1.0, 0.001, 1.66e-4][:nphase]
    bcov = ([1e-4] + [0.0] * (nphase - 1)) if eos == 3 else [0.0] * nphase
    A = [1.0 / (g - 1.0) for g in gam]
    B = [gam[k] * pinf[k] / (gam[k] - 1.0) for k in range(nphase)]
    rs, us, ps = shock_state(Ma, 0.0, 1.0, rho0[0], gam[0], pinf[0])
    centres = [(0.7, 0.2), (1.3, 0.15)][:nphase - 1]

    def pw(x, y, z):
        post = (x < 0.25) * 1.0
        al = [None] * nphase
        rest = 1.0
        for k, (cx, rad) in enumerate(centres):
            r2 = (x - cx) ** 2 + (y - 0.5) ** 2 + ((z - 0.5) ** 2 if dim == 3 else 0.0)
            a = _clip(xp, 0.5 * (1.0 + _tanh(xp, (rad - _sqrt(xp, r2)) / (2.0 * h))), 1e-6, 1.0)
            al[k + 1] = a
            rest = rest - a
        al[0] = _clip(xp, rest, 1e-6, 1.0)
        ssum = 0.0
        for a in al:
            ssum = ssum + a
        al = [a / ssum for a in al]
        rho_w = rho0[0] + post * (rs - rho0[0])
        dens = [rho_w] + rho0[1:]
        ar = [al[k] * dens[k] for k in range(nphase)]
        rho = 0.0
        for v in ar:
            rho = rho + v
        u = post * us
        p = 1.0 + post * (ps - 1.0)
        vel = [u, y * 0.0] + ([z * 0.0] if dim == 3 else [])
        ke = 0.0
        for v in vel:
            ke = ke + v * v
        are = []
        rho_e = 0.0
        for k in range(nphase):
            pk = p * (1.0 + dp * k)
            xi = 1.0 - bcov[k] * dens[k]
            e_k = (A[k] * xi) * (al[k] * pk) + (xi * al[k]) * B[k]
            are.append(e_k)
            rho_e = rho_e + e_k
        return al + ar + are + [rho * v for v in vel] + [rho_e + 0.5 * rho * ke]

    inputs = {"FiniteVolume.Scheme": scheme, "Physics.RiemannSolver": riemann, "prob.EOS.EOS": eos,
              "prob.EOS.gamma": gam, "prob.EOS.pinf": pinf, "Physics.pressure_relaxation": relaxation,
              "Physics.pressure_relaxation_trace": trace, "run.cfl": 0.3}
    if eos == 3:
        inputs["prob.EOS.b"] = bcov
        inputs["prob.EOS.q"] = [0.0] * nphase
    nx, ny, nz = 2 * n, n, (n if dim == 3 else 1)
    geom = dict(n=(nx, ny, nz), dx=dx, ng=ng, lo_bc=(2, 3, 0), hi_bc=(2, 2, 0))
    U = _average(physics, dim, (nx, ny, nz), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device, nphase=nphase)
    return physics, dim, inputs, geom, U


def shock_droplet(n=256, ng=3, quadrature=True, xp=None, device=None, Ma=2.4, relaxation=1):
    """3D SIXEQS shock-droplet in the unit cube: water droplet (phase 2, stiffened gas gamma 6.12,
    pinf 3.43e8, rho 1000) of radius 0.1 at the centre, air (phase 1, gamma 1.4, rho 1.2, p 1e5), a
    Mach-Ma air shock at x = 0.2 with the Rankine-Hugoniot state on its left; tanh interface of
    width 2 dx clipped to [1e-6, 1 - 1e-6]; outflow (code 2) on all faces; pressure relaxation
    after every stage. WENO5 + HLLC + TVD-RK3."""
    xp = _xp_of(xp)
    dim, physics = 3, SIXEQS
    dx = (1.0 / n, 1.0 / n, 1.0 / n)
    g1, g2, pinf2 = 1.4, 6.12, 3.43e8
    A = (1.0 / (g1 - 1.0), 1.0 / (g2 - 1.0))
    B = (0.0, g2 * pinf2 / (g2 - 1.0))
    p0, rho_air = 1e5, 1.2
    rs, us, ps = shock_state(Ma, 0.0, p0, rho_air, g1, 0.0)
    eps = 1e-6

    def pw(x, y, z):
        r = _sqrt(xp, (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
        a2 = _clip(xp, 0.5 * (1.0 + _tanh(xp, (0.1 - r) / (2.0 * dx[0]))), eps, 1.0 - eps)
        a1 = 1.0 - a2
        post = (x < 0.2) * 1.0
        rho1 = rho_air + post * (rs - rho_air)
        u = post * us
        p = p0 + post * (ps - p0)
        return _cons_from_prims(physics, dim, a1 * rho1, a2 * 1000.0, [u, y * 0.0, z * 0.0], p, a1, A, B, xp)

    inputs = {"FiniteVolume.Scheme": "WENO5", "Physics.RiemannSolver": "HLLC", "prob.EOS.EOS": 1,
              "prob.EOS.gamma_1": g1, "prob.EOS.gamma_2": g2, "prob.EOS.pinf_2": pinf2,
              "Physics.pressure_relaxation": relaxation, "run.cfl": 0.5}
    geom = dict(n=(n, n, n), dx=dx, ng=ng, lo_bc=(2, 2, 2), hi_bc=(2, 2, 2))
    U = _average(physics, dim, (n, n, n), dx, (0.0, 0.0, 0.0), pw, ng, quadrature, xp, device)
    return physics, dim, inputs, geom, U


def algorithmic_bytes_per_cell_stage(physics: int, dim: int, nphase: int = 2) -> float:
    """(8/3) N 8 B: stage 1 reads U and writes U1 (2N doubles), stages 2 and 3 read U^(s), U^0 and
    write (3N doubles); relaxation is fused and adds nothing."""
    return (8.0 / 3.0) * nstate(physics, dim, nphase) * 8.0


def batch_shock_bubbles(count=48, seed=0, xp=None, device=None, quadrature=True, scheme="WENO5B",
                        sides=tuple(range(64, 769, 64))):
    """Independent 2D FIVEEQS shock-bubble cases with parameters drawn from numpy's PCG64 with `seed`:
    grid side (cells in y) uniform in `sides` (64, 128, ..., 768), aspect ratio U[1, 2] (cells in x =
    side x aspect, square cells, domain [0, aspect] x [0, 1]), shock Mach U[1.1, 3], bubble/ambient
    density ratio log-uniform in [0.01, 1000], radius U[0.1, 0.3] (centred at x = 0.3 + r + 0.05).
    Returns a list of (physics, dim, inputs, geom, U, params)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        side = int(rng.choice(np.array(sides)))
        aspect = float(rng.uniform(1.0, 2.0))
        Ma = float(rng.uniform(1.1, 3.0))
        ratio = float(np.exp(rng.uniform(np.log(0.01), np.log(1000.0))))
        r = float(rng.uniform(0.1, 0.3))
        nx = int(round(side * aspect))
        length = nx / side
        phys, dim, inputs, geom, U = shock_bubble(nx=nx, ny=side, Ma=Ma, rho_b=ratio, radius=r,
                                                  center=(0.3 + r + 0.05, 0.5), scheme=scheme, length=length,
                                                  xp=xp, device=device, quadrature=quadrature)
        out.append((phys, dim, inputs, geom, U, dict(side=side, nx=nx, aspect=aspect, Ma=Ma, ratio=ratio, r=r)))
    return out

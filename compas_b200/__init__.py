"""compas_b200: B200-native finite-volume right-hand side and TVD-RK3 level advance of the COMPAS
five- and six-equation diffuse-interface models.

The compute path is the CUDA library ``libcompas_b200.so`` (sm_100a) behind the C ABI declared in
``include/compas_b200.h``; this module binds it with ctypes. There is no CPU fallback: importing the
bindings without the built library raises.

Names mirror the reference's plugin points (include/COMPAS.H, include/Classes_Physics/
Class_Compressible_PhaseField.H): ``compute_dUdt_FV``, ``ThirdOrderSSPRK`` stages, ``FillPatch``
(single-box physical boundaries), ``Relaxation``, and the inputs keys ``FiniteVolume.Scheme``,
``Physics.RiemannSolver``, ``prob.EOS.*``, ``run.cfl``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

FIVEEQS = 555
SIXEQS = 666
FIVEEQS_NPHASE = 55501
SIXEQS_IE_NPHASE = 66601
MAX_PHASES = 4

OK = 0
EARG, ECUDA, ENOMEM, ESTATE, EUNSUPPORTED = -1, -2, -3, -4, -5
ERR_NAN, ERR_COVOLUME, ERR_RELAX_NOROOT, ERR_CFL, ERR_TIMEOUT, ERR_BOUND = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcompas_b200.so")


class CompasError(RuntimeError):
    """A C-ABI call returned a non-zero status (the reference would have aborted)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"compas_b200 error {code}: {msg}")
        self.code = code


class Parm(ctypes.Structure):
    """ctypes mirror of ``compas_b200_parm`` (include/compas_b200.h)."""

    _fields_ = [
        ("physics", ctypes.c_int),
        ("dim", ctypes.c_int),
        ("eos", ctypes.c_int),
        ("gamma_1", ctypes.c_double), ("gamma_2", ctypes.c_double),
        ("pinf_1", ctypes.c_double), ("pinf_2", ctypes.c_double),
        ("b_1", ctypes.c_double), ("b_2", ctypes.c_double),
        ("q_1", ctypes.c_double), ("q_2", ctypes.c_double),
        ("A1", ctypes.c_double), ("A2", ctypes.c_double),
        ("B1", ctypes.c_double), ("B2", ctypes.c_double),
        ("C1", ctypes.c_double), ("C2", ctypes.c_double),
        ("D1", ctypes.c_double), ("D2", ctypes.c_double),
        ("id_limiter", ctypes.c_int),
        ("id_weno", ctypes.c_int),
        ("num_grow", ctypes.c_int),
        ("thinc", ctypes.c_int),
        ("thinc_use_normal", ctypes.c_int),
        ("thinc_eps", ctypes.c_double), ("thinc_beta", ctypes.c_double),
        ("thinc_normal_threshold", ctypes.c_double),
        ("id_riemann", ctypes.c_int),
        ("source_term", ctypes.c_int),
        ("relaxation", ctypes.c_int),
        ("relax_trace", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("change_limiter", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("phase_field", ctypes.c_int),
        ("pf_mechanism", ctypes.c_int),
        ("pf_explicit_rc", ctypes.c_int),
        ("pf_flux", ctypes.c_int),
        ("pf_phase2flux", ctypes.c_int),
        ("pf_lambda", ctypes.c_double), ("pf_eta", ctypes.c_double),
        ("pf_eta_factor", ctypes.c_double), ("pf_eta_multiplier", ctypes.c_double),
        ("pf_cfl", ctypes.c_double),
        ("pf_max_step", ctypes.c_int),
        ("pf_tol_rel", ctypes.c_double),
        ("nphase", ctypes.c_int),
        ("gamma_k", ctypes.c_double * MAX_PHASES), ("pinf_k", ctypes.c_double * MAX_PHASES),
        ("b_k", ctypes.c_double * MAX_PHASES), ("q_k", ctypes.c_double * MAX_PHASES),
        ("Ak", ctypes.c_double * MAX_PHASES), ("Bk", ctypes.c_double * MAX_PHASES),
        ("Ck", ctypes.c_double * MAX_PHASES), ("Dk", ctypes.c_double * MAX_PHASES),
        ("autotune", ctypes.c_int),
        ("tma", ctypes.c_int),
        ("cv_1", ctypes.c_double),
        ("cv_2", ctypes.c_double),
        ("amr_interp", ctypes.c_int),
        ("id_bound", ctypes.c_int),
        ("id_lambda", ctypes.c_int),
    ]


class Geom(ctypes.Structure):
    """ctypes mirror of ``compas_b200_geom``."""

    _fields_ = [
        ("n", ctypes.c_int * 3),
        ("ng", ctypes.c_int),
        ("dx", ctypes.c_double * 3),
        ("lo_bc", ctypes.c_int * 3),
        ("hi_bc", ctypes.c_int * 3),
    ]


_lib_handle = None

_SIGS = {
    "compas_b200_last_error": (ctypes.c_char_p, []),
    "compas_b200_parm_init": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.c_int, ctypes.c_int]),
    "compas_b200_parm_init_nphase": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "compas_b200_parm_set": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.c_char_p, ctypes.c_char_p]),
    "compas_b200_parm_finalize": (ctypes.c_int, [ctypes.POINTER(Parm)]),
    "compas_b200_state_bytes": (ctypes.c_longlong, [ctypes.POINTER(Parm), ctypes.POINTER(Geom)]),
    "compas_b200_fill_boundary": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "compas_b200_compute_dUdt": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_nc_terms": (ctypes.c_int, [ctypes.POINTER(Parm)]),
    "compas_b200_energy_bound_min": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_level_bound_restarts": (ctypes.c_longlong, [ctypes.c_void_p]),
    "compas_b200_amr_nbox": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "compas_b200_amr_fill": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_thinc_face_values": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_level_get_control": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                                     ctypes.POINTER(ctypes.c_int)]),
    "compas_b200_level_set_control": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_derive": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_amr_tag": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "compas_b200_amr_regrid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_tag_cells": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_fma_peak": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                            ctypes.c_void_p]),
    "compas_b200_face_fluxes": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_void_p * 3, ctypes.c_void_p * 3,
                                               ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_rk3_stage": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_relaxation": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_rk3_step_noalloc": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                                    ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p]),
    "compas_b200_level_create": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom),
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "compas_b200_level_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "compas_b200_level_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_void_p]),
    "compas_b200_level_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_level_set_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_level_state": (ctypes.c_void_p, [ctypes.c_void_p]),
    "compas_b200_level_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                 ctypes.c_void_p]),
    "compas_b200_level_sync": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint)]),
    "compas_b200_level_dts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "compas_b200_level_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
    "compas_b200_level_step_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_void_p]),
    "compas_b200_level_pf_substeps": (ctypes.c_longlong, [ctypes.c_void_p]),
    "compas_b200_level_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int)]),
    "compas_b200_level_set_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "compas_b200_level_tma": (ctypes.c_int, [ctypes.c_void_p]),
    "compas_b200_batch_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int)]),
    "compas_b200_batch_set_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "compas_b200_amr_create": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "compas_b200_amr_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "compas_b200_amr_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_void_p]),
    "compas_b200_amr_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p]),
    "compas_b200_amr_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]),
    "compas_b200_amr_sync": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint)]),
    "compas_b200_amr_dts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "compas_b200_amr_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
    "compas_b200_level_pf_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_pf_grad_q": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                             ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_pf_compute_dUdt": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "compas_b200_pf_rk3_stage": (ctypes.c_int, [ctypes.POINTER(Parm), ctypes.POINTER(Geom), ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "compas_b200_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "compas_b200_batch_create_nphase": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "compas_b200_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "compas_b200_batch_add": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Parm), ctypes.POINTER(Geom),
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "compas_b200_batch_remove": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_batch_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "compas_b200_batch_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "compas_b200_batch_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.c_void_p]),
    "compas_b200_batch_bytes": (ctypes.c_longlong, [ctypes.c_void_p]),
    "compas_b200_batch_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
}

EXPORTED_SYMBOLS = tuple(_SIGS)


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it was not built (there is no fallback path)."""
    global _lib_handle
    if _lib_handle is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib_handle = h
    return _lib_handle


def _check(rc: int) -> None:
    if rc != OK:
        raise CompasError(rc, lib().compas_b200_last_error().decode())


def nstate(physics: int, dim: int, nphase: int = 2) -> int:
    """NSTATE of the model (include/Macros.H:73, :89, :114)."""
    if physics == FIVEEQS_NPHASE:
        return 2 * nphase + dim + 1
    if physics == SIXEQS_IE_NPHASE:
        return 3 * nphase + dim + 1
    return (4 if physics == FIVEEQS else 5) + dim


def parm_nstate(p: Parm) -> int:
    return nstate(p.physics, p.dim, p.nphase)


def _inputs_value(v) -> str:
    if isinstance(v, (list, tuple)):
        return " ".join(str(x) for x in v)
    return str(v)


def make_parm(physics: int, dim: int, inputs: dict | None = None, nphase: int | None = None) -> Parm:
    """A parameter block from reference defaults plus inputs keys, e.g.
    {"FiniteVolume.Scheme": "WENO5", "prob.EOS.gamma_2": 4.4, "run.cfl": 0.5}; for FIVEEQS_NPHASE and
    SIXEQS_IE_NPHASE the per-phase lists {"prob.EOS.gamma": [1.4, 1.5, 1.5]} and `nphase` (the
    compile-time NPHASE)."""
    p = Parm()
    if nphase is None:
        g = (inputs or {}).get("prob.EOS.gamma")
        nphase = (len(g) if physics in (FIVEEQS_NPHASE, SIXEQS_IE_NPHASE) and isinstance(g, (list, tuple))
                  else 2)
    _check(lib().compas_b200_parm_init_nphase(ctypes.byref(p), physics, dim, int(nphase)))
    for k, v in (inputs or {}).items():
        _check(lib().compas_b200_parm_set(ctypes.byref(p), k.encode(), _inputs_value(v).encode()))
    _check(lib().compas_b200_parm_finalize(ctypes.byref(p)))
    return p


def make_geom(n, dx, ng=3, lo_bc=(0, 0, 0), hi_bc=(0, 0, 0)) -> Geom:
    g = Geom()
    n = list(n) + [1] * (3 - len(n))
    dx = list(dx) + [1.0] * (3 - len(dx))
    for d in range(3):
        g.n[d] = int(n[d])
        g.dx[d] = float(dx[d])
        g.lo_bc[d] = int(lo_bc[d]) if d < len(lo_bc) else 0
        g.hi_bc[d] = int(hi_bc[d]) if d < len(hi_bc) else 0
    g.ng = int(ng)
    return g


def padded_shape(p: Parm, g: Geom) -> tuple:
    """(N, PZ, PY, PX) of a state array with ghosts (no z ghosts in 2D)."""
    gz = g.ng if p.dim == 3 else 0
    nz = g.n[2] if p.dim == 3 else 1
    return (parm_nstate(p), nz + 2 * gz, g.n[1] + 2 * g.ng, g.n[0] + 2 * g.ng)


def valid_view(a, p: Parm, g: Geom):
    """The valid cells of a padded array (numpy or torch), shape (N, nz, ny, nx)."""
    gz = g.ng if p.dim == 3 else 0
    nz = g.n[2] if p.dim == 3 else 1
    return a[:, gz:gz + nz, g.ng:g.ng + g.n[1], g.ng:g.ng + g.n[0]]


def _ptr(x) -> int:
    if x is None:
        return 0
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return int(x)


def _stream_ptr(stream) -> int:
    if stream is None:
        return 0
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)


# ---- drop-in kernels on caller-owned device arrays (torch CUDA tensors or raw pointers) ----------

def FillPatch(p: Parm, g: Geom, U, stream=None) -> None:
    """Physical and periodic ghost cells of a single-box level (COMPAS::FillPatch, source/COMPAS.cpp:1629-1732)."""
    _check(lib().compas_b200_fill_boundary(ctypes.byref(p), ctypes.byref(g), _ptr(U), _stream_ptr(stream)))


def compute_dUdt_FV(p: Parm, g: Geom, U, dUdt, cmax=None, err=None, stream=None) -> None:
    """dUdt of the valid cells from U with filled ghosts
    (Compressible_PhaseField::compute_dUdt_FV, source/Class_Compressible_PhaseField.cpp:3472-3537)."""
    _check(lib().compas_b200_compute_dUdt(ctypes.byref(p), ctypes.byref(g), _ptr(U), _ptr(dUdt), _ptr(cmax),
                                          _ptr(err), _stream_ptr(stream)))


def fma_peak(fp64: bool, iters: int = 1 << 14, stream=None) -> float:
    """Measured sustained FMA throughput (FLOP/s) of the FP32 or FP64 pipe of the current GPU."""
    out = ctypes.c_double()
    _check(lib().compas_b200_fma_peak(int(bool(fp64)), int(iters), ctypes.byref(out), _stream_ptr(stream)))
    return out.value


class TagCriterion(ctypes.Structure):
    """ctypes mirror of ``compas_b200_tag_criterion``."""

    _fields_ = [("var", ctypes.c_int), ("derived", ctypes.c_int), ("kind", ctypes.c_int),
                ("v0", ctypes.c_double), ("v1", ctypes.c_double)]


TAG_GRAD, TAG_LESS, TAG_GREATER, TAG_RANGE = 0, 1, 2, 3

# vnamesC / vnamesD of the two-phase models (include/Physics_Compressible5Eq/Variables_Compressible5Eq.H:18-19,
# include/Physics_Compressible6Eq/Variables_Compressible6Eq.H:18-19)
_STATE_NAMES = {
    FIVEEQS: lambda dim: ["a1rho1", "a2rho2", "rho_u", "rho_v", "rho_w"][:2 + dim] + ["rho_E", "a1"],
    SIXEQS: lambda dim: ["a1rho1", "a2rho2", "rho_u", "rho_v", "rho_w"][:2 + dim] + ["a1rho1E1", "a2rho2E2", "a1"],
}
_DERIVED_NAMES = {
    FIVEEQS: ["a1rho1", "a2rho2", "rho_u", "rho_v", "rho_w", "rho_E", "a1", "rho", "u", "v", "w", "P", "T", "c",
              "Mach", "vorticity_mag", "q_criterion", "lambda2"],
    SIXEQS: ["a1rho1", "a2rho2", "rho_u", "rho_v", "rho_w", "a1rho1E1", "a2rho2E2", "a1", "rho", "u", "v", "w", "P",
             "a1P1", "a2P2", "T", "c", "Mach", "vorticity_mag", "q_criterion", "lambda2"],
}


def tag_variable(physics: int, dim: int, name: str) -> tuple:
    """(index, derived) of a refinement variable name, state names first (the reference's
    VariableRegistry, include/Tagging.H:25-76)."""
    state = _STATE_NAMES[physics](dim)
    if name in state:
        return state.index(name), 0
    derived = _DERIVED_NAMES[physics]
    if name in derived:
        return derived.index(name), 1
    raise CompasError(EARG, f"Unknown refinement variable: {name}")


def _floats(v):
    if isinstance(v, str):
        return [float(x) for x in v.split()]
    if isinstance(v, (list, tuple)):
        return [float(x) for x in v]
    return [float(v)]


def tag_criteria(physics: int, dim: int, inputs: dict, lev: int, max_level: int | None = None) -> list:
    """The criteria ErrorEst applies on level `lev` from the run.refine.* inputs keys
    (source/COMPAS.cpp:1473-1532 reads them, :835-905 applies them): run.refine.ref_vars names the
    variables; run.refine.<name>.grad / value_less / value_greater hold one threshold per level,
    value_range two, run.refine.<name>.max_level the first level not tagged. max_level is the
    hierarchy's amr.max_level (default: the inputs key, else lev + 1); a threshold list too short for
    the levels tagged is an error, as in the reference."""
    if max_level is None:
        max_level = int(inputs.get("amr.max_level", lev + 1))
    names = inputs.get("run.refine.ref_vars", [])
    names = names.split() if isinstance(names, str) else list(names)
    out = []
    for name in names:
        var, derived = tag_variable(physics, dim, name)
        vmax = int(inputs.get(f"run.refine.{name}.max_level", 1 << 30))
        n_tag = max(0, min(vmax, max_level))
        for opt, kind, per in (("grad", TAG_GRAD, 1), ("value_less", TAG_LESS, 1),
                               ("value_greater", TAG_GREATER, 1), ("value_range", TAG_RANGE, 2)):
            key = f"run.refine.{name}.{opt}"
            if key not in inputs:
                continue
            vals = _floats(inputs[key])
            if len(vals) < per * n_tag:
                raise CompasError(EARG, f"run.refine.{name}.{opt} has {len(vals)} values, but {per * n_tag} are "
                                        f"needed to tag levels 0 to {n_tag - 1}")
            if lev >= vmax:
                continue
            c = TagCriterion(var, derived, kind, vals[per * lev], vals[per * lev + 1] if per == 2 else 0.0)
            out.append(c)
    return out


def tag_cells(p: Parm, g: Geom, U, criteria, tags, stream=None) -> None:
    """Refinement tags (1 tagged, 0 not) of the valid cells of one box into the device byte array
    tags (n[0] x n[1] x n[2], x fastest) from the ghost-filled padded state U (ErrorEst,
    source/COMPAS.cpp:767-932)."""
    arr = (TagCriterion * max(1, len(criteria)))(*criteria)
    _check(lib().compas_b200_tag_cells(ctypes.byref(p), ctypes.byref(g), _ptr(U), ctypes.addressof(arr),
                                       len(criteria), _ptr(tags), _stream_ptr(stream)))


def thinc_face_values(beta, sigma, abar, side, out, stream=None) -> None:
    """THINC face values of alpha1 (the stage kernels' device function) for device arrays of parameters
    (float64 beta, sigma, abar; int32 side) into the float64 device array out."""
    _check(lib().compas_b200_thinc_face_values(_ptr(beta), _ptr(sigma), _ptr(abar), _ptr(side), int(out.numel()),
                                               _ptr(out), _stream_ptr(stream)))


def derive(p: Parm, g: Geom, U, names, out, stream=None) -> None:
    """Plot variables `names` (state or derived names of the model, resolved as tag_variable does) of
    the valid cells of the ghost-filled padded device state U into the device array out, shape
    (len(names), nz, ny, nx)."""
    idx = [tag_variable(p.physics, p.dim, nm) for nm in names]
    vars_ = (ctypes.c_int * max(1, len(idx)))(*[v for v, _ in idx])
    der = (ctypes.c_int * max(1, len(idx)))(*[d for _, d in idx])
    _check(lib().compas_b200_derive(ctypes.byref(p), ctypes.byref(g), _ptr(U), ctypes.addressof(vars_),
                                    ctypes.addressof(der), len(idx), _ptr(out), _stream_ptr(stream)))


FACES_ALL, FACES_BOUNDARY = 0, 1


def nc_terms(p: Parm) -> int:
    """Non-conservative face terms of the model (NC_TERMS: 1 five-equation, 3 six-equation)."""
    n = lib().compas_b200_nc_terms(ctypes.byref(p))
    if n <= 0:
        _check(n)
    return n


def energy_bound_min(p: Parm, g: Geom, U, out=None, stream=None):
    """Smallest energy bound over the valid cells of the device state U (FIVEEQS): the value the
    reference's MinEnergyBound (source/Class_Compressible_PhaseField.cpp:3596-3635) checks after every
    stage under FiniteVolume.ID_Bound = 1. Into the device double `out` when given, else returned."""
    import torch

    res = out if out is not None else torch.empty(1, dtype=torch.float64, device="cuda")
    _check(lib().compas_b200_energy_bound_min(ctypes.byref(p), ctypes.byref(g), _ptr(U), _ptr(res),
                                              _stream_ptr(stream)))
    if out is None:
        return float(res.item())
    return None


def face_shape(p: Parm, g: Geom, d: int, ncomp: int) -> tuple:
    """Shape (components, z, y, x) of the face array of direction d (a face MultiFab without ghosts)."""
    n = [g.n[0] + (d == 0), g.n[1] + (d == 1), (g.n[2] + (d == 2)) if p.dim == 3 else 1]
    return (ncomp, n[2], n[1], n[0])


def face_fluxes(p: Parm, g: Geom, Us, flux, flux_nc=None, which=FACES_ALL, area_scaled=True, err=None,
                stream=None) -> None:
    """Face fluxes of one box from its ghost-filled stage state for the flux registers, area-scaled as
    ScaleFaceFluxesByArea (source/Class_Compressible_PhaseField.cpp:3433-3466) unless area_scaled is
    False; flux[d] / flux_nc[d] are device arrays of face_shape(p, g, d, ...) or None."""
    fl = (ctypes.c_void_p * 3)(*[_ptr(flux[d]) if flux is not None and d < len(flux) else None for d in range(3)])
    fn = (ctypes.c_void_p * 3)(*[_ptr(flux_nc[d]) if flux_nc is not None and d < len(flux_nc) else None
                                 for d in range(3)])
    _check(lib().compas_b200_face_fluxes(ctypes.byref(p), ctypes.byref(g), _ptr(Us), int(which), int(bool(area_scaled)),
                                         fl, fn, _ptr(err), _stream_ptr(stream)))


def ThirdOrderSSPRK_stage(p: Parm, g: Geom, stage: int, Us, Uold, Unew, dt_dev, cmax=None, err=None,
                          stream=None) -> None:
    """One fused stage of ThirdOrderSSPRK plus PostTimeStage (source/Class_Compressible_PhaseField.cpp:3937-4107)."""
    _check(lib().compas_b200_rk3_stage(ctypes.byref(p), ctypes.byref(g), stage, _ptr(Us), _ptr(Uold), _ptr(Unew),
                                       _ptr(dt_dev), _ptr(cmax), _ptr(err), _stream_ptr(stream)))


def ThirdOrderSSPRK_step_noalloc(p: Parm, g: Geom, U, dt: float, cmax=None, err=None, stream=None) -> None:
    """One whole TVD-RK3 step in place on U (device) without allocating device memory: the stage
    states live in the library's fixed scratch array (states up to 16 MiB; see compas_b200.h)."""
    _check(lib().compas_b200_rk3_step_noalloc(ctypes.byref(p), ctypes.byref(g), _ptr(U), float(dt), _ptr(cmax),
                                              _ptr(err), _stream_ptr(stream)))


def PhaseField_GradQPF(p: Parm, g: Geom, U, dt: float, gq, stream=None) -> np.ndarray:
    """Mechanism evolution over dt and the face gradients of the regularisation potential Q into the
    device arrays gq[d] (PhaseFieldMechanism_Evolve + PhaseField_GradQPF,
    source/Class_Compressible_PhaseField.cpp:596-711, :2132-2401). Returns the info vector
    (max|u|, mobility, eta, mechanism sub-steps, solver iterations, max|grad Q|, relative residual)."""
    info = (ctypes.c_double * 7)()
    ptrs = [_ptr(gq[d]) if d < len(gq) else None for d in range(3)]
    _check(lib().compas_b200_pf_grad_q(ctypes.byref(p), ctypes.byref(g), _ptr(U), float(dt), ptrs[0], ptrs[1],
                                       ptrs[2], info, _stream_ptr(stream)))
    return np.array(info[:])


def PhaseField_compute_dUdt_FV(p: Parm, g: Geom, U, dUdt, gq, err=None, stream=None) -> None:
    """Phase-Field right-hand side (source/Class_Compressible_PhaseField.cpp:950-1004)."""
    ptrs = [_ptr(gq[d]) if d < len(gq) else None for d in range(3)]
    _check(lib().compas_b200_pf_compute_dUdt(ctypes.byref(p), ctypes.byref(g), _ptr(U), _ptr(dUdt), ptrs[0],
                                             ptrs[1], ptrs[2], _ptr(err), _stream_ptr(stream)))


def PhaseField_ThirdOrderSSPRK_stage(p: Parm, g: Geom, stage: int, Us, Uold, Unew, dt_dev, gq, err=None,
                                     stream=None) -> None:
    """One stage of PhaseField_ThirdOrderSSPRK (source/Class_Compressible_PhaseField.cpp:2619-2752)."""
    ptrs = [_ptr(gq[d]) if d < len(gq) else None for d in range(3)]
    _check(lib().compas_b200_pf_rk3_stage(ctypes.byref(p), ctypes.byref(g), int(stage), _ptr(Us), _ptr(Uold),
                                          _ptr(Unew), _ptr(dt_dev), ptrs[0], ptrs[1], ptrs[2], _ptr(err),
                                          _stream_ptr(stream)))


def Relaxation(p: Parm, g: Geom, U, err=None, stream=None) -> None:
    """SIXEQS pressure relaxation in place (source/Class_Compressible6Eq_PhaseField.cpp:437-474)."""
    _check(lib().compas_b200_relaxation(ctypes.byref(p), ctypes.byref(g), _ptr(U), _ptr(err), _stream_ptr(stream)))


@dataclass
class SyncInfo:
    t: float
    steps: int
    status: int


class Level:
    """One single-box level with device-resident state and the reference's time-step control."""

    def __init__(self, p: Parm, g: Geom):
        self.p, self.g = p, g
        self._h = ctypes.c_void_p()
        _check(lib().compas_b200_level_create(ctypes.byref(p), ctypes.byref(g), ctypes.byref(self._h)))
        self.shape = padded_shape(p, g)
        self.nbytes = int(lib().compas_b200_state_bytes(ctypes.byref(p), ctypes.byref(g)))

    def close(self) -> None:
        if self._h:
            lib().compas_b200_level_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, U, t0: float = 0.0, stream=None) -> None:
        """Copy a padded state in (numpy host array, or a torch tensor on host or device)."""
        if isinstance(U, np.ndarray):
            U = np.ascontiguousarray(U, dtype=np.float64)
            assert U.nbytes == self.nbytes, (U.shape, self.shape)
            _check(lib().compas_b200_level_upload(self._h, U.ctypes.data, 0, t0, _stream_ptr(stream)))
            # the copy from pageable memory is staged before the call returns
        else:
            assert U.numel() * 8 == self.nbytes
            _check(lib().compas_b200_level_upload(self._h, U.data_ptr(), 1 if U.is_cuda else 0, t0,
                                                  _stream_ptr(stream)))

    def step_host(self, host_in, host_out, slabs: int = 32, stream=None) -> None:
        """One step from the padded host state host_in to host_out (pinned torch tensors or numpy
        arrays), the copies in both directions overlapped with the stages slab by slab."""
        def ptr(x):
            if isinstance(x, np.ndarray):
                assert x.dtype == np.float64 and x.flags.c_contiguous and x.nbytes == self.nbytes
                return x.ctypes.data
            assert not x.is_cuda and x.numel() * 8 == self.nbytes
            return x.data_ptr()
        _check(lib().compas_b200_level_step_host(self._h, ptr(host_in), ptr(host_out), int(slabs),
                                                 _stream_ptr(stream)))

    def set_state(self, U, stream=None) -> None:
        """Replace the state only (keeps the time and the time-step control)."""
        if isinstance(U, np.ndarray):
            U = np.ascontiguousarray(U, dtype=np.float64)
            _check(lib().compas_b200_level_set_state(self._h, U.ctypes.data, 0, _stream_ptr(stream)))
        else:
            _check(lib().compas_b200_level_set_state(self._h, U.data_ptr(), 1 if U.is_cuda else 0,
                                                     _stream_ptr(stream)))

    def download(self, out=None, stream=None):
        """Copy the padded state out (into `out`, numpy or torch, or a new numpy array)."""
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        if isinstance(out, np.ndarray):
            _check(lib().compas_b200_level_download(self._h, out.ctypes.data, 0, _stream_ptr(stream)))
            self.sync(check=False)
        else:
            _check(lib().compas_b200_level_download(self._h, out.data_ptr(), 1 if out.is_cuda else 0,
                                                    _stream_ptr(stream)))
        return out

    def state_ptr(self) -> int:
        return int(lib().compas_b200_level_state(self._h))

    def get_control(self) -> dict:
        """Time, previous step size, the last step's largest face wave speed and the step count."""
        t, dtp, cm, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().compas_b200_level_get_control(self._h, ctypes.byref(t), ctypes.byref(dtp), ctypes.byref(cm),
                                                   ctypes.byref(n)))
        return {"t": t.value, "dt_prev": dtp.value, "cmax": cm.value, "steps": n.value}

    def set_control(self, t: float, dt_prev: float, cmax: float, steps: int, stream=None) -> None:
        """Restore the step control of a checkpoint (the next advance continues the checkpointed run)."""
        _check(lib().compas_b200_level_set_control(self._h, float(t), float(dt_prev), float(cmax), int(steps),
                                                   _stream_ptr(stream)))

    def advance(self, nsteps: int, stop_time: float = 1.0e300, use_graph: bool = True, stream=None) -> None:
        _check(lib().compas_b200_level_advance(self._h, int(nsteps), float(stop_time), 1 if use_graph else 0,
                                               _stream_ptr(stream)))

    def sync(self, check: bool = True) -> SyncInfo:
        t = ctypes.c_double()
        s = ctypes.c_int()
        st = ctypes.c_uint()
        rc = lib().compas_b200_level_sync(self._h, ctypes.byref(t), ctypes.byref(s), ctypes.byref(st))
        if check:
            _check(rc)
        return SyncInfo(t.value, s.value, st.value)

    def dts(self, n: int) -> np.ndarray:
        out = (ctypes.c_double * n)()
        _check(lib().compas_b200_level_dts(self._h, out, n))
        return np.array(out[:], dtype=np.float64)

    def launches(self) -> int:
        return int(lib().compas_b200_level_launches(self._h))

    def kernel(self) -> tuple:
        """(launch shape, tile order) of the stage kernel: the autotuner's pick after the first advance."""
        sh, od = ctypes.c_int(), ctypes.c_int()
        _check(lib().compas_b200_level_kernel(self._h, ctypes.byref(sh), ctypes.byref(od)))
        return sh.value, od.value

    def set_kernel(self, shape: int, order: int) -> None:
        """Force a launch shape and tile order (no tuning for this level)."""
        _check(lib().compas_b200_level_set_kernel(self._h, int(shape), int(order)))

    def tma(self) -> bool:
        """Whether the stage kernel stages its halo slabs by TMA (3D mixed form)."""
        return bool(lib().compas_b200_level_tma(self._h))

    def bound_restarts(self) -> int:
        """Steps taken again because a stage violated the energy bound (FiniteVolume.ID_Bound = 1)."""
        return int(lib().compas_b200_level_bound_restarts(self._h))

    def pf_substeps(self) -> int:
        """Phase-Field sub-steps taken so far (PhaseField.phase_field = 1)."""
        return int(lib().compas_b200_level_pf_substeps(self._h))

    def pf_info(self) -> dict:
        """Counters of the last Phase-Field step."""
        v = (ctypes.c_double * 7)()
        _check(lib().compas_b200_level_pf_info(self._h, v))
        keys = ("max_v", "mobility", "eta", "mechanism_steps", "solver_iterations", "max_grad_q", "residual")
        return dict(zip(keys, v[:]))


class AmrBox(ctypes.Structure):
    """ctypes mirror of ``compas_b200_amr_box``."""

    _fields_ = [("lev", ctypes.c_int), ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3)]


class Amr:
    """Multi-level advance of a fixed box hierarchy (refinement ratio 2, subcycling, refluxing):
    boxes = [(lev, lo, hi), ...] with inclusive corners in each level's index space; g0 is level 0."""

    def __init__(self, p: Parm, g0: Geom, boxes):
        self._h = None
        arr = (AmrBox * len(boxes))()
        for b, (lev, lo, hi) in enumerate(boxes):
            arr[b].lev = lev
            for d in range(3):
                arr[b].lo[d] = lo[d]
                arr[b].hi[d] = hi[d]
        self.boxes = list(boxes)
        self.p, self.g0 = p, g0
        h = ctypes.c_void_p()
        nlev = 1 + max(b[0] for b in boxes)
        _check(lib().compas_b200_amr_create(ctypes.byref(p), ctypes.byref(g0), nlev, arr, len(boxes), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h is not None:
            lib().compas_b200_amr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, box: int, U, stream=None) -> None:
        """Padded state of box `box` (numpy host array, or a torch tensor on host or device)."""
        if isinstance(U, np.ndarray):
            U = np.ascontiguousarray(U, dtype=np.float64)
            _check(lib().compas_b200_amr_upload(self._h, box, U.ctypes.data, 0, _stream_ptr(stream)))
        else:
            _check(lib().compas_b200_amr_upload(self._h, box, U.data_ptr(), 1 if U.is_cuda else 0, _stream_ptr(stream)))

    def download(self, box: int, out=None, stream=None):
        lev, lo, hi = self.boxes[box]
        n = [hi[d] - lo[d] + 1 for d in range(3)]
        ng = self.g0.ng
        dim = self.p.dim
        shape = (parm_nstate(self.p), (n[2] + 2 * ng) if dim == 3 else 1, n[1] + 2 * ng, n[0] + 2 * ng)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        if isinstance(out, np.ndarray):
            _check(lib().compas_b200_amr_download(self._h, box, out.ctypes.data, 0, _stream_ptr(stream)))
            self.sync(check=False)
        else:
            _check(lib().compas_b200_amr_download(self._h, box, out.data_ptr(), 1 if out.is_cuda else 0,
                                                  _stream_ptr(stream)))
        return out

    def advance(self, nsteps: int, stop_time: float = 1.0e300, stream=None) -> None:
        _check(lib().compas_b200_amr_advance(self._h, int(nsteps), float(stop_time), _stream_ptr(stream)))

    def level_boxes(self, lev: int) -> list:
        """Indices (in self.boxes) of the boxes of level lev, in the object's order."""
        return [b for b, (l, _, _) in enumerate(self.boxes) if l == lev]

    def tag(self, lev: int, criteria, stream=None) -> list:
        """Refinement tags of level lev (ErrorEst): one uint8 array (nz, ny, nx) per box of the level, in
        level_boxes order, computed on the device from the state resident there."""
        import torch

        ids = self.level_boxes(lev)
        sizes = []
        for b in ids:
            _, lo, hi = self.boxes[b]
            n = [hi[d] - lo[d] + 1 for d in range(3)]
            sizes.append((n[2] if self.p.dim == 3 else 1, n[1], n[0]))
        total = sum(int(np.prod(s)) for s in sizes)
        tags = torch.zeros(max(total, 1), dtype=torch.uint8, device="cuda")
        arr = (TagCriterion * max(1, len(criteria)))(*criteria)
        _check(lib().compas_b200_amr_tag(self._h, int(lev), ctypes.addressof(arr), len(criteria), tags.data_ptr(),
                                         _stream_ptr(stream)))
        host = tags.cpu().numpy()
        out, off = [], 0
        for s in sizes:
            m = int(np.prod(s))
            out.append(host[off:off + m].reshape(s))
            off += m
        return out

    def fill(self, lev: int, stream=None) -> None:
        """Ghost cells of every box of level lev at its current time (the FillPatch of a stage)."""
        _check(lib().compas_b200_amr_fill(self._h, int(lev), _stream_ptr(stream)))

    def regrid(self, boxes, stream=None) -> None:
        """Replace the boxes of levels >= 1 (level 0 unchanged), the state staying on the device."""
        arr = (AmrBox * len(boxes))()
        for b, (lev, lo, hi) in enumerate(boxes):
            arr[b].lev = lev
            for d in range(3):
                arr[b].lo[d] = lo[d]
                arr[b].hi[d] = hi[d]
        _check(lib().compas_b200_amr_regrid(self._h, arr, len(boxes), _stream_ptr(stream)))
        self.boxes = list(boxes)

    def sync(self, check: bool = True):
        t, s, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_uint()
        _check(lib().compas_b200_amr_sync(self._h, ctypes.byref(t), ctypes.byref(s), ctypes.byref(st)))
        return SyncInfo(t.value, s.value, st.value)

    def dts(self, n: int) -> np.ndarray:
        out = (ctypes.c_double * n)()
        _check(lib().compas_b200_amr_dts(self._h, out, n))
        return np.array(out[:], dtype=np.float64)

    def launches(self) -> int:
        return int(lib().compas_b200_amr_launches(self._h))


@dataclass
class CaseInfo:
    id: int
    t: float
    steps: int
    done: bool
    status: int


class Batch:
    """Many independent single-box cases (uneven sizes, own EOS and boundaries, own time-step control)
    advanced together, one persistent launch per RK stage over a device-side box list."""

    def __init__(self, physics: int, dim: int, id_limiter: int = 5, precision: int = 0, capacity: int = 1024,
                 nphase: int = 2):
        self.physics, self.dim, self.nphase = physics, dim, nphase
        self._h = ctypes.c_void_p()
        _check(lib().compas_b200_batch_create_nphase(physics, dim, nphase, id_limiter, precision, capacity,
                                                     ctypes.byref(self._h)))
        self.capacity = capacity
        self._shapes = {}

    def close(self) -> None:
        if self._h:
            lib().compas_b200_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, p: Parm, g: Geom, U, stop_time: float = 1.0e300, max_steps: int = 2 ** 31 - 1,
            stream=None) -> int:
        cid = ctypes.c_int()
        if isinstance(U, np.ndarray):
            U = np.ascontiguousarray(U, dtype=np.float64)
            ptr, dev = U.ctypes.data, 0
        else:
            ptr, dev = U.data_ptr(), 1 if U.is_cuda else 0
        _check(lib().compas_b200_batch_add(self._h, ctypes.byref(p), ctypes.byref(g), ptr, dev, float(stop_time),
                                           int(max_steps), _stream_ptr(stream), ctypes.byref(cid)))
        self._shapes[cid.value] = padded_shape(p, g)
        return cid.value

    def remove(self, case_id: int, stream=None) -> None:
        _check(lib().compas_b200_batch_remove(self._h, int(case_id), _stream_ptr(stream)))
        self._shapes.pop(case_id, None)

    def advance(self, nsteps: int, use_graph: bool = True, stream=None) -> None:
        _check(lib().compas_b200_batch_advance(self._h, int(nsteps), 1 if use_graph else 0, _stream_ptr(stream)))

    def poll(self) -> list:
        cap = max(len(self._shapes), 1)
        ids = (ctypes.c_int * cap)()
        ts = (ctypes.c_double * cap)()
        st = (ctypes.c_int * cap)()
        dn = (ctypes.c_int * cap)()
        er = (ctypes.c_uint * cap)()
        n = lib().compas_b200_batch_poll(self._h, ids, ts, st, dn, er, cap)
        if n < 0:
            _check(n)
        return [CaseInfo(ids[i], ts[i], st[i], bool(dn[i]), er[i]) for i in range(min(n, cap))]

    def download(self, case_id: int, out=None, stream=None):
        if out is None:
            out = np.empty(self._shapes[case_id], dtype=np.float64)
        if isinstance(out, np.ndarray):
            _check(lib().compas_b200_batch_download(self._h, int(case_id), out.ctypes.data, 0, _stream_ptr(stream)))
        else:
            _check(lib().compas_b200_batch_download(self._h, int(case_id), out.data_ptr(), 1 if out.is_cuda else 0,
                                                    _stream_ptr(stream)))
        return out

    def bytes(self) -> int:
        return int(lib().compas_b200_batch_bytes(self._h))

    def launches(self) -> int:
        return int(lib().compas_b200_batch_launches(self._h))

    def kernel(self) -> tuple:
        sh, od = ctypes.c_int(), ctypes.c_int()
        _check(lib().compas_b200_batch_kernel(self._h, ctypes.byref(sh), ctypes.byref(od)))
        return sh.value, od.value

    def set_kernel(self, shape: int, order: int) -> None:
        _check(lib().compas_b200_batch_set_kernel(self._h, int(shape), int(order)))

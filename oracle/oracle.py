"""Test infrastructure: ctypes loader of the CPU oracles of the finite-volume RHS / TVD-RK3 path.

Two libraries export the same C interface (oracle/oracle_api.h):
  * ``oracle/liboracle.so``  - plain-C restatement of the reference algorithm (oracle/compas_oracle.c),
    built from committed sources anywhere gcc is available;
  * ``oracle/_ref/libref_<model>_<dim>d.so`` - the reference's own include/Physics_* and
    include/Operators_* headers compiled against oracle/refshim (built only where the reference
    tree is present; see oracle/Makefile).

Only tests, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use this module; the
product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_LIB = os.path.join(HERE, "liboracle.so")

FIVEEQS, SIXEQS, FIVEEQS_NPHASE, SIXEQS_IE_NPHASE = 555, 666, 55501, 66601


class Case(ctypes.Structure):
    _fields_ = [
        ("physics", ctypes.c_int),
        ("dim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("ng", ctypes.c_int),
        ("dx", ctypes.c_double * 3),
        ("lo_bc", ctypes.c_int * 3),
        ("hi_bc", ctypes.c_int * 3),
        ("A1", ctypes.c_double), ("A2", ctypes.c_double),
        ("B1", ctypes.c_double), ("B2", ctypes.c_double),
        ("C1", ctypes.c_double), ("C2", ctypes.c_double),
        ("D1", ctypes.c_double), ("D2", ctypes.c_double),
        ("id_limiter", ctypes.c_int),
        ("id_weno", ctypes.c_int),
        ("id_riemann", ctypes.c_int),
        ("source_term", ctypes.c_int),
        ("relaxation", ctypes.c_int),
        ("relax_trace", ctypes.c_double),
        ("thinc", ctypes.c_int),
        ("thinc_use_normal", ctypes.c_int),
        ("thinc_eps", ctypes.c_double), ("thinc_beta", ctypes.c_double),
        ("thinc_normal_threshold", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("change_limiter", ctypes.c_int),
        ("nphase", ctypes.c_int),
        ("Ak", ctypes.c_double * 4), ("Bk", ctypes.c_double * 4),
        ("Ck", ctypes.c_double * 4), ("Dk", ctypes.c_double * 4),
        ("amr_interp", ctypes.c_int),
        ("id_bound", ctypes.c_int),
        ("id_lambda", ctypes.c_int),
    ]


_P = ctypes.POINTER(Case)
_D = ctypes.c_void_p
_SIGS = {
    "cmp_nstate": (ctypes.c_int, [_P]),
    "cmp_fill_ghosts": (ctypes.c_int, [_P, _D]),
    "cmp_compute_dudt": (ctypes.c_int, [_P, _D, _D, ctypes.POINTER(ctypes.c_double)]),
    "cmp_relax": (ctypes.c_int, [_P, _D]),
    "cmp_rk3_step": (ctypes.c_int, [_P, _D, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
    "cmp_advance": (ctypes.c_int, [_P, _D, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double), _D]),
    "cmp_threads": (ctypes.c_int, []),
    "cmp_pf_step": (ctypes.c_int, [_P, ctypes.c_void_p, _D, ctypes.c_double, _D]),
    "cmp_pf_grad_q": (ctypes.c_int, [_P, ctypes.c_void_p, _D, ctypes.c_double, _D, _D, _D, _D]),
    "cmp_pf_dudt": (ctypes.c_int, [_P, ctypes.c_void_p, _D, _D, _D, _D, _D]),
    "cmp_advance_pf": (ctypes.c_int, [_P, ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double,
                                      ctypes.POINTER(ctypes.c_double), _D]),
    "cmp_amr_advance": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_double, ctypes.POINTER(ctypes.c_double), _D]),
    "cmp_tag": (ctypes.c_int, [_P, _D, _D, ctypes.c_void_p, ctypes.c_int, _D]),
}
# bound where the library has them (a library built before they existed still loads)
_OPTIONAL_SIGS = {
    "cmp_derive": (ctypes.c_int, [_P, _D, _D, _D, _D, ctypes.c_int, _D]),
    "cmp_thinc_face": (ctypes.c_int, [_D, _D, _D, _D, ctypes.c_longlong, _D]),
    "cmp_energy_bound_min": (ctypes.c_int, [_P, _D, ctypes.POINTER(ctypes.c_double)]),
    "cmp_bound_restarts": (ctypes.c_int, []),
}


def thinc_face_values(beta, sigma, abar, side, physics=SIXEQS, dim=3) -> np.ndarray:
    """The reference's THINC face value (reference-header build) for numpy parameter arrays."""
    lib = load("reference", physics, dim)
    b, s, a = (np.ascontiguousarray(x, dtype=np.float64) for x in (beta, sigma, abar))
    sd = np.ascontiguousarray(side, dtype=np.int32)
    out = np.zeros(b.size)
    rc = lib.cmp_thinc_face(b.ctypes.data, s.ctypes.data, a.ctypes.data, sd.ctypes.data, b.size, out.ctypes.data)
    if rc < 0:
        raise RuntimeError("cmp_thinc_face failed")
    return out


class TagCrit(ctypes.Structure):
    """ctypes mirror of ``cmp_tag_crit`` (oracle/oracle_api.h)."""

    _fields_ = [("var", ctypes.c_int), ("derived", ctypes.c_int), ("kind", ctypes.c_int),
                ("v0", ctypes.c_double), ("v1", ctypes.c_double)]


class AmrBox(ctypes.Structure):
    """ctypes mirror of ``cmp_amr_box`` (oracle/oracle_api.h)."""

    _fields_ = [("lev", ctypes.c_int), ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3)]


class PfCase(ctypes.Structure):
    """ctypes mirror of ``cmp_pf`` (oracle/oracle_api.h)."""

    _fields_ = [
        ("mechanism", ctypes.c_int), ("explicit_rc", ctypes.c_int),
        ("lambda_", ctypes.c_double), ("eta", ctypes.c_double), ("eta_factor", ctypes.c_double),
        ("eta_multiplier", ctypes.c_double), ("cfl", ctypes.c_double), ("max_step", ctypes.c_int),
        ("tol_rel", ctypes.c_double), ("phase2flux", ctypes.c_int), ("flux", ctypes.c_int),
    ]


def pf_from(parm, tol_rel=None) -> PfCase:
    """Oracle Phase-Field parameters from a compas_b200 Parm (tol_rel overrides LinearSystem.tol_rel)."""
    q = PfCase()
    q.mechanism, q.explicit_rc = parm.pf_mechanism, parm.pf_explicit_rc
    q.lambda_, q.eta, q.eta_factor = parm.pf_lambda, parm.pf_eta, parm.pf_eta_factor
    q.eta_multiplier, q.cfl, q.max_step = parm.pf_eta_multiplier, parm.pf_cfl, parm.pf_max_step
    q.tol_rel = parm.pf_tol_rel if tol_rel is None else tol_rel
    q.phase2flux = parm.pf_phase2flux
    q.flux = parm.pf_flux
    return q

_cache: dict = {}


def ref_lib_path(physics: int, dim: int, nphase: int = 2) -> str:
    if physics == FIVEEQS_NPHASE:
        return os.path.join(REF_DIR, f"libref_5eqn{nphase}_{dim}d.so")
    if physics == SIXEQS_IE_NPHASE:
        return os.path.join(REF_DIR, f"libref_6eqn{nphase}_{dim}d.so")
    model = "5eq" if physics == FIVEEQS else "6eq"
    return os.path.join(REF_DIR, f"libref_{model}_{dim}d.so")


def have_ref(physics: int, dim: int, nphase: int = 2) -> bool:
    return os.path.exists(ref_lib_path(physics, dim, nphase))


def build_port() -> str:
    """Compile the plain-C restatement if needed (gcc, OpenMP)."""
    src = os.path.join(HERE, "compas_oracle.c")
    if not os.path.exists(PORT_LIB) or os.path.getmtime(PORT_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "port"])
    return PORT_LIB


def load(kind: str, physics: int, dim: int, nphase: int = 2) -> ctypes.CDLL:
    """kind 'reference' (reference headers) or 'port' (C restatement)."""
    path = ref_lib_path(physics, dim, nphase) if kind == "reference" else build_port()
    if path not in _cache:
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        h = ctypes.CDLL(path)
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        for name, (res, args) in _OPTIONAL_SIGS.items():
            if hasattr(h, name):
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
        _cache[path] = h
    return _cache[path]


def case_from(parm, geom) -> Case:
    """Oracle case from a compas_b200 Parm / Geom pair (same field meanings)."""
    c = Case()
    c.physics, c.dim = parm.physics, parm.dim
    for d in range(3):
        c.n[d] = geom.n[d]
        c.dx[d] = geom.dx[d]
        c.lo_bc[d] = geom.lo_bc[d]
        c.hi_bc[d] = geom.hi_bc[d]
    if parm.dim == 2:
        c.n[2] = 1
    c.ng = geom.ng
    for k in ("A1", "A2", "B1", "B2", "C1", "C2", "D1", "D2", "id_limiter", "id_weno", "id_riemann", "source_term",
              "relaxation", "relax_trace", "thinc", "thinc_use_normal", "thinc_eps", "thinc_beta",
              "thinc_normal_threshold", "cfl", "change_limiter"):
        setattr(c, k, getattr(parm, k))
    c.nphase = getattr(parm, "nphase", 2)
    c.amr_interp = getattr(parm, "amr_interp", 0)
    c.id_bound = getattr(parm, "id_bound", 0)
    c.id_lambda = getattr(parm, "id_lambda", 1)
    if parm.physics in (FIVEEQS_NPHASE, SIXEQS_IE_NPHASE):
        for k in range(4):
            c.Ak[k], c.Bk[k], c.Ck[k], c.Dk[k] = parm.Ak[k], parm.Bk[k], parm.Ck[k], parm.Dk[k]
    return c


class Oracle:
    def __init__(self, kind: str, parm, geom, thinc_ulp: bool = False):
        """thinc_ulp (port only): move every THINC face value up by one ulp, to measure how strongly
        a case amplifies last-bit differences of exp/log/tanh between math libraries."""
        self.kind = kind
        # parm: a compas_b200 Parm (with geom), or an oracle Case already filled (oracle.parm)
        self.case = parm if isinstance(parm, Case) else case_from(parm, geom)
        self.lib = load(kind, self.case.physics, self.case.dim, self.case.nphase)
        self.thinc_ulp = bool(thinc_ulp)
        if self.thinc_ulp and kind != "port":
            raise ValueError("the one-ulp THINC control exists in the port only")
        if kind == "port":
            self.lib.cmp_set_thinc_ulp.argtypes = [ctypes.c_int]
            self.lib.cmp_set_thinc_ulp.restype = None

    def _call(self, rc):
        if rc < 0:
            raise RuntimeError(f"oracle ({self.kind}) failed: {rc}")
        return rc

    @property
    def _c(self):
        # the one-ulp control is process-wide in the port: set it for this instance before each call
        if self.kind == "port":
            self.lib.cmp_set_thinc_ulp(int(self.thinc_ulp))
        return ctypes.byref(self.case)

    def fill_ghosts(self, U: np.ndarray) -> None:
        assert U.flags.c_contiguous and U.dtype == np.float64
        self._call(self.lib.cmp_fill_ghosts(self._c, U.ctypes.data))

    def compute_dudt(self, U: np.ndarray):
        dU = np.zeros_like(U)
        cm = ctypes.c_double()
        self._call(self.lib.cmp_compute_dudt(self._c, U.ctypes.data, dU.ctypes.data,
                                             ctypes.byref(cm)))
        return dU, cm.value

    def relax(self, U: np.ndarray) -> None:
        self._call(self.lib.cmp_relax(self._c, U.ctypes.data))

    def rk3_step(self, U: np.ndarray, dt: float) -> float:
        cm = ctypes.c_double()
        self._call(self.lib.cmp_rk3_step(self._c, U.ctypes.data, dt, ctypes.byref(cm)))
        return cm.value

    def advance(self, U: np.ndarray, nsteps: int, stop_time: float = 1e300, t0: float = 0.0):
        t = ctypes.c_double(t0)
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        n = self._call(self.lib.cmp_advance(self._c, U.ctypes.data, nsteps, stop_time,
                                            ctypes.byref(t), dts.ctypes.data))
        return t.value, dts[:n]

    # ---- Phase-Field step (reference-header build only) ----------------------------------------
    def _pf(self, pf):
        if self.kind != "reference":
            raise RuntimeError("the Phase-Field step is in the reference-header oracle only")
        return ctypes.byref(pf)

    def pf_step(self, U: np.ndarray, pf, dt: float):
        info = np.zeros(6)
        self._call(self.lib.cmp_pf_step(self._c, self._pf(pf), U.ctypes.data, dt, info.ctypes.data))
        return info

    def pf_grad_q(self, U: np.ndarray, pf, dt: float):
        c = self.case
        dim = c.dim
        n = [c.n[0], c.n[1], c.n[2] if dim == 3 else 1]
        out = []
        for d in range(3):
            if d < dim:
                shp = [n[2] + (d == 2), n[1] + (d == 1), n[0] + (d == 0)]
                out.append(np.zeros(shp))
            else:
                out.append(None)
        info = np.zeros(6)
        ptr = [o.ctypes.data if o is not None else None for o in out]
        self._call(self.lib.cmp_pf_grad_q(self._c, self._pf(pf), U.ctypes.data, dt, ptr[0], ptr[1], ptr[2],
                                          info.ctypes.data))
        return out[:dim], info

    def pf_dudt(self, U: np.ndarray, pf, gq) -> np.ndarray:
        """Phase-Field right-hand side of U (ghosts filled here) for the face gradients gq (one array
        per direction, as pf_grad_q returns them); padded, valid cells written."""
        out = np.zeros_like(U)
        g = [np.ascontiguousarray(x) for x in gq]
        ptr = [g[d].ctypes.data if d < len(g) else None for d in range(3)]
        self._call(self.lib.cmp_pf_dudt(self._c, self._pf(pf), U.ctypes.data, ptr[0], ptr[1], ptr[2],
                                        out.ctypes.data))
        return out

    def advance_pf(self, U: np.ndarray, pf, nsteps: int, stop_time: float = 1e300, t0: float = 0.0):
        t = ctypes.c_double(t0)
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        n = self._call(self.lib.cmp_advance_pf(self._c, self._pf(pf), U.ctypes.data, nsteps, stop_time,
                                               ctypes.byref(t), dts.ctypes.data))
        return t.value, dts[:n]

    # ---- multi-level advance (reference-header build only) ---------------------------------------
    def amr_advance(self, boxes, states, nsteps: int, stop_time: float = 1e300, t0: float = 0.0):
        """boxes: [(lev, lo, hi)], states: padded float64 arrays (advanced in place); self's case is
        level 0."""
        if self.kind != "reference":
            raise RuntimeError("the multi-level advance is in the reference-header oracle only")
        arr = (AmrBox * len(boxes))()
        for b, (lev, lo, hi) in enumerate(boxes):
            arr[b].lev = lev
            for d in range(3):
                arr[b].lo[d] = lo[d]
                arr[b].hi[d] = hi[d]
        for U in states:
            assert U.flags.c_contiguous and U.dtype == np.float64
        ptrs = (ctypes.c_void_p * len(states))(*[U.ctypes.data for U in states])
        t = ctypes.c_double(t0)
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        nlev = 1 + max(b[0] for b in boxes)
        n = self._call(self.lib.cmp_amr_advance(self._c, nlev, arr, len(boxes), ptrs, nsteps, stop_time,
                                                ctypes.byref(t), dts.ctypes.data))
        return t.value, dts[:n]

    # ---- refinement tags (reference-header build only) ---------------------------------------------
    def tag(self, U: np.ndarray, criteria, cv=(1.0, 1.0)) -> np.ndarray:
        """ErrorEst tags (1/0) of the valid cells, shape (nz, ny, nx), of the ghost-filled padded U for
        criteria given as (var, derived, kind, v0, v1) tuples."""
        if self.kind != "reference":
            raise RuntimeError("tagging is in the reference-header oracle only")
        c = self.case
        nz = c.n[2] if c.dim == 3 else 1
        tags = np.zeros((nz, c.n[1], c.n[0]), dtype=np.uint8)
        arr = (TagCrit * max(1, len(criteria)))(*[TagCrit(*t) for t in criteria])
        cvv = np.array(cv, dtype=np.float64)
        assert U.flags.c_contiguous and U.dtype == np.float64
        self._call(self.lib.cmp_tag(self._c, cvv.ctypes.data, U.ctypes.data, ctypes.addressof(arr), len(criteria),
                                    tags.ctypes.data))
        return tags

    def derive(self, U: np.ndarray, vars_derived, cv=(1.0, 1.0)) -> np.ndarray:
        """Plot variables (var, derived) of the valid cells of the ghost-filled padded U, shape
        (nvars, nz, ny, nx) (reference-header build only)."""
        if self.kind != "reference":
            raise RuntimeError("derived variables are in the reference-header oracle only")
        c = self.case
        nz = c.n[2] if c.dim == 3 else 1
        out = np.zeros((len(vars_derived), nz, c.n[1], c.n[0]))
        v = np.array([x for x, _ in vars_derived] or [0], dtype=np.int32)
        dflag = np.array([y for _, y in vars_derived] or [0], dtype=np.int32)
        cvv = np.array(cv, dtype=np.float64)
        self._call(self.lib.cmp_derive(self._c, cvv.ctypes.data, U.ctypes.data, v.ctypes.data, dflag.ctypes.data,
                                       len(vars_derived), out.ctypes.data))
        return out

    # ---- bound-preserving path (FiniteVolume.ID_Bound = 1; reference-header build only) -----------
    def energy_bound_min(self, U: np.ndarray) -> float:
        """MinEnergyBound of the valid cells of U."""
        out = ctypes.c_double()
        self._call(self.lib.cmp_energy_bound_min(self._c, U.ctypes.data, ctypes.byref(out)))
        return out.value

    def bound_restarts(self) -> int:
        """Steps the last advance took again after a failed energy check."""
        return int(self.lib.cmp_bound_restarts())

    def threads(self) -> int:
        return int(self.lib.cmp_threads())

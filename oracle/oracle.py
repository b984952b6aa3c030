"""ctypes wrapper of the FP64 CPU oracle (liboracle: nelson_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as part of the nelson_b200 product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnelson_oracle.so")

KIND_BA, KIND_LINEAR = 0, 1
TRACE_STRIDE = 8

LM_REASONS = ["SuccessAtStart", "SuccessSmallIncrement", "SuccessEpsB", "SuccessSmallResiduals",
              "SolverFailure", "MaxIterationReached", "MaxSubIterationReached"]
GN_REASONS = LM_REASONS[:6]


class LMSettings(C.Structure):
    """LevenbergMarquardtSettings with the defaults of nelson/LevenbergMarquardt.cpp:6-19."""
    _fields_ = [("maxNumIt", C.c_int), ("maxNumSubIt", C.c_int), ("minNumIt", C.c_int),
                ("epsBVector", C.c_double), ("epsIncSquare", C.c_double), ("epsChi2", C.c_double),
                ("tau", C.c_double), ("penaltyV", C.c_double), ("initV", C.c_double),
                ("maxScaleFactor", C.c_double), ("minScaleFactor", C.c_double)]

    def __init__(self, **kw):
        d = dict(maxNumIt=100, maxNumSubIt=10, minNumIt=0, epsBVector=1e-15, epsIncSquare=1e-30,
                 epsChi2=1e-15, tau=1e-3, penaltyV=2.0, initV=2.0, maxScaleFactor=2.0 / 3.0,
                 minScaleFactor=1.0 / 3.0)
        d.update(kw)
        super().__init__(**d)


class GNSettings(C.Structure):
    """GaussNewtonSettings with the defaults of nelson/GaussNewton.cpp:12-22."""
    _fields_ = [("maxNumIt", C.c_int), ("minNumIt", C.c_int), ("epsBVector", C.c_double),
                ("epsIncSquare", C.c_double), ("epsChi2", C.c_double), ("absLambda", C.c_double),
                ("relLambda", C.c_double)]

    def __init__(self, **kw):
        d = dict(maxNumIt=100, minNumIt=0, epsBVector=1e-15, epsIncSquare=1e-30, epsChi2=1e-15,
                 absLambda=0.0, relLambda=0.0)
        d.update(kw)
        super().__init__(**d)


_lib = None


def build() -> str:
    """Compile liboracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE, "liborc"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        P = np.ctypeslib.ndpointer
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i, i, i, i, i, i, i, i]
        L.orc_destroy.argtypes = [vp]
        for name in ["orc_max_abs_hdiag", "orc_inc_sqnorm", "orc_max_abs_b", "orc_chi2"]:
            getattr(L, name).restype = d
            getattr(L, name).argtypes = [vp]
        L.orc_rho.restype = d
        L.orc_rho.argtypes = [vp, d, d]
        L.orc_set_intrinsics.argtypes = [vp, d, d, d]
        L.orc_compute_increment.argtypes = [vp, d, d]
        L.orc_adjoint_ba.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.orc_update.argtypes = [vp, i, C.POINTER(d)]
        L.orc_lm_solve.argtypes = [vp, C.POINTER(LMSettings), vp, i, C.POINTER(i), vp]
        L.orc_gn_solve.argtypes = [vp, C.POINTER(GNSettings), vp, i, C.POINTER(i), vp]
        L.orc_dense_cholesky.argtypes = [vp, i, i, i]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One nelson problem (DoubleSection + SolverCholeskySchur + LM/GN) on the CPU."""

    def __init__(self, kind, bu, bv, nu_var, nu_fix, nv_var, nv_fix, threads=0):
        self.L = lib()
        self.kind, self.bu, self.bv = kind, bu, bv
        self.nu_var, self.nu_fix, self.nv_var, self.nv_fix = nu_var, nu_fix, nv_var, nv_fix
        h = self.L.orc_create(kind, bu, bv, nu_var, nu_fix, nv_var, nv_fix, threads)
        if not h:
            raise ValueError("orc_create rejected the problem description")
        # kept as a pointer object: the entry points declared without argtypes
        # would pass a plain Python int as a 32-bit C int and cut the address
        self.h = C.c_void_p(h)
        self.ne = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def _chk(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed with {rc}")

    # -- construction -----------------------------------------------------------------------
    @classmethod
    def from_ba(cls, prob, threads=0, perm=None):
        o = cls(KIND_BA, prob.bc, 3, prob.nc_var, prob.nc_fix, prob.np_var, prob.np_fix, threads)
        o._chk(o.L.orc_set_intrinsics(o.h, prob.f, prob.cx, prob.cy), "set_intrinsics")
        o.set_params(prob.cams, prob.pts)
        ne = prob.ne
        cf = None if prob.cam_fixed is None else np.ascontiguousarray(prob.cam_fixed, np.int32)
        pf = None if prob.pt_fixed is None else np.ascontiguousarray(prob.pt_fixed, np.int32)
        w = None if prob.weight is None else np.ascontiguousarray(prob.weight, np.float64)
        o._chk(o.L.orc_add_ba_edges(o.h, ne, _p(prob.cam_idx), _p(cf), _p(prob.pt_idx), _p(pf),
                                    _p(np.ascontiguousarray(prob.obs, np.float64)), _p(w)),
               "add_ba_edges")
        o.ne = ne
        if perm is not None:
            o.set_user2internal(perm)
        o.structure_ready()
        return o

    @classmethod
    def from_linear(cls, lp, threads=0, perm=None):
        o = cls(KIND_LINEAR, lp.bu, lp.bv, lp.nu_var, lp.nu_fix, lp.nv_var, lp.nv_fix, threads)
        o.set_params(lp.u, lp.v)
        for e in lp.edges:
            A1 = np.ascontiguousarray(e.A1, np.float64)
            A2 = None if e.A2 is None else np.ascontiguousarray(e.A2, np.float64)
            z = np.ascontiguousarray(e.z, np.float64)
            o._chk(o.L.orc_add_linear_edge(o.h, e.type, e.id1, 0, max(e.id2, 0), 0, len(z), _p(A1),
                                           _p(A2), _p(z)), "add_linear_edge")
            o.ne += 1
        if perm is not None:
            o.set_user2internal(perm)
        o.structure_ready()
        return o

    def set_user2internal(self, perm):
        perm = np.ascontiguousarray(perm, np.int32)
        self._chk(self.L.orc_set_user2internal_u(self.h, _p(perm)), "set_user2internal")

    def structure_ready(self):
        self._chk(self.L.orc_structure_ready(self.h), "structure_ready")
        c = np.zeros(4, np.int32)
        self.L.orc_get_counts(self.h, _p(c))
        self.nU, self.nV, self.nW, self.ne = [int(x) for x in c]

    # -- parameters ---------------------------------------------------------------------------
    def set_params(self, u, v):
        u = np.ascontiguousarray(u, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        self._chk(self.L.orc_set_params(self.h, _p(u), _p(v)), "set_params")

    def get_params(self):
        u = np.zeros((self.nu_var + self.nu_fix, self.bu))
        v = np.zeros((self.nv_var + self.nv_fix, self.bv))
        self.L.orc_get_params(self.h, _p(u), _p(v))
        return u, v

    def camera_state(self):
        s = np.zeros((self.nu_var + self.nu_fix, 16))
        self._chk(self.L.orc_get_camera_state(self.h, _p(s)), "camera_state")
        return s

    # -- structure ----------------------------------------------------------------------------
    def patterns(self):
        u = np.zeros((self.nU, 2), np.int32)
        v = np.zeros((self.nV, 2), np.int32)
        w = np.zeros((self.nW, 2), np.int32)
        self.L.orc_get_patterns(self.h, _p(u), _p(v), _p(w))
        return u, v, w

    def edge_uids(self):
        a = np.zeros(self.ne, np.int32)
        b = np.zeros(self.ne, np.int32)
        c = np.zeros(self.ne, np.int32)
        self.L.orc_get_edge_uids(self.h, _p(a), _p(b), _p(c))
        return a, b, c

    # -- problem concept ----------------------------------------------------------------------
    def update(self, hessian=True):
        chi2 = C.c_double()
        self._chk(self.L.orc_update(self.h, 1 if hessian else 0, C.byref(chi2)), "update")
        return chi2.value

    def hessian(self):
        bu, bv = self.bu, self.bv
        U = np.zeros((self.nU, bu, bu))
        V = np.zeros((self.nV, bv, bv))
        W = np.zeros((self.nW, bu, bv))
        bU = np.zeros(self.nu_var * bu)
        bV = np.zeros(self.nv_var * bv)
        self.L.orc_get_hessian(self.h, _p(U), _p(V), _p(W), _p(bU), _p(bV))
        return U, V, W, bU, bV

    def residuals(self, dr=2):
        r = np.zeros((self.ne, dr))
        self.L.orc_get_residuals(self.h, _p(r))
        return r

    def max_abs_hdiag(self):
        return self.L.orc_max_abs_hdiag(self.h)

    def compute_increment(self, rel, abs_):
        return bool(self.L.orc_compute_increment(self.h, rel, abs_))

    def increment(self):
        du = np.zeros(self.nu_var * self.bu)
        dv = np.zeros(self.nv_var * self.bv)
        self.L.orc_get_increment(self.h, _p(du), _p(dv))
        return du, dv

    def schur(self):
        n = C.c_int()
        self.L.orc_get_schur(self.h, None, None, C.byref(n))
        S = np.zeros((n.value, n.value))
        bS = np.zeros(n.value)
        self.L.orc_get_schur(self.h, _p(S), _p(bS), C.byref(n))
        return S, bS

    def inc_sqnorm(self):
        return self.L.orc_inc_sqnorm(self.h)

    def oplus(self):
        self.L.orc_oplus(self.h)

    def backup(self):
        self.L.orc_backup(self.h)

    def rollback(self):
        self.L.orc_rollback(self.h)

    def chi2(self):
        return self.L.orc_chi2(self.h)

    def max_abs_b(self):
        return self.L.orc_max_abs_b(self.h)

    def rho(self, mu, old_chi2):
        return self.L.orc_rho(self.h, mu, old_chi2)

    # -- solvers ------------------------------------------------------------------------------
    def lm_solve(self, settings=None, trace_cap=4096):
        s = settings or LMSettings()
        tr = np.zeros((trace_cap, TRACE_STRIDE))
        n = C.c_int()
        its = np.zeros(2, np.int32)
        reason = self.L.orc_lm_solve(self.h, C.byref(s), _p(tr), trace_cap, C.byref(n), _p(its))
        if reason < 0:
            raise RuntimeError("orc_lm_solve failed")
        return LM_REASONS[reason], tr[:n.value].copy(), int(its[0]), int(its[1])

    def adjoint(self, dL_dpts=None, dL_dcams=None):
        """FP64 implicit-function adjoint at the current (converged)
        parameters: (dL/dobs (ne, 2), dL/dweight (ne,), mu_cams, mu_pts)."""
        g_obs = np.zeros((self.ne, 2))
        g_w = np.zeros(self.ne)
        mu_c = np.zeros((self.nu_var, self.bu))
        mu_p = np.zeros((self.nv_var, 3))
        dc = None if dL_dcams is None else np.ascontiguousarray(dL_dcams, np.float64).reshape(self.nu_var, self.bu)
        dp = None if dL_dpts is None else np.ascontiguousarray(dL_dpts, np.float64).reshape(self.nv_var, 3)
        rc = self.L.orc_adjoint_ba(self.h, _p(dc), _p(dp), _p(g_obs), _p(g_w), _p(mu_c), _p(mu_p))
        if rc != 1:
            raise RuntimeError(f"orc_adjoint_ba failed ({rc})")
        return g_obs, g_w, mu_c, mu_p

    def gn_solve(self, settings=None, trace_cap=4096):
        s = settings or GNSettings()
        tr = np.zeros((trace_cap, TRACE_STRIDE))
        n = C.c_int()
        its = np.zeros(2, np.int32)
        reason = self.L.orc_gn_solve(self.h, C.byref(s), _p(tr), trace_cap, C.byref(n), _p(its))
        if reason < 0:
            raise RuntimeError("orc_gn_solve failed")
        return GN_REASONS[reason], tr[:n.value].copy(), int(its[0])


def dense_cholesky(A: np.ndarray, threads=0) -> bool:
    """In-place lower Cholesky of a row-major float64 matrix."""
    assert A.dtype == np.float64 and A.flags.c_contiguous
    n = A.shape[0]
    return bool(lib().orc_dense_cholesky(_p(A), n, n, threads))

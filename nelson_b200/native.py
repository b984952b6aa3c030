"""ctypes binding of libnelson_b200.so (the C ABI of include/nelson_b200.h).

`BAProblemGPU` mirrors nelson's DoubleSection + SolverCholeskySchur +
LevenbergMarquardt / GaussNewton interface on the device-resident engine.
There is no CPU fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

PREC_FP64, PREC_MIXED = 0, 1
SOLVER_DENSE, SOLVER_ENVELOPE = 0, 1
TRACE_STRIDE = 8
REASONS = ["SuccessAtStart", "SuccessSmallIncrement", "SuccessEpsB", "SuccessSmallResiduals",
           "SolverFailure", "MaxIterationReached", "MaxSubIterationReached"]


class NelsonError(RuntimeError):
    pass


class ProblemDesc(C.Structure):
    _fields_ = [("bc", C.c_int), ("nc_var", C.c_int), ("nc_fix", C.c_int), ("np_var", C.c_int),
                ("np_fix", C.c_int), ("precision", C.c_int), ("f", C.c_double), ("cx", C.c_double),
                ("cy", C.c_double), ("refine_sweeps", C.c_int), ("device", C.c_int)]


class LMSettings(C.Structure):
    """nl_lm_settings; defaults of nelson/LevenbergMarquardt.cpp:6-19."""
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
    """nl_gn_settings; defaults of nelson/GaussNewton.cpp:12-22."""
    _fields_ = [("maxNumIt", C.c_int), ("minNumIt", C.c_int), ("epsBVector", C.c_double),
                ("epsIncSquare", C.c_double), ("epsChi2", C.c_double), ("absLambda", C.c_double),
                ("relLambda", C.c_double)]

    def __init__(self, **kw):
        d = dict(maxNumIt=100, minNumIt=0, epsBVector=1e-15, epsIncSquare=1e-30, epsChi2=1e-15,
                 absLambda=0.0, relLambda=0.0)
        d.update(kw)
        super().__init__(**d)


class SolveReport(C.Structure):
    _fields_ = [("reason", C.c_int), ("iterations", C.c_int), ("subiterations", C.c_int),
                ("n_trace", C.c_int), ("chi2", C.c_double), ("mu", C.c_double), ("device_ms", C.c_double)]


class PhaseTimes(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("vinv_ms", "wvinv_bs_ms", "schur_ms", "factor_ms", "solve_ms",
                                          "backsub_ms", "total_ms", "eval_ms", "update_ms")] + \
        [("update_launches", C.c_int), ("update_flop", C.c_double), ("update_bytes", C.c_double),
         ("panel_ms", C.c_float), ("panels", C.c_int), ("wait_ms", C.c_float), ("first_ms", C.c_float)]


class AdjointReport(C.Structure):
    _fields_ = [("ok", C.c_int), ("sweeps", C.c_int), ("grad_norm", C.c_double), ("residual_norm", C.c_double),
                ("device_ms", C.c_double)]


class UnrollReport(C.Structure):
    _fields_ = [("steps", C.c_int), ("ok", C.c_int), ("chi2", C.c_double), ("device_ms", C.c_double)]


class SolverDesc(C.Structure):
    _fields_ = [("bu", C.c_int), ("nu", C.c_int), ("nv", C.c_int), ("nU", C.c_int), ("nV", C.c_int),
                ("nW", C.c_int), ("precision", C.c_int), ("refine_sweeps", C.c_int), ("device", C.c_int)]


EXPORTS = [
    "nl_create", "nl_destroy", "nl_set_params", "nl_get_params", "nl_get_camera_state", "nl_add_ba_edges",
    "nl_set_user2internal_u", "nl_structure_ready", "nl_set_observations", "nl_get_counts", "nl_get_patterns",
    "nl_get_edge_uids", "nl_update", "nl_get_hessian", "nl_solver_init", "nl_max_abs_hdiag",
    "nl_compute_increment", "nl_get_increment", "nl_inc_sqnorm", "nl_get_schur", "nl_oplus", "nl_backup",
    "nl_rollback", "nl_max_abs_b", "nl_chi2", "nl_rho", "nl_lm_solve", "nl_gn_solve", "nl_phase_timings",
    "nl_kernel_launches", "nl_solver_create", "nl_solver_destroy", "nl_solver_set_hessian",
    "nl_solver_max_abs_hdiag", "nl_solver_compute_increment", "nl_selftest_tc_update", "nl_ba_cost_noalloc",
    "nl_adjoint", "nl_lm_solve_batch", "nl_set_timing_detail", "nl_set_solver_kind", "nl_solver_set_kind",
    "nl_permute_rcm_u", "nl_get_user2internal_u", "nl_rcm_order",
    "nl_permute_amd_u", "nl_amd_order_camera_graph", "nl_amd_order", "nl_symbolic_fill",
    "nl_set_wait_limit", "nl_check_wait_timeout", "nl_unroll_record", "nl_unroll_adjoint",
    "nl_batch_create", "nl_batch_destroy", "nl_batch_autotune", "nl_batch_lm_solve",
    "nl_pose2d_create", "nl_pose2d_destroy", "nl_pose2d_set_poses", "nl_pose2d_get_poses", "nl_pose2d_add_edge",
    "nl_pose2d_set_user2internal", "nl_pose2d_permute_amd", "nl_pose2d_permute_rcm", "nl_pose2d_structure_ready",
    "nl_pose2d_set_solver_kind", "nl_pose2d_update", "nl_pose2d_get_hessian", "nl_pose2d_lm_solve",
    "nl_pose2d_gn_solve",
    "nl_section_create", "nl_section_destroy", "nl_section_add_edges", "nl_section_set_user2internal_u",
    "nl_section_permute_amd_u", "nl_section_get_user2internal_u", "nl_section_structure_ready",
    "nl_section_get_counts", "nl_section_layout",
    "nl_section_get_patterns", "nl_section_set_callbacks", "nl_section_set_solver_kind", "nl_section_update",
    "nl_section_get_hessian", "nl_section_compute_increment", "nl_section_lm_solve", "nl_section_gn_solve",
    "nl_selftest_tc_update_k",
    "nl_status_string",
    "nl_version",
]

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the CUDA library (building it first if needed).  Raises when it cannot."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_build.LIB):
        if not build_if_missing:
            raise NelsonError(f"{_build.LIB} is missing; run nelson_b200.build.build()")
        _build.build()
    L = C.CDLL(_build.LIB)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.nl_create.argtypes = [C.POINTER(ProblemDesc), C.POINTER(vp)]
    L.nl_status_string.restype = C.c_char_p
    L.nl_version.restype = C.c_char_p
    L.nl_compute_increment.argtypes = [vp, d, d, C.POINTER(i)]
    L.nl_rho.argtypes = [vp, d, d, C.POINTER(d)]
    L.nl_update.argtypes = [vp, i, C.POINTER(d)]
    L.nl_lm_solve.argtypes = [vp, C.POINTER(LMSettings), C.POINTER(SolveReport), vp, i]
    L.nl_gn_solve.argtypes = [vp, C.POINTER(GNSettings), C.POINTER(SolveReport), vp, i]
    L.nl_solver_create.argtypes = [C.POINTER(SolverDesc), vp, vp, vp, C.POINTER(vp)]
    L.nl_solver_compute_increment.argtypes = [vp, d, d, vp, vp, C.POINTER(i)]
    L.nl_selftest_tc_update.argtypes = [i, C.c_ulonglong, i, C.POINTER(d)]
    L.nl_selftest_tc_update_k.argtypes = [i, i, C.c_ulonglong, i, i, C.POINTER(d), C.POINTER(d)]
    L.nl_lm_solve_batch.argtypes = [C.POINTER(vp), i, C.POINTER(LMSettings), vp, vp]
    L.nl_adjoint.argtypes = [vp, vp, vp, i, vp, vp, vp, vp, C.POINTER(AdjointReport)]
    L.nl_ba_cost_noalloc.argtypes = [i, i, vp, vp, vp, vp, vp, vp, d, d, d, vp, vp]
    L.nl_set_wait_limit.argtypes = [vp, C.c_longlong]
    L.nl_unroll_record.argtypes = [vp, i, vp, C.POINTER(UnrollReport)]
    L.nl_batch_create.argtypes = [C.POINTER(vp), i, C.POINTER(vp)]
    L.nl_batch_destroy.argtypes = [vp]
    L.nl_batch_autotune.argtypes = [vp, C.POINTER(LMSettings), C.POINTER(i), C.POINTER(i)]
    L.nl_batch_lm_solve.argtypes = [vp, C.POINTER(LMSettings), i, i, vp, vp, C.POINTER(d)]
    L.nl_unroll_adjoint.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.POINTER(UnrollReport)]
    L.nl_check_wait_timeout.argtypes = [vp]
    L.nl_pose2d_create.argtypes = [i, i, i, i, C.POINTER(vp)]
    L.nl_pose2d_destroy.argtypes = [vp]
    L.nl_pose2d_set_poses.argtypes = [vp, vp, vp]
    L.nl_pose2d_get_poses.argtypes = [vp, vp]
    L.nl_pose2d_add_edge.argtypes = [vp, i, i, i, i, i, vp, vp, vp]
    L.nl_pose2d_set_user2internal.argtypes = [vp, vp]
    L.nl_pose2d_permute_amd.argtypes = [vp]
    L.nl_pose2d_permute_rcm.argtypes = [vp]
    L.nl_pose2d_structure_ready.argtypes = [vp]
    L.nl_pose2d_set_solver_kind.argtypes = [vp, i]
    L.nl_pose2d_get_hessian.argtypes = [vp, vp, vp]
    L.nl_section_create.argtypes = [i, i, i, i, i, C.POINTER(vp)]
    L.nl_section_destroy.argtypes = [vp]
    L.nl_section_add_edges.argtypes = [vp, i, vp, vp, vp, vp]
    L.nl_section_set_user2internal_u.argtypes = [vp, vp]
    L.nl_section_permute_amd_u.argtypes = [vp]
    L.nl_section_get_user2internal_u.argtypes = [vp, vp]
    L.nl_section_structure_ready.argtypes = [vp]
    L.nl_section_get_counts.argtypes = [vp, vp, vp, vp, vp]
    L.nl_section_layout.argtypes = [vp, vp, vp]
    L.nl_section_get_patterns.argtypes = [vp, vp, vp]
    L.nl_section_set_callbacks.argtypes = [vp, C.POINTER(SectionCallbacks)]
    L.nl_section_set_solver_kind.argtypes = [vp, i]
    L.nl_section_update.argtypes = [vp, i, C.POINTER(d)]
    L.nl_section_get_hessian.argtypes = [vp, vp, vp, vp, vp, vp]
    L.nl_section_compute_increment.argtypes = [vp, d, d, vp, vp, C.POINTER(i)]
    L.nl_section_lm_solve.argtypes = [vp, C.POINTER(LMSettings), C.POINTER(SolveReport), vp, i]
    L.nl_section_gn_solve.argtypes = [vp, C.POINTER(GNSettings), C.POINTER(SolveReport), vp, i]
    L.nl_pose2d_update.argtypes = [vp, i, C.POINTER(d)]
    L.nl_pose2d_lm_solve.argtypes = [vp, C.POINTER(LMSettings), C.POINTER(SolveReport), vp, i]
    L.nl_pose2d_gn_solve.argtypes = [vp, C.POINTER(GNSettings), C.POINTER(SolveReport), vp, i]
    for name in EXPORTS:  # fails loudly if the library lacks an entry point
        if name not in ("nl_status_string", "nl_version"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _chk(L, rc, what):
    if rc != 0:
        raise NelsonError(f"{what}: {L.nl_status_string(rc).decode()} ({rc})")


class BAProblemGPU:
    """Device-resident BA section: DoubleSection<cameras, points> with the
    projection EdgeBinaryUV, solved by the CUDA SolverCholeskySchur."""

    def __init__(self, bc, nc_var, np_var, nc_fix=0, np_fix=0, precision=PREC_FP64, f=500.0, cx=320.0,
                 cy=240.0, refine_sweeps=-1, device=0):
        self.L = load()
        self.bc, self.nc_var, self.np_var, self.nc_fix, self.np_fix = bc, nc_var, np_var, nc_fix, np_fix
        self.precision = precision
        desc = ProblemDesc(bc=bc, nc_var=nc_var, nc_fix=nc_fix, np_var=np_var, np_fix=np_fix,
                           precision=precision, f=f, cx=cx, cy=cy, refine_sweeps=refine_sweeps, device=device)
        h = C.c_void_p()
        _chk(self.L, self.L.nl_create(C.byref(desc), C.byref(h)), "nl_create")
        self.h = h
        self.ne = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.nl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc, what):
        _chk(self.L, rc, what)

    @classmethod
    def from_ba(cls, prob, precision=PREC_FP64, perm=None, refine_sweeps=-1, device=0):
        g = cls(prob.bc, prob.nc_var, prob.np_var, prob.nc_fix, prob.np_fix, precision, prob.f, prob.cx, prob.cy,
                refine_sweeps, device)
        g.set_params(prob.cams, prob.pts)
        cf = None if prob.cam_fixed is None else np.ascontiguousarray(prob.cam_fixed, np.int32)
        pf = None if prob.pt_fixed is None else np.ascontiguousarray(prob.pt_fixed, np.int32)
        w = None if prob.weight is None else np.ascontiguousarray(prob.weight, np.float64)
        g._c(g.L.nl_add_ba_edges(g.h, prob.ne, _p(np.ascontiguousarray(prob.cam_idx, np.int32)), _p(cf),
                                 _p(np.ascontiguousarray(prob.pt_idx, np.int32)), _p(pf),
                                 _p(np.ascontiguousarray(prob.obs, np.float64)), _p(w)), "nl_add_ba_edges")
        if isinstance(perm, str) and perm == "rcm":
            g._c(g.L.nl_permute_rcm_u(g.h), "nl_permute_rcm_u")
        elif isinstance(perm, str) and perm == "amd":
            g._c(g.L.nl_permute_amd_u(g.h), "nl_permute_amd_u")
        elif perm is not None:
            g._c(g.L.nl_set_user2internal_u(g.h, _p(np.ascontiguousarray(perm, np.int32))), "set_user2internal")
        g.structure_ready()
        return g

    def structure_ready(self):
        self._c(self.L.nl_structure_ready(self.h), "nl_structure_ready")
        c = np.zeros(4, np.int32)
        self._c(self.L.nl_get_counts(self.h, _p(c)), "nl_get_counts")
        self.nU, self.nV, self.nW, self.ne = [int(x) for x in c]

    def set_params(self, cams, pts):
        self._c(self.L.nl_set_params(self.h, _p(np.ascontiguousarray(cams, np.float64)),
                                     _p(np.ascontiguousarray(pts, np.float64))), "nl_set_params")

    def set_observations(self, obs, weight=None):
        w = None if weight is None else np.ascontiguousarray(weight, np.float64)
        self._c(self.L.nl_set_observations(self.h, _p(np.ascontiguousarray(obs, np.float64)), _p(w)),
                "nl_set_observations")

    def get_params(self):
        u = np.zeros((self.nc_var + self.nc_fix, self.bc))
        v = np.zeros((self.np_var + self.np_fix, 3))
        self._c(self.L.nl_get_params(self.h, _p(u), _p(v)), "nl_get_params")
        return u, v

    def camera_state(self):
        s = np.zeros((self.nc_var + self.nc_fix, 16))
        self._c(self.L.nl_get_camera_state(self.h, _p(s)), "nl_get_camera_state")
        return s

    def patterns(self):
        u = np.zeros((self.nU, 2), np.int32)
        v = np.zeros((self.nV, 2), np.int32)
        w = np.zeros((self.nW, 2), np.int32)
        self._c(self.L.nl_get_patterns(self.h, _p(u), _p(v), _p(w)), "nl_get_patterns")
        return u, v, w

    def edge_uids(self):
        a, b, c = (np.zeros(self.ne, np.int32) for _ in range(3))
        self._c(self.L.nl_get_edge_uids(self.h, _p(a), _p(b), _p(c)), "nl_get_edge_uids")
        return a, b, c

    def update(self, hessian=True):
        chi2 = C.c_double()
        self._c(self.L.nl_update(self.h, 1 if hessian else 0, C.byref(chi2)), "nl_update")
        return chi2.value

    def hessian(self):
        bu = self.bc
        U = np.zeros((self.nU, bu, bu))
        V = np.zeros((self.nV, 3, 3))
        W = np.zeros((self.nW, bu, 3))
        bU = np.zeros(self.nc_var * bu)
        bV = np.zeros(self.np_var * 3)
        self._c(self.L.nl_get_hessian(self.h, _p(U), _p(V), _p(W), _p(bU), _p(bV)), "nl_get_hessian")
        return U, V, W, bU, bV

    def max_abs_hdiag(self):
        v = C.c_double()
        self._c(self.L.nl_max_abs_hdiag(self.h, C.byref(v)), "nl_max_abs_hdiag")
        return v.value

    def compute_increment(self, rel, abs_):
        ok = C.c_int()
        self._c(self.L.nl_compute_increment(self.h, rel, abs_, C.byref(ok)), "nl_compute_increment")
        return bool(ok.value)

    def increment(self):
        du = np.zeros(self.nc_var * self.bc)
        dv = np.zeros(self.np_var * 3)
        self._c(self.L.nl_get_increment(self.h, _p(du), _p(dv)), "nl_get_increment")
        return du, dv

    def inc_sqnorm(self):
        v = C.c_double()
        self._c(self.L.nl_inc_sqnorm(self.h, C.byref(v)), "nl_inc_sqnorm")
        return v.value

    def schur(self):
        n = C.c_int()
        self._c(self.L.nl_get_schur(self.h, None, None, C.byref(n)), "nl_get_schur")
        S = np.zeros((n.value, n.value))
        bS = np.zeros(n.value)
        self._c(self.L.nl_get_schur(self.h, _p(S), _p(bS), C.byref(n)), "nl_get_schur")
        return S, bS

    def oplus(self):
        self._c(self.L.nl_oplus(self.h), "nl_oplus")

    def backup(self):
        self._c(self.L.nl_backup(self.h), "nl_backup")

    def rollback(self):
        self._c(self.L.nl_rollback(self.h), "nl_rollback")

    def chi2(self):
        v = C.c_double()
        self._c(self.L.nl_chi2(self.h, C.byref(v)), "nl_chi2")
        return v.value

    def max_abs_b(self):
        v = C.c_double()
        self._c(self.L.nl_max_abs_b(self.h, C.byref(v)), "nl_max_abs_b")
        return v.value

    def rho(self, mu, old_chi2):
        v = C.c_double()
        self._c(self.L.nl_rho(self.h, mu, old_chi2, C.byref(v)), "nl_rho")
        return v.value

    def lm_solve(self, settings=None, trace_cap=4096, report=False):
        s = settings or LMSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_lm_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_lm_solve")
        out = (REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations, rep.subiterations)
        if report:
            return out + ({n: getattr(rep, n) for n, _ in SolveReport._fields_},)
        return out

    def gn_solve(self, settings=None, trace_cap=4096):
        s = settings or GNSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_gn_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_gn_solve")
        return REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations

    def adjoint(self, dL_dpts=None, dL_dcams=None, sweeps=3, want_mu=False):
        """Implicit-function adjoint at the current (converged) solution:
        returns (dL/dobs (ne, 2), dL/dweight (ne,), report[, mu_cams, mu_pts])."""
        g_obs = np.zeros((self.ne, 2))
        g_w = np.zeros(self.ne)
        mu_c = np.zeros((self.nc_var, self.bc)) if want_mu else None
        mu_p = np.zeros((self.np_var, 3)) if want_mu else None
        dc = None if dL_dcams is None else np.ascontiguousarray(dL_dcams, np.float64).reshape(self.nc_var, self.bc)
        dp = None if dL_dpts is None else np.ascontiguousarray(dL_dpts, np.float64).reshape(self.np_var, 3)
        rep = AdjointReport()
        self._c(self.L.nl_adjoint(self.h, _p(dc), _p(dp), sweeps, _p(g_obs), _p(g_w), _p(mu_c), _p(mu_p),
                                  C.byref(rep)), "nl_adjoint")
        r = {n: getattr(rep, n) for n, _ in AdjointReport._fields_}
        return (g_obs, g_w, r, mu_c, mu_p) if want_mu else (g_obs, g_w, r)

    def unroll_record(self, mus):
        """nl_unroll_record: len(mus) damped steps from the current parameters
        with per-step checkpoints; returns the report as a dict."""
        m = np.ascontiguousarray(mus, np.float64)
        rep = UnrollReport()
        self._c(self.L.nl_unroll_record(self.h, int(m.size), _p(m), C.byref(rep)), "nl_unroll_record")
        return {n: getattr(rep, n) for n, _ in UnrollReport._fields_}

    def unroll_adjoint(self, dL_dpts=None, dL_dcams=None):
        """nl_unroll_adjoint: gradients of L(x_K) through the recorded steps:
        (dL/dobs (ne, 2), dL/dweight (ne,), dL/dcams0 (nc_var, bc), dL/dpts0
        (np_var, 3), report)."""
        g_obs = np.zeros((self.ne, 2))
        g_w = np.zeros(self.ne)
        g_c = np.zeros((self.nc_var, self.bc))
        g_p = np.zeros((self.np_var, 3))
        dc = None if dL_dcams is None else np.ascontiguousarray(dL_dcams, np.float64).reshape(self.nc_var, self.bc)
        dp = None if dL_dpts is None else np.ascontiguousarray(dL_dpts, np.float64).reshape(self.np_var, 3)
        rep = UnrollReport()
        self._c(self.L.nl_unroll_adjoint(self.h, _p(dc), _p(dp), _p(g_obs), _p(g_w), _p(g_c), _p(g_p),
                                         C.byref(rep)), "nl_unroll_adjoint")
        return g_obs, g_w, g_c, g_p, {n: getattr(rep, n) for n, _ in UnrollReport._fields_}

    def phase_times(self):
        t = PhaseTimes()
        self._c(self.L.nl_phase_timings(self.h, C.byref(t)), "nl_phase_timings")
        return {n: getattr(t, n) for n, _ in PhaseTimes._fields_}

    def user2internal(self):
        """The user -> internal camera permutation (nl_get_user2internal_u)."""
        perm = np.zeros(self.nc_var, np.int32)
        self._c(self.L.nl_get_user2internal_u(self.h, _p(perm)), "nl_get_user2internal_u")
        return perm

    def set_solver_kind(self, kind: int):
        """SOLVER_DENSE (default) or SOLVER_ENVELOPE (nl_set_solver_kind): the
        envelope solver skips the tiles of S outside its Cholesky envelope,
        with bit-identical increments."""
        self._c(self.L.nl_set_solver_kind(self.h, C.c_int(kind)), "nl_set_solver_kind")

    def set_timing_detail(self, detail: bool):
        """Time every critical-path step of the factorisation in the next
        compute_increment calls (slower: see nl_set_timing_detail)."""
        self._c(self.L.nl_set_timing_detail(self.h, C.c_int(1 if detail else 0)), "nl_set_timing_detail")

    def set_wait_limit(self, polls: int):
        """Bound of the triangular solves' flag waits, in polls (<= 0: the
        default); nl_set_wait_limit."""
        self._c(self.L.nl_set_wait_limit(self.h, C.c_longlong(int(polls))), "nl_set_wait_limit")

    def check_wait_timeout(self) -> int:
        """nl_check_wait_timeout: the forward solve with one tile's flag
        withheld; returns the status code (7 = NL_ERR_TIMEOUT when every wait
        gave up as designed)."""
        return int(self.L.nl_check_wait_timeout(self.h))

    def kernel_launches(self):
        v = C.c_longlong()
        self._c(self.L.nl_kernel_launches(self.h, C.byref(v)), "nl_kernel_launches")
        return v.value


def rcm_order(nc, np_, cam_idx, pt_idx):
    """nl_rcm_order: the reverse Cuthill-McKee internal camera order of a
    camera / point edge list (host only, no device); perm[camera] = position."""
    L = load()
    cam = np.ascontiguousarray(cam_idx, np.int32)
    pt = np.ascontiguousarray(pt_idx, np.int32)
    perm = np.zeros(nc, np.int32)
    _chk(L, L.nl_rcm_order(C.c_int(nc), C.c_int(np_), C.c_int(cam.size), _p(cam), _p(pt), _p(perm)),
         "nl_rcm_order")
    return perm


def amd_order_camera_graph(nc, np_, cam_idx, pt_idx):
    """nl_amd_order_camera_graph: the approximate minimum degree internal
    camera order of a camera / point edge list (the pattern of U + W W');
    perm[camera] = position."""
    L = load()
    cam = np.ascontiguousarray(cam_idx, np.int32)
    pt = np.ascontiguousarray(pt_idx, np.int32)
    perm = np.zeros(nc, np.int32)
    _chk(L, L.nl_amd_order_camera_graph(C.c_int(nc), C.c_int(np_), C.c_int(cam.size), _p(cam), _p(pt), _p(perm)),
         "nl_amd_order_camera_graph")
    return perm


def amd_order(n, rows, cols):
    """nl_amd_order: approximate minimum degree order of a symmetric pattern
    given as (row, col) entries; perm[node] = position."""
    L = load()
    r = np.ascontiguousarray(rows, np.int32)
    c = np.ascontiguousarray(cols, np.int32)
    perm = np.zeros(n, np.int32)
    _chk(L, L.nl_amd_order(C.c_int(n), C.c_int(r.size), _p(r), _p(c), _p(perm)), "nl_amd_order")
    return perm


def symbolic_fill(n, rows, cols, perm):
    """nl_symbolic_fill: (entries of the Cholesky factor below the diagonal,
    elimination tree parent array) of the pattern under perm."""
    L = load()
    r = np.ascontiguousarray(rows, np.int32)
    c = np.ascontiguousarray(cols, np.int32)
    pm = np.ascontiguousarray(perm, np.int32)
    par = np.zeros(max(n, 1), np.int32)
    fill = C.c_longlong(0)
    _chk(L, L.nl_symbolic_fill(C.c_int(n), C.c_int(r.size), _p(r), _p(c), _p(pm), _p(par), C.byref(fill)),
         "nl_symbolic_fill")
    return int(fill.value), par[:n]


def lm_solve_batch(problems, settings=None):
    """LM on many BAProblemGPU handles at once (nl_lm_solve_batch): returns
    (reasons, final chi2 array, iterations array, per-problem latency in ms)."""
    L = load()
    n = len(problems)
    hs = (C.c_void_p * n)(*[p.h for p in problems])
    reps = (SolveReport * n)()
    lat = np.zeros(n)
    s = settings or LMSettings()
    _chk(L, L.nl_lm_solve_batch(hs, n, C.byref(s), C.cast(reps, C.c_void_p), _p(lat)), "nl_lm_solve_batch")
    return ([REASONS[r.reason] for r in reps], np.array([r.chi2 for r in reps]),
            np.array([r.iterations for r in reps]), lat)


class PersistentBatch:
    """nl_batch_*: many BAProblemGPU handles solved by one persistent launch
    (a device work queue over the problems, one CTA per problem at a time,
    FP64).  Results are written back to the handles."""

    def __init__(self, problems):
        self.L = load()
        self.problems = list(problems)
        n = len(self.problems)
        hs = (C.c_void_p * n)(*[p.h for p in self.problems])
        b = C.c_void_p()
        _chk(self.L, self.L.nl_batch_create(hs, n, C.byref(b)), "nl_batch_create")
        self.b = b

    def close(self):
        if getattr(self, "b", None):
            self.L.nl_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, settings=None):
        """Times every launch shape on this batch; returns (threads, ctas_per_sm)."""
        s = settings or LMSettings()
        nt, cps = C.c_int(), C.c_int()
        _chk(self.L, self.L.nl_batch_autotune(self.b, C.byref(s), C.byref(nt), C.byref(cps)), "nl_batch_autotune")
        return nt.value, cps.value

    def lm_solve(self, settings=None, threads=0, ctas_per_sm=0):
        """Returns (reasons, final chi2, iterations, per-problem latency ms,
        per-problem solve ms, launch device ms)."""
        n = len(self.problems)
        s = settings or LMSettings()
        reps = (SolveReport * n)()
        lat = np.zeros(n)
        dms = C.c_double()
        _chk(self.L, self.L.nl_batch_lm_solve(self.b, C.byref(s), threads, ctas_per_sm, C.cast(reps, C.c_void_p),
                                              _p(lat), C.byref(dms)), "nl_batch_lm_solve")
        return ([REASONS[r.reason] for r in reps], np.array([r.chi2 for r in reps]),
                np.array([r.iterations for r in reps]), lat, np.array([r.device_ms for r in reps]), dms.value)


def selftest_tc_update(ntiles=8, seed=1, device=0) -> float:
    """Max relative difference between the tensor-core and CUDA-core trailing updates."""
    L = load()
    err = C.c_double()
    _chk(L, L.nl_selftest_tc_update(ntiles, seed, device, C.byref(err)), "nl_selftest_tc_update")
    return err.value


def selftest_tc_update_k(ntiles=48, npanels=4, seed=1, reps=5, device=0):
    """(max relative difference against the CUDA-core update, best launch ms)
    of one rank-(128 npanels) tensor-core update of the trailing tiles."""
    L = load()
    err, ms = C.c_double(), C.c_double()
    _chk(L, L.nl_selftest_tc_update_k(ntiles, npanels, seed, device, reps, C.byref(err), C.byref(ms)),
         "nl_selftest_tc_update_k")
    return err.value, ms.value


class SchurSolverGPU:
    """Solver-only drop-in: SolverCholeskySchur on a Hessian assembled by the
    caller (U any pattern in upper CSC order, V block diagonal 3x3, W CSR),
    i.e. init / maxAbsHDiag / computeIncrement of nelson/SolverCholeskySchur.hpp:44-157."""

    def __init__(self, bu, nu, nv, u_rc, v_rc, w_rc, precision=PREC_FP64, refine_sweeps=-1, device=0):
        self.L = load()
        self.bu, self.nu, self.nv = bu, nu, nv
        u_rc = np.ascontiguousarray(u_rc, np.int32).reshape(-1, 2)
        v_rc = np.ascontiguousarray(v_rc, np.int32).reshape(-1, 2)
        w_rc = np.ascontiguousarray(w_rc, np.int32).reshape(-1, 2)
        d = SolverDesc(bu=bu, nu=nu, nv=nv, nU=len(u_rc), nV=len(v_rc), nW=len(w_rc), precision=precision,
                       refine_sweeps=refine_sweeps, device=device)
        h = C.c_void_p()
        _chk(self.L, self.L.nl_solver_create(C.byref(d), _p(u_rc), _p(v_rc), _p(w_rc), C.byref(h)),
             "nl_solver_create")
        self.h = h

    def set_solver_kind(self, kind: int):
        """SOLVER_DENSE (default) or SOLVER_ENVELOPE (nl_solver_set_kind)."""
        _chk(self.L, self.L.nl_solver_set_kind(self.h, C.c_int(kind)), "nl_solver_set_kind")

    def close(self):
        if getattr(self, "h", None):
            self.L.nl_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_hessian(self, U, V, W, bU, bV):
        a = [np.ascontiguousarray(x, np.float64) for x in (U, V, W, bU, bV)]
        _chk(self.L, self.L.nl_solver_set_hessian(self.h, *[_p(x) for x in a]), "nl_solver_set_hessian")

    def max_abs_hdiag(self):
        v = C.c_double()
        _chk(self.L, self.L.nl_solver_max_abs_hdiag(self.h, C.byref(v)), "nl_solver_max_abs_hdiag")
        return v.value

    def compute_increment(self, rel, abs_):
        du = np.zeros(self.nu * self.bu)
        dv = np.zeros(self.nv * 3)
        ok = C.c_int()
        _chk(self.L, self.L.nl_solver_compute_increment(self.h, rel, abs_, _p(du), _p(dv), C.byref(ok)),
             "nl_solver_compute_increment")
        return bool(ok.value), du, dv


class Pose2DGPU:
    """Device SingleSection of SE(2) poses with point-to-line edges (nl_pose2d_*):
    addEdge / permuteAMD / setUser2InternalIndexes / structureReady / update
    of nelson/SingleSection.hpp:26-139 with the edge of
    nelson/tests/testGaussNewton2DScansAlign.cpp:36-120, solved by
    LevenbergMarquardt / GaussNewton with the tiled Cholesky of U."""

    def __init__(self, nv, nf=1, precision=PREC_FP64, device=0):
        self.L = load()
        self.nv, self.nf = nv, nf
        h = C.c_void_p()
        _chk(self.L, self.L.nl_pose2d_create(C.c_int(nv), C.c_int(nf), C.c_int(precision), C.c_int(device),
                                             C.byref(h)), "nl_pose2d_create")
        self.h = h

    @classmethod
    def from_scan_align(cls, prob, precision=PREC_FP64, order="natural", perm=None, device=0):
        """Build the section of a ScanAlignProblem: scan 0 is the fixed pose,
        scan i > 0 the variable pose i - 1; edge (i, j) holds scan i's points
        and normals as the model and scan j's points as the target."""
        g = cls(len(prob.poses0), 1, precision, device)
        g.set_poses(prob.poses0, prob.poses_true[:1])
        for i, j in prob.edges:
            g.add_edge(i - 1 if i else 0, i == 0, j - 1 if j else 0, j == 0, prob.scans[i], prob.normals[i],
                       prob.scans[j])
        if order == "amd":
            g.permute_amd()
        elif order == "rcm":
            g.permute_rcm()
        elif perm is not None:
            g.set_user2internal(perm)
        g.structure_ready()
        return g

    def close(self):
        if getattr(self, "h", None):
            self.L.nl_pose2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc, what):
        _chk(self.L, rc, what)

    def set_poses(self, var_xyt, fix_xyt=None):
        v = np.ascontiguousarray(var_xyt, np.float64).reshape(self.nv, 3)
        f = None if fix_xyt is None else np.ascontiguousarray(fix_xyt, np.float64).reshape(self.nf, 3)
        self._c(self.L.nl_pose2d_set_poses(self.h, _p(v), _p(f)), "nl_pose2d_set_poses")

    def get_poses(self):
        out = np.zeros((self.nv, 3))
        self._c(self.L.nl_pose2d_get_poses(self.h, _p(out)), "nl_pose2d_get_poses")
        return out

    def add_edge(self, a, a_fixed, b, b_fixed, model_pts, model_normals, target_pts):
        m = np.ascontiguousarray(model_pts, np.float64).reshape(-1, 2)
        n = np.ascontiguousarray(model_normals, np.float64).reshape(-1, 2)
        t = np.ascontiguousarray(target_pts, np.float64).reshape(-1, 2)
        if not (len(m) == len(n) == len(t)):
            raise NelsonError("add_edge: model points, normals and target points differ in length")
        self._c(self.L.nl_pose2d_add_edge(self.h, C.c_int(a), C.c_int(int(a_fixed)), C.c_int(b),
                                          C.c_int(int(b_fixed)), C.c_int(len(m)), _p(m), _p(n), _p(t)),
                "nl_pose2d_add_edge")

    def set_user2internal(self, perm):
        p = np.ascontiguousarray(perm, np.int32)
        self._c(self.L.nl_pose2d_set_user2internal(self.h, _p(p)), "nl_pose2d_set_user2internal")

    def permute_amd(self):
        self._c(self.L.nl_pose2d_permute_amd(self.h), "nl_pose2d_permute_amd")

    def permute_rcm(self):
        self._c(self.L.nl_pose2d_permute_rcm(self.h), "nl_pose2d_permute_rcm")

    def structure_ready(self):
        self._c(self.L.nl_pose2d_structure_ready(self.h), "nl_pose2d_structure_ready")

    def set_solver_kind(self, kind: int):
        self._c(self.L.nl_pose2d_set_solver_kind(self.h, C.c_int(kind)), "nl_pose2d_set_solver_kind")

    def update(self, hessian=True):
        v = C.c_double()
        self._c(self.L.nl_pose2d_update(self.h, C.c_int(int(hessian)), C.byref(v)), "nl_pose2d_update")
        return v.value

    def hessian(self):
        """(H, b) of the last update(True): dense, user pose order."""
        n = 3 * self.nv
        H = np.zeros((n, n))
        b = np.zeros(n)
        self._c(self.L.nl_pose2d_get_hessian(self.h, _p(H), _p(b)), "nl_pose2d_get_hessian")
        return H, b

    def lm_solve(self, settings=None, trace_cap=4096):
        s = settings or LMSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_pose2d_lm_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_pose2d_lm_solve")
        self.last_report = {n: getattr(rep, n) for n, _ in SolveReport._fields_}
        return REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations

    def gn_solve(self, settings=None, trace_cap=4096):
        s = settings or GNSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_pose2d_gn_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_pose2d_gn_solve")
        self.last_report = {n: getattr(rep, n) for n, _ in SolveReport._fields_}
        return REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations


EDGE_UV, EDGE_UU, EDGE_U, EDGE_V = 0, 1, 2, 3
_EVAL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p)
_OPLUS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)
_STATE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)


class SectionCallbacks(C.Structure):
    _fields_ = [("user", C.c_void_p), ("evaluate", _EVAL_FN), ("oplus", _OPLUS_FN), ("backup", _STATE_FN),
                ("rollback", _STATE_FN)]


class SectionGPU:
    """A DoubleSection with user-defined edges (nl_section_*): the caller's
    code evaluates every edge's whitened residual and Jacobian blocks into the
    section's device arrays; the section assembles U / V / W / b on the device,
    solves with the Schur complement and runs LevenbergMarquardt / GaussNewton
    (nelson/DoubleSection.hpp:338-365 with user EdgeBinary / EdgeUnary edges,
    nelson/BaseSection.cpp:5-86).

    Callbacks are Python callables; device arrays are passed as integer
    addresses:
      evaluate(jacobians: bool, r_ptr, J_ptr, stream_ptr)
      oplus(incU_ptr, incV_ptr, stream_ptr)   (increments in user order)
      backup(stream_ptr), rollback(stream_ptr)
    An exception raised in a callback ends the library call, which then
    raises it."""

    def __init__(self, bu, nu, nv, precision=PREC_FP64, device=0):
        self.L = load()
        self.bu, self.nu, self.nv = bu, nu, nv
        h = C.c_void_p()
        _chk(self.L, self.L.nl_section_create(C.c_int(bu), C.c_int(nu), C.c_int(nv), C.c_int(precision),
                                              C.c_int(device), C.byref(h)), "nl_section_create")
        self.h = h
        self.ne = 0
        self._exc = None
        self._cb = None

    def close(self):
        if getattr(self, "h", None):
            self.L.nl_section_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc, what):
        if self._exc is not None:
            e, self._exc = self._exc, None
            raise e
        _chk(self.L, rc, what)

    def add_edges(self, kind, a, b, m):
        k = np.ascontiguousarray(kind, np.int32)
        aa = np.ascontiguousarray(a, np.int32)
        bb = np.ascontiguousarray(b, np.int32)
        mm = np.ascontiguousarray(m, np.int32)
        if not (k.size == aa.size == bb.size == mm.size):
            raise NelsonError("add_edges: kind, a, b and m differ in length")
        self._c(self.L.nl_section_add_edges(self.h, C.c_int(k.size), _p(k), _p(aa), _p(bb), _p(mm)),
                "nl_section_add_edges")
        self.ne += k.size

    def set_user2internal(self, perm):
        p = np.ascontiguousarray(perm, np.int32)
        self._c(self.L.nl_section_set_user2internal_u(self.h, _p(p)), "nl_section_set_user2internal_u")

    def permute_amd(self):
        self._c(self.L.nl_section_permute_amd_u(self.h), "nl_section_permute_amd_u")

    def user2internal(self):
        p = np.zeros(self.nu, np.int32)
        self._c(self.L.nl_section_get_user2internal_u(self.h, _p(p)), "nl_section_get_user2internal_u")
        return p

    def structure_ready(self):
        self._c(self.L.nl_section_structure_ready(self.h), "nl_section_structure_ready")

    def counts(self):
        nU, nW, rl, jl = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong()
        self._c(self.L.nl_section_get_counts(self.h, C.byref(nU), C.byref(nW), C.byref(rl), C.byref(jl)),
                "nl_section_get_counts")
        return nU.value, nW.value, rl.value, jl.value

    def layout(self):
        r = np.zeros(self.ne + 1, np.int64)
        j = np.zeros(self.ne + 1, np.int64)
        self._c(self.L.nl_section_layout(self.h, _p(r), _p(j)), "nl_section_layout")
        return r, j

    def patterns(self):
        nU, nW, _, _ = self.counts()
        u = np.zeros((max(nU, 1), 2), np.int32)
        w = np.zeros((max(nW, 1), 2), np.int32)
        self._c(self.L.nl_section_get_patterns(self.h, _p(u), _p(w)), "nl_section_get_patterns")
        return u[:nU], w[:nW]

    def set_callbacks(self, evaluate, oplus, backup=None, rollback=None):
        def guard(fn):
            def run(*args):
                try:
                    fn(*args)
                    return 0
                except BaseException as e:   # reported by the library call that ran it
                    self._exc = e
                    return 1
            return run

        ev = _EVAL_FN(guard(lambda u, st, jac, r, J: evaluate(bool(jac), r, J, st)))
        op = _OPLUS_FN(guard(lambda u, st, du, dv: oplus(du, dv, st)))
        bk = _STATE_FN(guard(lambda u, st: backup(st))) if backup else _STATE_FN()
        rb = _STATE_FN(guard(lambda u, st: rollback(st))) if rollback else _STATE_FN()
        cb = SectionCallbacks(None, ev, op, bk, rb)
        self._cb = (cb, ev, op, bk, rb)   # keep the trampolines alive
        self._c(self.L.nl_section_set_callbacks(self.h, C.byref(cb)), "nl_section_set_callbacks")

    def set_solver_kind(self, kind: int):
        self._c(self.L.nl_section_set_solver_kind(self.h, C.c_int(kind)), "nl_section_set_solver_kind")

    def update(self, hessian=True):
        v = C.c_double()
        self._c(self.L.nl_section_update(self.h, C.c_int(int(hessian)), C.byref(v)), "nl_section_update")
        return v.value

    def hessian(self):
        """(U, V, W, bU, bV) of the last update(True): blocks in pattern order,
        bU in internal order."""
        nU, nW, _, _ = self.counts()
        bu = self.bu
        U = np.zeros((nU, bu, bu))
        V = np.zeros((self.nv, 3, 3))
        W = np.zeros((nW, bu, 3))
        bU = np.zeros(self.nu * bu)
        bV = np.zeros(self.nv * 3)
        self._c(self.L.nl_section_get_hessian(self.h, _p(U), _p(V), _p(W), _p(bU), _p(bV)), "nl_section_get_hessian")
        return U, V, W, bU, bV

    def compute_increment(self, rel, abs_):
        du = np.zeros(self.nu * self.bu)
        dv = np.zeros(self.nv * 3)
        ok = C.c_int()
        self._c(self.L.nl_section_compute_increment(self.h, rel, abs_, _p(du), _p(dv), C.byref(ok)),
                "nl_section_compute_increment")
        return bool(ok.value), du, dv

    def lm_solve(self, settings=None, trace_cap=4096):
        s = settings or LMSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_section_lm_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_section_lm_solve")
        self.last_report = {n: getattr(rep, n) for n, _ in SolveReport._fields_}
        return REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations

    def gn_solve(self, settings=None, trace_cap=4096):
        s = settings or GNSettings()
        rep = SolveReport()
        tr = np.zeros((max(trace_cap, 1), TRACE_STRIDE))
        self._c(self.L.nl_section_gn_solve(self.h, C.byref(s), C.byref(rep), _p(tr), trace_cap), "nl_section_gn_solve")
        self.last_report = {n: getattr(rep, n) for n, _ in SolveReport._fields_}
        return REASONS[rep.reason], tr[:rep.n_trace].copy(), rep.iterations

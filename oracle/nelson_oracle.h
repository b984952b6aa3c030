/*
 * nelson_oracle.h -- C ABI of the FP64 CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++/OpenMP restatement of
 * nelson's Schur-complement Levenberg-Marquardt / Gauss-Newton path.  It is
 * the checker for the CUDA library (tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py); nothing in the nelson_b200 product links,
 * loads or calls it.
 *
 * Each entry point states the reference code it restates (paths relative to
 * the nelson source tree).
 */
#ifndef NELSON_ORACLE_H
#define NELSON_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Problem kinds. */
#define ORC_KIND_BA 0      /* bundle adjustment: U = cameras, V = 3D points  */
#define ORC_KIND_LINEAR 1  /* vector parameters, constant-Jacobian edges     */

/* Linear edge types (nelson/tests/testDoubleSectionSchurCommon.h:28-321). */
#define ORC_EDGE_UNARY_U 0
#define ORC_EDGE_UNARY_V 1
#define ORC_EDGE_BINARY_UU 2
#define ORC_EDGE_BINARY_UV 3

/* LevenbergMarquardtSettings (nelson/LevenbergMarquardt.h:18-34). */
typedef struct {
  int maxNumIt, maxNumSubIt, minNumIt;
  double epsBVector, epsIncSquare, epsChi2, tau, penaltyV, initV;
  double maxScaleFactor, minScaleFactor;
} orc_lm_settings;

/* GaussNewtonSettings (nelson/GaussNewton.h:18-30). */
typedef struct {
  int maxNumIt, minNumIt;
  double epsBVector, epsIncSquare, epsChi2, absLambda, relLambda;
} orc_gn_settings;

/* One record per sub-iteration: it, subit, chi2, mu, rho, |inc|^2, ok, accepted. */
#define ORC_TRACE_STRIDE 8

void* orc_create(int kind, int bu, int bv, int nu_var, int nu_fix, int nv_var,
                 int nv_fix, int num_threads);
void orc_destroy(void* h);

/* BA intrinsics: principal point and, for 6-parameter cameras, the fixed focal. */
int orc_set_intrinsics(void* h, double f, double cx, double cy);

/* Parameters.  BA cameras are (axis-angle[3], t[3] [, f, k1, k2]) per camera,
 * variable ones first, then fixed; BA points and linear parameters are plain
 * vectors.  Layouts are dense row-major. */
int orc_set_params(void* h, const double* u, const double* v);
int orc_get_params(void* h, double* u, double* v);
/* BA camera state as stored: R[9] row-major, t[3], f, k1, k2, pad (16 doubles). */
int orc_get_camera_state(void* h, double* states);

/* DoubleSection::addEdge (nelson/DoubleSection.hpp:338-365), vectorised:
 * edge e joins camera cam[e] (fixed if cam_fixed[e]) and point pt[e]. */
int orc_add_ba_edges(void* h, int ne, const int* cam, const int* cam_fixed,
                     const int* pt, const int* pt_fixed, const double* obs,
                     const double* weight);
/* One linear edge r = A1 x1 + A2 x2 - z (A row-major dr x B). */
int orc_add_linear_edge(void* h, int type, int id1, int fixed1, int id2,
                        int fixed2, int dr, const double* A1, const double* A2,
                        const double* z);

/* DoubleSection::setUser2InternalIndexesU (nelson/DoubleSection.hpp:23-27). */
int orc_set_user2internal_u(void* h, const int* perm);
/* DoubleSection::structureReady (nelson/DoubleSection.hpp:83-246). */
int orc_structure_ready(void* h);

/* Structure queries: counts = {nUblocks, nVblocks, nWblocks, nEdges}. */
int orc_get_counts(void* h, int* counts);
/* Block coordinates (internal row, col) of each UID, for U, V and W. */
int orc_get_patterns(void* h, int* u_rc, int* v_rc, int* w_rc);
/* Per-edge block UIDs H_11, H_12, H_22 (-1 when absent), in insertion order. */
int orc_get_edge_uids(void* h, int* h11, int* h12, int* h22);

/* DoubleSection::update (nelson/DoubleSection.hpp:452-467). */
int orc_update(void* h, int hessian, double* chi2);
/* Hessian blocks in UID order, each block row-major; bU in internal order. */
int orc_get_hessian(void* h, double* U, double* V, double* W, double* bU,
                    double* bV);
/* Per-edge residuals (dr values each, insertion order). */
int orc_get_residuals(void* h, double* r);

/* SolverCholeskySchur (nelson/SolverCholeskySchur.hpp:44-157). */
int orc_solver_init(void* h);
double orc_max_abs_hdiag(void* h);
/* Returns 1 when the solve succeeded, 0 otherwise (increment zeroed). */
int orc_compute_increment(void* h, double rel_lambda, double abs_lambda);
int orc_get_increment(void* h, double* incU, double* incV);
double orc_inc_sqnorm(void* h);
/* Reduced camera system as formed (dense n x n, upper triangle valid) and bS. */
int orc_get_schur(void* h, double* S, double* bS, int* n);

/* Problem concept used by LevenbergMarquardt::solve. */
int orc_oplus(void* h);
int orc_backup(void* h);
int orc_rollback(void* h);
double orc_max_abs_b(void* h);
double orc_chi2(void* h);
double orc_rho(void* h, double mu, double old_chi2);

/* LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146).
 * Returns the termination reason (LevenbergMarquardtTerminationReason order);
 * fills up to trace_cap records of ORC_TRACE_STRIDE doubles; *n_trace gets the
 * number written; its/subits get numIterations()/numSubIterations(). */
int orc_lm_solve(void* h, const orc_lm_settings* s, double* trace,
                 int trace_cap, int* n_trace, int* its);
/* GaussNewton::solve (nelson/GaussNewton.hpp:32-127). */
int orc_gn_solve(void* h, const orc_gn_settings* s, double* trace,
                 int trace_cap, int* n_trace, int* its);

/* Implicit-function adjoint of a converged BA solve (no counterpart in the
 * reference): H mu = dL/dx with the exact Hessian H of the cost at the
 * current parameters (complex-step derivatives of each edge's gradient),
 * then per edge dL/dz = w J mu and dL/dw = -(J mu) . r.  dL_dcams: variable
 * cameras in user order (tangent [dw, dt (, df, dk1, dk2)]); dL_dpts:
 * variable points; either may be NULL.  Outputs (any may be NULL): g_obs (2
 * per edge), g_w (1 per edge) in insertion order, mu in the layout of the
 * inputs.  Returns 1 when the solve succeeded, 0 when H was not positive
 * definite, -1 on a bad handle. */
int orc_adjoint_ba(void* h, const double* dL_dcams, const double* dL_dpts,
                   double* g_obs, double* g_w, double* mu_cams, double* mu_pts);

/* Dense blocked Cholesky of an n x n row-major SPD matrix (lower triangle
 * used), exposed so its accuracy can be tested on its own.  Returns 1 on
 * success. */
int orc_dense_cholesky(double* A, int n, int lda, int num_threads);

#ifdef __cplusplus
}
#endif
#endif

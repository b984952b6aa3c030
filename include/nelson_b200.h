/*
 * nelson_b200.h -- C ABI of the B200-native Schur-complement LM/GN engine.
 *
 * This is the drop-in boundary for nelson's SolverCholeskySchur hot path.
 * The reference binds its solver at compile time (SolverTraits<id>::Solver,
 * nelson/SolverTraits.h:16-56) and drives it from LevenbergMarquardt /
 * GaussNewton through two concepts:
 *   - the Solver concept: init(H, b), maxAbsHDiag(), computeIncrement(H, b,
 *     relLambda, absLambda) -> bool, incrementVector(),
 *     incrementVectorSquaredNorm()   (nelson/SolverCholeskySchur.h:96-115);
 *   - the problem concept: update(bool), hessian().chi2()/maxAbsValBVect(),
 *     oplus(inc), backupSolution(), rollbackSolution(),
 *     computeRhoChi2Change(mu, inc, oldChi2)
 *     (nelson/LevenbergMarquardt.hpp:41-136, nelson/DoubleSection.h:300-311).
 * Each entry point below replaces one of those calls; the C++ headers in
 * include/nelson_b200/ wrap them back into the reference's class shapes.
 *
 * Conventions: plain pointers and sizes, host memory unless a name says
 * "device"; every function returns an nl_status (0 = ok).  A handle owns its
 * device memory and one CUDA stream; calls on one handle must not overlap,
 * calls on different handles may run from different threads.
 */
#ifndef NELSON_B200_H
#define NELSON_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum {
  NL_OK = 0,
  NL_ERR_ARG = 1,          /* bad argument / size / index                      */
  NL_ERR_STATE = 2,        /* call out of order (e.g. update before structure) */
  NL_ERR_CUDA = 3,         /* a CUDA runtime / cuBLAS call failed              */
  NL_ERR_UNSUPPORTED = 4,  /* structure outside the device solver's scope      */
  NL_ERR_NOT_SPD = 5,      /* a damped block or the reduced system not SPD     */
  NL_ERR_NONFINITE = 6,    /* non-finite cost / increment                      */
  NL_ERR_TIMEOUT = 7,      /* a bounded device-side wait gave up               */
  NL_ERR_NOMEM = 8,        /* device allocation failed                         */
  NL_ERR_CALLBACK = 9      /* a user callback returned non-zero                */
} nl_status;

/* ---- precision modes ---------------------------------------------------- */
#define NL_PREC_FP64 0  /* Jacobians, Hessian, Schur and Cholesky in FP64      */
#define NL_PREC_MIXED 1 /* FP32 Jacobians/Hessian/Schur, tensor-core trailing
                           updates, FP32 diagonal tiles, FP64 refinement residual,
                           solve accumulators and cost                          */

/* Factorisation of the reduced camera system S (nl_set_solver_kind). */
#define NL_SOLVER_DENSE 0    /* every 128-tile of S, as SolverCholeskySchur's dense
                                LDLT (nelson/SolverCholeskySchur.hpp:136-140)     */
#define NL_SOLVER_ENVELOPE 1 /* only the tiles inside the Cholesky envelope of S:
                                the same factor (there is no fill before a row's
                                first nonzero), far less work when the camera
                                order keeps camera pairs near the diagonal        */

/* ---- settings (same fields and defaults as the reference) --------------- */
/* LevenbergMarquardtSettings, nelson/LevenbergMarquardt.h:18-34;
 * defaults nelson/LevenbergMarquardt.cpp:6-19. */
typedef struct {
  int maxNumIt, maxNumSubIt, minNumIt;
  double epsBVector, epsIncSquare, epsChi2, tau, penaltyV, initV;
  double maxScaleFactor, minScaleFactor;
} nl_lm_settings;

/* GaussNewtonSettings, nelson/GaussNewton.h:18-30; defaults GaussNewton.cpp:12-22. */
typedef struct {
  int maxNumIt, minNumIt;
  double epsBVector, epsIncSquare, epsChi2, absLambda, relLambda;
} nl_gn_settings;

/* Termination reasons, in the order of nelson/LevenbergMarquardt.h:36-44
 * (GN uses the first six, nelson/GaussNewton.h:34-41). */
#define NL_SUCCESS_AT_START 0
#define NL_SUCCESS_SMALL_INCREMENT 1
#define NL_SUCCESS_EPS_B 2
#define NL_SUCCESS_SMALL_RESIDUALS 3
#define NL_SOLVER_FAILURE 4
#define NL_MAX_ITERATION_REACHED 5
#define NL_MAX_SUBITERATION_REACHED 6

/* One trace record per sub-iteration: it, subit, chi2, mu, rho, |inc|^2, ok,
 * accepted (the LevenbergMarquardtStats content, nelson/LevenbergMarquardt.h:57-85,
 * plus the damping and gain ratio). */
#define NL_TRACE_STRIDE 8

typedef struct {
  int reason;          /* NL_SUCCESS_* / NL_*_REACHED / NL_SOLVER_FAILURE */
  int iterations;      /* numIterations() */
  int subiterations;   /* total computeIncrement calls */
  int n_trace;         /* records written */
  double chi2;         /* final cost */
  double mu;           /* final damping */
  double device_ms;    /* device time of the solve (CUDA events on the handle's stream) */
} nl_solve_report;

/* Per-phase device time of the last computeIncrement, milliseconds
 * (the phases of SolverCholeskySchurIterationTimeStat, nelson/SolverCholeskySchur.h:25-38). */
typedef struct {
  float vinv_ms, wvinv_bs_ms, schur_ms, factor_ms, solve_ms, backsub_ms, total_ms;
  float eval_ms;     /* device time of the last nl_update(h, 1, ...) */
  float update_ms;   /* device time of the trailing updates inside factor_ms */
  int update_launches;
  double update_flop;  /* algorithmic flops of those updates (2 * multiply-adds) */
  double update_bytes; /* algorithmic bytes of those updates: each updated
                          128 x 128 tile read and written once per launch */
  /* The three critical-path fields below are filled only after
   * nl_set_timing_detail(h, 1) (mixed precision); otherwise they are 0. */
  float panel_ms;      /* summed device time of the diagonal-tile factorisations
                          on the critical path (from their enqueue on the main
                          stream, so including any wait for an SM) */
  int panels;          /* number of those factorisations */
  float wait_ms;       /* main-stream time between a diagonal-tile factor's end
                          and the start of the next row-tile TRSM (waiting for
                          the auxiliary stream's column updates) */
  float first_ms;      /* main-stream time of the row-tile TRSMs and the
                          diagonal-tile updates (8-CTA kernels), incl. launch gaps */
} nl_phase_times;

/* ---- problem: device-resident BA section -------------------------------- */
typedef struct nl_problem nl_problem;

typedef struct {
  int bc;              /* camera block size: 6 (pose) or 9 (pose, f, k1, k2) */
  int nc_var, nc_fix;  /* variable / fixed cameras  (numParametersU + numFixedParametersU) */
  int np_var, np_fix;  /* variable / fixed points   (numParametersV + numFixedParametersV) */
  int precision;       /* NL_PREC_FP64 or NL_PREC_MIXED */
  double f, cx, cy;    /* focal (6-parameter cameras) and principal point */
  int refine_sweeps;   /* iterative-refinement sweeps on S (mixed); -1 = default */
  int device;          /* CUDA device ordinal */
} nl_problem_desc;

/* DoubleSection constructor + parametersReady (nelson/DoubleSection.hpp:67-80). */
nl_status nl_create(const nl_problem_desc* desc, nl_problem** out);
nl_status nl_destroy(nl_problem* h);

/* Parameter blocks: cameras (axis-angle[3], t[3] [, f, k1, k2]) variable first
 * then fixed; points xyz.  Replaces the user's parameterU/parameterV storage
 * (nelson/DoubleSection.h:226-229). */
nl_status nl_set_params(nl_problem* h, const double* cams, const double* pts);
nl_status nl_get_params(nl_problem* h, double* cams, double* pts);
/* Camera state as stored on the device: R[9] row-major, t[3], f, k1, k2, pad. */
nl_status nl_get_camera_state(nl_problem* h, double* states);

/* DoubleSection::addEdge(NodeId cam, NodeId pt, EdgeBinaryUV*)
 * (nelson/DoubleSection.hpp:338-365), vectorised; cam_fixed / pt_fixed mark
 * NodeType::Fixed ids (nelson/EdgeInterface.h:35-55); weight may be NULL. */
nl_status nl_add_ba_edges(nl_problem* h, int ne, const int* cam, const int* cam_fixed,
                          const int* pt, const int* pt_fixed, const double* obs,
                          const double* weight);
/* DoubleSection::setUser2InternalIndexesU (nelson/DoubleSection.hpp:23-27). */
nl_status nl_set_user2internal_u(nl_problem* h, const int* perm);
/* DoubleSection::structureReady (nelson/DoubleSection.hpp:83-246): builds the
 * U/V/W patterns and block UIDs exactly as the reference and uploads the
 * edge -> block maps. */
nl_status nl_structure_ready(nl_problem* h);
/* In place of DoubleSection::permuteAMD_SchurU (nelson/DoubleSection.hpp:30-63):
 * an internal camera order from the same camera graph (variable cameras that
 * observe a common variable point, the pattern of U + W W'), computed by
 * reverse Cuthill-McKee instead of AMD -- it narrows the envelope of S that
 * NL_SOLVER_ENVELOPE factors (AMD aims at the fill of a sparse factor, which
 * this library does not build).  Sets the user -> internal permutation; call
 * after the edges are added and before nl_structure_ready. */
nl_status nl_permute_rcm_u(nl_problem* h);
/* The same ordering as a host function that needs no device: nc cameras, np
 * points, ne edges (cam[e], pt[e]); writes perm[camera] = internal position
 * (reverse Cuthill-McKee of the graph of cameras sharing a point). */
nl_status nl_rcm_order(int nc, int np, int ne, const int* cam, const int* pt, int* perm);
/* DoubleSection::permuteAMD_SchurU (nelson/DoubleSection.hpp:30-63): the
 * approximate minimum degree order (Amestoy, Davis & Duff 1996) of the
 * pattern of U + W W' -- variable cameras that observe a common variable
 * point -- as the user -> internal permutation.  Call after the edges are
 * added and before nl_structure_ready.  The reference takes the order from
 * Eigen::AMDOrdering; this is the same published algorithm in its own code,
 * so ties may be broken differently (the fill it leads to is what matters). */
nl_status nl_permute_amd_u(nl_problem* h);
/* The same order as a host function: nc cameras, np points, ne edges
 * (cam[e], pt[e]); perm[camera] = internal position. */
nl_status nl_amd_order_camera_graph(int nc, int np, int ne, const int* cam, const int* pt, int* perm);
/* SingleSection::permuteAMD (nelson/SingleSection.hpp:33-52) for any
 * symmetric pattern: n nodes, nnz entries (row[k], col[k]) of either triangle
 * or both (diagonal and duplicates ignored); perm[node] = position. */
nl_status nl_amd_order(int n, int nnz, const int* row, const int* col, int* perm);
/* Symbolic Cholesky of that pattern under perm: the elimination tree
 * (parent[new index], -1 at a root; may be null) and the number of entries of
 * the factor strictly below the diagonal. */
nl_status nl_symbolic_fill(int n, int nnz, const int* row, const int* col, const int* perm, int* parent,
                           long long* fill);
/* The user -> internal camera permutation in effect (nc_var entries; the
 * identity unless set): increments come in internal order. */
nl_status nl_get_user2internal_u(nl_problem* h, int* perm);
/* Replace observations / weights of an existing structure (same edge order). */
nl_status nl_set_observations(nl_problem* h, const double* obs, const double* weight);

/* counts = {U blocks, V blocks, W blocks, edges}; patterns are (row, col)
 * per UID; edge UIDs are EdgeBinaryBase::H_11/12/22_Uid (nelson/EdgeBinary.h:12-14). */
nl_status nl_get_counts(nl_problem* h, int* counts);
nl_status nl_get_patterns(nl_problem* h, int* u_rc, int* v_rc, int* w_rc);
nl_status nl_get_edge_uids(nl_problem* h, int* h11, int* h12, int* h22);

/* DoubleSection::update(bool) (nelson/DoubleSection.hpp:452-467). */
nl_status nl_update(nl_problem* h, int hessian, double* chi2);
/* Hessian blocks in UID order (row-major blocks), bU in internal order, FP64. */
nl_status nl_get_hessian(nl_problem* h, double* U, double* V, double* W, double* bU, double* bV);

/* SolverCholeskySchur::init / maxAbsHDiag / computeIncrement /
 * incrementVector / incrementVectorSquaredNorm (nelson/SolverCholeskySchur.hpp:44-157). */
nl_status nl_solver_init(nl_problem* h);
nl_status nl_max_abs_hdiag(nl_problem* h, double* out);
nl_status nl_compute_increment(nl_problem* h, double rel_lambda, double abs_lambda, int* ok);
nl_status nl_get_increment(nl_problem* h, double* incU, double* incV);
nl_status nl_inc_sqnorm(nl_problem* h, double* out);
/* The damped reduced camera system as formed (n x n row-major, the upper
 * triangle holds S as the reference builds it) and bS; *n gets the size. */
nl_status nl_get_schur(nl_problem* h, double* S, double* bS, int* n);

/* Problem concept: oplus / backupSolution / rollbackSolution /
 * maxAbsValBVect / chi2 / computeRhoChi2Change. */
nl_status nl_oplus(nl_problem* h);
nl_status nl_backup(nl_problem* h);
nl_status nl_rollback(nl_problem* h);
nl_status nl_max_abs_b(nl_problem* h, double* out);
nl_status nl_chi2(nl_problem* h, double* out);
nl_status nl_rho(nl_problem* h, double mu, double old_chi2, double* out);

/* LevenbergMarquardt<Solver>::solve (nelson/LevenbergMarquardt.hpp:36-146)
 * with the whole iteration on the device; trace may be NULL. */
nl_status nl_lm_solve(nl_problem* h, const nl_lm_settings* s, nl_solve_report* rep,
                      double* trace, int trace_cap);
/* LevenbergMarquardt<Solver>::solve on n independent problems at once (the
 * reference solves one problem per call).  All handles must be ready and on
 * the same device; each problem's LM sub-iteration is captured once as a CUDA
 * graph on its handle's streams and replayed, the problems interleaved with at
 * most two sub-iterations in flight each.  reps (may be NULL) get each
 * problem's report; latency_ms (may be NULL) each problem's device time from
 * the common start to its completion.  No trace is recorded. */
nl_status nl_lm_solve_batch(nl_problem** hs, int n, const nl_lm_settings* s, nl_solve_report* reps,
                            double* latency_ms);
/* ---- many small problems in one persistent launch ----------------------- */
/* LevenbergMarquardt<SolverCholeskySchur>::solve (nelson/LevenbergMarquardt.hpp:
 * 36-146) for n independent BA sections of uneven sizes in ONE kernel launch
 * (the reference solves one problem per call): the launch's CTAs take
 * problems from a device work queue, largest first, and each CTA runs one
 * problem's whole LM solve -- Jacobians and Hessian blocks, the Schur
 * complement, a blocked Cholesky of S in shared memory, the solves, the
 * back-substitution and the LM decisions -- in FP64, then takes the next.
 * No CTA waits for another.  A problem's result does not depend on the launch
 * shape or on the other problems of the batch.
 * nl_batch_create packs the sections (ready handles on the current device, all
 * with the same camera block size, at most 768 reduced-system rows each) into
 * one device arena; the observations and weights are taken as they are at
 * that moment.  nl_batch_lm_solve copies each handle's current parameters in,
 * solves, and writes the results back to the handles (read them with
 * nl_get_params).  threads (128, 256 or 512) and ctas_per_sm (1..4) choose the
 * launch shape; 0 takes the choice of nl_batch_autotune, which times every
 * candidate on the batch itself (each from the handles' parameters, so it
 * changes nothing) and keeps the fastest.  reps (may be NULL): per problem,
 * device_ms is its own solve time; latency_ms (may be NULL): per problem, the
 * time from the first problem's start to its end; device_ms_total (may be
 * NULL): the launch's device time. */
typedef struct nl_batch nl_batch;
nl_status nl_batch_create(nl_problem** hs, int n, nl_batch** out);
nl_status nl_batch_destroy(nl_batch* b);
nl_status nl_batch_autotune(nl_batch* b, const nl_lm_settings* s, int* threads, int* ctas_per_sm);
nl_status nl_batch_lm_solve(nl_batch* b, const nl_lm_settings* s, int threads, int ctas_per_sm,
                            nl_solve_report* reps, double* latency_ms, double* device_ms_total);

/* GaussNewton<Solver>::solve (nelson/GaussNewton.hpp:32-127). */
nl_status nl_gn_solve(nl_problem* h, const nl_gn_settings* s, nl_solve_report* rep,
                      double* trace, int trace_cap);

/* ---- adjoint of a converged solve (implicit-function theorem) ------------ */
/* No counterpart in the reference (it has no differentiation).  At a
 * converged solution x* (the local gradient J'W r vanishes) and for a loss
 * L(x*) with gradient dL/dx, computes
 *     mu = H^-1 dL/dx          (H: exact Hessian of the cost at x*, FP64
 *                               Hessian-vector products incl. second-order terms)
 *     dL/dz_e = w_e J_e mu_e   (observations, 2 per edge)
 *     dL/dw_e = -(J_e mu_e) . r_e   (per-edge weights)
 * mu is found by `sweeps` rounds of iterative refinement preconditioned by
 * the Schur factorisation of J'WJ at x* (factored once, reused each round).
 * H must be non-singular: hold the gauge (e.g. two cameras as fixed nodes).
 * Inputs, host memory: dL_dcams (variable cameras in user order, camera
 * tangent [dw, dt (, df, dk1, dk2)]) and dL_dpts (variable points, xyz);
 * either may be NULL for zero.  Outputs (any may be NULL): g_obs (2 per edge)
 * and g_weight (1 per edge) in the order the edges were added; mu_cams /
 * mu_pts in the layout of the inputs.  The gradient w.r.t. the initial
 * parameters of a converged solve is zero and is not returned.  On return the
 * Hessian blocks are those of x* and the gradient vector b is overwritten:
 * call nl_update(h, 1, ...) before reading b-dependent quantities. */
typedef struct {
  int ok;               /* 1 when every factorisation / solve succeeded */
  int sweeps;           /* refinement rounds after the first solve */
  double grad_norm;     /* |dL/dx| */
  double residual_norm; /* |dL/dx - H mu| after the last round */
  double device_ms;     /* device time of the adjoint */
} nl_adjoint_report;
nl_status nl_adjoint(nl_problem* h, const double* dL_dcams, const double* dL_dpts, int sweeps, double* g_obs,
                     double* g_weight, double* mu_cams, double* mu_pts, nl_adjoint_report* rep);

/* ---- unrolled differentiation of K LM steps (per-step checkpoints) ------- */
/* No counterpart in the reference.  The unrolled map is K accepted
 * LevenbergMarquardt steps from the current parameters x_0,
 *     x_{k+1} = x_k (+) delta_k,   delta_k = -(J'WJ(x_k) + mu_k I)^-1 b(x_k),
 * exactly the increments of nelson/LevenbergMarquardt.hpp:63-141 with the
 * damping mu_k of the accepted sub-iterations held fixed (the accept / reject
 * choices and the mu updates are discrete and not differentiated; rejected
 * sub-iterations leave x unchanged).  Pass the mu of an LM trace's accepted
 * records to differentiate that LM run.
 * nl_unroll_record takes the K steps from the current parameters, saving x_k
 * (cameras and points, a few hundred kilobytes per step at 64 cameras / 5,000
 * points) before each one; on return the parameters are x_K.  A step whose
 * damped system is not positive definite stops the record (NL_ERR_NOT_SPD).
 * nl_unroll_adjoint then runs backwards through the recorded steps: for each
 * k it restores x_k from its checkpoint, re-forms J'WJ and the step (the
 * factorisation is recomputed, not stored) and applies the step's
 * vector-Jacobian product.  Inputs: dL/dx_K as in nl_adjoint (dL_dcams in the
 * camera tangent [dw, dt (, df, dk1, dk2)] at x_K, user order; dL_dpts;
 * either may be NULL).  Outputs (any may be NULL): g_obs (2 per edge) and
 * g_weight (1 per edge) in the order the edges were added, g_cams0 the
 * gradient w.r.t. the initial camera parameters as nl_set_params takes them
 * (axis-angle, t (, f, k1, k2); variable cameras, user order), g_pts0 w.r.t.
 * the initial points.  On return the parameters are x_K again; the Hessian
 * blocks and b are those of x_0 (call nl_update before reading them). */
typedef struct {
  int steps;        /* steps recorded / differentiated */
  int ok;           /* 1 when every factorisation succeeded */
  double chi2;      /* cost at x_K (nl_unroll_record) */
  double device_ms; /* device time of the call */
} nl_unroll_report;
nl_status nl_unroll_record(nl_problem* h, int nsteps, const double* mu, nl_unroll_report* rep);
nl_status nl_unroll_adjoint(nl_problem* h, const double* dL_dcams, const double* dL_dpts, double* g_obs,
                            double* g_weight, double* g_cams0, double* g_pts0, nl_unroll_report* rep);

nl_status nl_phase_timings(nl_problem* h, nl_phase_times* out);
/* detail = 1: nl_compute_increment also times every step of the
 * factorisation's critical path (panel_ms, wait_ms, first_ms).  That costs one
 * event record per kernel boundary on the host and disables the early launch
 * of the chain's kernels, so the factorisation itself runs slower; 0 (the
 * default) times the phases and the trailing updates only. */
nl_status nl_set_timing_detail(nl_problem* h, int detail);
/* NL_SOLVER_DENSE (default) or NL_SOLVER_ENVELOPE for the computeIncrements
 * that follow.  The envelope solver is the tile-level profile Cholesky of the
 * same S in the same (internal) camera order: its increments are
 * bit-identical to the dense solver's, the trailing updates, panel TRSMs and
 * triangular solves skip the tiles that are zero in the factor.  It is the
 * dense-kernel step toward the block-sparse
 * SolverDiagonalBlocksInverseWWtMultSchur
 * (nelson/SolverDiagonalBlocksInverseWWtMultSchur.hpp:36-140), without that
 * solver's AMD reordering (nelson/DoubleSection.hpp:30-63). */
nl_status nl_set_solver_kind(nl_problem* h, int kind);
/* Bound of the flag waits between the CTAs of the triangular solves: a CTA
 * that has polled a tile's flag `polls` times without seeing it published
 * records a timeout, returns, and the call reports NL_ERR_TIMEOUT (the wait
 * ends instead of hanging the GPU).  polls <= 0 restores the default
 * (2^24 polls, about a second).  (No counterpart in the reference: its solves
 * run on the host.) */
nl_status nl_set_wait_limit(nl_problem* h, long long polls);
/* Check of that bound: runs the forward triangular solve of the handle's
 * current factor with the flag of the first tile never published (its CTA is
 * not launched), so every other CTA's first wait runs out.  Returns
 * NL_ERR_TIMEOUT when the waits gave up as designed, NL_ERR_STATE when the
 * reduced system has fewer than two 128-row tiles.  The handle stays usable:
 * the next nl_compute_increment solves normally.  (No counterpart in the
 * reference.) */
nl_status nl_check_wait_timeout(nl_problem* h);
/* Number of kernels of this library launched on the handle since creation. */
nl_status nl_kernel_launches(nl_problem* h, long long* out);

/* ---- solver-only drop-in: host Hessian in, increment out ------------------ */
/* SolverCholeskySchur on a Hessian the caller assembled (any U pattern, any W
 * pattern, block-diagonal V with 3x3 blocks): patterns are (row, col) per UID
 * in the reference's storage order (U upper CSC, V diagonal, W CSR). */
typedef struct nl_solver nl_solver;
typedef struct {
  int bu;          /* U block size, 1..9 */
  int nu, nv;      /* number of U / V parameter blocks */
  int nU, nV, nW;  /* block counts */
  int precision;
  int refine_sweeps;
  int device;
} nl_solver_desc;
nl_status nl_solver_create(const nl_solver_desc* d, const int* u_rc, const int* v_rc,
                           const int* w_rc, nl_solver** out);
nl_status nl_solver_destroy(nl_solver* s);
/* Upload U, V, W blocks (row-major per block) and bU, bV (FP64 host). */
nl_status nl_solver_set_hessian(nl_solver* s, const double* U, const double* V,
                                const double* W, const double* bU, const double* bV);
nl_status nl_solver_max_abs_hdiag(nl_solver* s, double* out);
nl_status nl_solver_compute_increment(nl_solver* s, double rel_lambda, double abs_lambda,
                                      double* incU, double* incV, int* ok);
/* nl_set_solver_kind for the solver-only handle. */
nl_status nl_solver_set_kind(nl_solver* s, int kind);

/* ---- SingleSection on the device: SE(2) pose graphs of 2D scans --------- */
/* The reference's single-section problem as its tests build it
 * (nelson/SingleSection.hpp:63-139, nelson/tests/testGaussNewton2DScansAlign.cpp:
 * 36-120): nv variable and nf fixed SE(2) poses (x, y, theta); every edge
 * joins a model pose a and a target pose b with npts point-to-line terms
 * e_k = (T_a m_k - T_b q_k) . (R_a n_k) (model points m and normals n in a's
 * frame, target points q in b's frame).  Edge evaluation, the Hessian blocks
 * (U, b), the damped tiled Cholesky of U (SolverCholeskyDense,
 * nelson/SolverCholeskyDense.hpp:39-67) and the left SE(2) update
 * T <- exp(d) T run on the device; LM / GN control on the host. */
typedef struct nl_pose2d nl_pose2d;
/* nv >= 1 variable poses, nf >= 0 fixed poses */
nl_status nl_pose2d_create(int nv, int nf, int precision, int device, nl_pose2d** out);
nl_status nl_pose2d_destroy(nl_pose2d* h);
/* poses as (x, y, theta) triples; either pointer may be null */
nl_status nl_pose2d_set_poses(nl_pose2d* h, const double* var_xyt, const double* fix_xyt);
nl_status nl_pose2d_get_poses(nl_pose2d* h, double* var_xyt);
/* SingleSection::addEdge with a point-to-line edge; a_fixed / b_fixed select
 * the fixed poses (not both).  Points are (x, y) pairs. */
nl_status nl_pose2d_add_edge(nl_pose2d* h, int a, int a_fixed, int b, int b_fixed, int npts,
                             const double* model_pts, const double* model_normals, const double* target_pts);
/* SingleSection::setUser2InternalIndexes / permuteAMD (nelson/SingleSection.hpp:
 * 26-52); before nl_pose2d_structure_ready */
nl_status nl_pose2d_set_user2internal(nl_pose2d* h, const int* perm);
nl_status nl_pose2d_permute_amd(nl_pose2d* h);
/* Reverse Cuthill-McKee order of the pose graph (no counterpart in the
 * reference): the narrow-profile order for NL_SOLVER_ENVELOPE */
nl_status nl_pose2d_permute_rcm(nl_pose2d* h);
nl_status nl_pose2d_structure_ready(nl_pose2d* h);
/* NL_SOLVER_DENSE (default) or NL_SOLVER_ENVELOPE for the Cholesky of U */
nl_status nl_pose2d_set_solver_kind(nl_pose2d* h, int kind);
/* SingleSection::update: the cost (sum of e_k^2) and, with hessian, U and b */
nl_status nl_pose2d_update(nl_pose2d* h, int hessian, double* chi2);
/* The Hessian of the last update with hessian set, as a dense symmetric
 * (3 nv) x (3 nv) row-major matrix, and b, both in user pose order (the
 * section's hessian().H / b); either pointer may be null */
nl_status nl_pose2d_get_hessian(nl_pose2d* h, double* H, double* b);
/* LevenbergMarquardt::solve / GaussNewton::solve on the section; trace
 * records as for nl_lm_solve (8 doubles: iteration, sub-iteration, chi2, mu,
 * rho, |delta|^2, ok, accepted). */
nl_status nl_pose2d_lm_solve(nl_pose2d* h, const nl_lm_settings* st, nl_solve_report* rep, double* trace,
                             int trace_cap);
nl_status nl_pose2d_gn_solve(nl_pose2d* h, const nl_gn_settings* st, nl_solve_report* rep, double* trace,
                             int trace_cap);

/* ---- user-defined edges: a DoubleSection whose edges the caller evaluates -
 * The reference's DoubleSection with user EdgeBinary / EdgeUnary subclasses
 * (nelson/DoubleSection.hpp:338-365, nelson/EdgeBinary.h:133-157,
 * nelson/EdgeUnary.h:84-92, accumulated by BaseSection::updateHessianBlocks,
 * nelson/BaseSection.cpp:5-86).  The caller owns the parameters and the edge
 * code on the device; the section owns the Hessian, the Schur solve and the
 * LM / GN control.  U blocks have bu = 2, 3, 6 or 9 parameters, V blocks 3. */
typedef struct nl_section nl_section;
#define NL_EDGE_UV 0 /* binary, U block a and V block b */
#define NL_EDGE_UU 1 /* binary, U blocks a != b         */
#define NL_EDGE_U 2  /* unary on U block a              */
#define NL_EDGE_V 3  /* unary on V block a              */
/* Callbacks, run on the calling thread after the section's stream has drained.
 * Device work they start must be on `stream` (a cudaStream_t) or finished when
 * they return.  Return 0 on success; anything else ends the call with
 * NL_ERR_CALLBACK.
 *   evaluate: every edge's whitened residual into r and, if jacobians != 0,
 *     its Jacobian blocks into J (device arrays, offsets of nl_section_layout:
 *     edge e's residual at r + r_off[e] (m_e values), its J_a (m_e x dim_a,
 *     row-major) at J + j_off[e], then J_b (m_e x dim_b) for a binary edge;
 *     dim is bu for a U block, 3 for a V block).  The cost is sum r'r.
 *   oplus: apply the increment (device, user order: incU nu x bu, incV nv x 3).
 *   backup / rollback: keep / restore the parameters (LM only). */
typedef struct {
  void* user;
  int (*evaluate)(void* user, void* stream, int jacobians, double* r, double* J);
  int (*oplus)(void* user, void* stream, const double* incU, const double* incV);
  int (*backup)(void* user, void* stream);
  int (*rollback)(void* user, void* stream);
} nl_section_callbacks;
/* nu >= 1 U blocks of bu parameters, nv >= 0 V blocks of 3 */
nl_status nl_section_create(int bu, int nu, int nv, int precision, int device, nl_section** out);
nl_status nl_section_destroy(nl_section* s);
/* addEdge for n edges: kind NL_EDGE_*, blocks a (and b for binary kinds),
 * residual dimension m (1..64) */
nl_status nl_section_add_edges(nl_section* s, int n, const int* kind, const int* a, const int* b, const int* m);
/* setUser2InternalIndexesU / permuteAMD_SchurU (nelson/DoubleSection.hpp:
 * 23-63); before nl_section_structure_ready */
nl_status nl_section_set_user2internal_u(nl_section* s, const int* perm);
nl_status nl_section_permute_amd_u(nl_section* s);
/* perm[user U block] = internal position */
nl_status nl_section_get_user2internal_u(nl_section* s, int* perm);
nl_status nl_section_structure_ready(nl_section* s);
/* counts after structure_ready: U / W blocks, residual and Jacobian lengths */
nl_status nl_section_get_counts(nl_section* s, int* nU, int* nW, long long* r_len, long long* j_len);
/* per-edge offsets into r and J (ne + 1 entries each) */
nl_status nl_section_layout(nl_section* s, long long* r_off, long long* j_off);
/* the U pattern (nU (row, col) pairs, internal order, upper CSC) and the W
 * pattern (nW (U block, V block) pairs, internal order, CSR) */
nl_status nl_section_get_patterns(nl_section* s, int* u_rc, int* w_rc);
nl_status nl_section_set_callbacks(nl_section* s, const nl_section_callbacks* cb);
nl_status nl_section_set_solver_kind(nl_section* s, int kind);
/* update(hessian): evaluate and accumulate; chi2 may be null */
nl_status nl_section_update(nl_section* s, int hessian, double* chi2);
/* the blocks of the last update with hessian set, in pattern order (U: nU x
 * bu x bu, V: nv x 3 x 3, W: nW x bu x 3, row-major), bU in internal order;
 * any pointer may be null */
nl_status nl_section_get_hessian(nl_section* s, double* U, double* V, double* W, double* bU, double* bV);
/* computeIncrement(rel, abs) on the current Hessian; increments in user order */
nl_status nl_section_compute_increment(nl_section* s, double rel, double abs_, double* incU, double* incV, int* ok);
nl_status nl_section_lm_solve(nl_section* s, const nl_lm_settings* st, nl_solve_report* rep, double* trace,
                              int trace_cap);
nl_status nl_section_gn_solve(nl_section* s, const nl_gn_settings* st, nl_solve_report* rep, double* trace,
                              int trace_cap);

/* Device self-test of the mixed path's tensor-core trailing update: builds a
 * random FP32 matrix of ntiles x 128 rows on `device`, applies the panel-0
 * update with the tcgen05 kernel and with the CUDA-core kernel, and returns
 * max |difference| / max |CUDA-core result| over the updated lower tiles.
 * (No counterpart in the reference: it checks the B200 kernel itself.) */
nl_status nl_selftest_tc_update(int ntiles, unsigned long long seed, int device, double* max_rel_err);
/* The same for the rank-K update of the factorisation's panel groups: panels
 * 0 .. np-1 (np <= 4, K = 128 np) applied in one launch to the trailing tiles
 * np .. ntiles-1, checked against the CUDA-core update panel by panel; then
 * `reps` more launches timed alone (best_ms, CUDA events; may be null). */
nl_status nl_selftest_tc_update_k(int ntiles, int np, unsigned long long seed, int device, int reps,
                                  double* max_rel_err, double* best_ms);

/* ---- cost without any device allocation ---------------------------------- */
/* No counterpart in the reference.  The FP64 cost chi2 = sum_e w_e |r_e|^2 of
 * the projection edges (the value nl_update reports), for callers that must
 * not allocate device memory while they run: a program whose memory pool owns
 * the whole device, a real-time loop that keeps the allocator out of its
 * frames, a host context where allocation calls are forbidden.  It creates no
 * handle and calls no allocator; every input and the output are the caller's
 * device buffers:
 *   d_cam_state  cameras in the device state layout of nl_get_camera_state
 *                (16 doubles: R[9] row-major, t[3], f, k1, k2, pad);
 *   d_pts        points, 3 doubles each;
 *   d_edge_cam / d_edge_pt  per edge, the camera / point row in those arrays;
 *   d_obs        per edge the measured pixel (2 doubles); d_weight per-edge
 *                weights or NULL for 1;
 *   f            focal length of 6-parameter cameras (bc = 6); cx, cy the
 *                principal point;
 *   d_chi2       one double, written on `stream` (a cudaStream_t, 0 = the
 *                default stream); the call returns after enqueueing.
 * Its scratch (32 KB of partial sums) is a fixed array inside the library,
 * present on every GPU that loads it until the process exits.  At most
 * NL_NOALLOC_MAX_EDGES edges; larger ne is rejected with NL_ERR_ARG.  The
 * first call on a device looks up that array's address (with that device
 * current); make it before any stream capture.  That address is kept for the
 * life of the process: after cudaDeviceReset on a device, do not call this
 * function on that device again (the kept address would be stale).  All calls
 * share the array:
 * calls whose work overlaps on the GPU (other streams, other threads) race and
 * must be serialised by the caller. */
#define NL_NOALLOC_MAX_EDGES 16777216
nl_status nl_ba_cost_noalloc(int bc, int ne, const double* d_cam_state, const double* d_pts,
                             const int* d_edge_cam, const int* d_edge_pt, const double* d_obs,
                             const double* d_weight, double f, double cx, double cy, double* d_chi2,
                             void* stream);

const char* nl_status_string(int status);
/* Library build identification: "nelson_b200 <version> sm_100a". */
const char* nl_version(void);

#ifdef __cplusplus
}
#endif
#endif

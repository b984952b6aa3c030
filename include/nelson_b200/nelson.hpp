// nelson.hpp -- header-only C++ classes over the C ABI of nelson_b200.h, in
// the shapes nelson's own code uses, so that a nelson user swaps the solver
// id and the section type and keeps the rest of the program:
//
//   nelson                                          nelson_b200
//   DoubleSection<..., EdgeBinaryUV projection>     BASection
//     (nelson/DoubleSection.h:24-330)
//   SolverCholeskySchur (SolverCholeskySchur.h)     SolverCholeskySchurCuda
//   LevenbergMarquardt<Solver> (LevenbergMarquardt.h/.hpp)
//                                                   LevenbergMarquardt<Solver>
//   GaussNewton<Solver> (GaussNewton.h/.hpp)        GaussNewton<Solver>
//   LevenbergMarquardtSettings / GaussNewtonSettings  same names and defaults
//   DoubleSection subclass with user EdgeBinary /  DeviceEdgeSection subclass
//     EdgeUnary edges (DoubleSection.hpp:338-365)    with device edge code
//   SingleSection of SE(2) poses, point-to-line     ScanAlignSection
//     edges (tests/testGaussNewton2DScansAlign.cpp)
//
// The solvers meet the reference's Solver concept (nelson/SolverCholeskySchur.h:
// 71-115: Type, hasSettings, Settings, init(H, b), maxAbsHDiag(),
// computeIncrement(H, b, relLambda, absLambda), incrementVector(),
// incrementVectorSquaredNorm()) and BASection meets the problem concept
// LevenbergMarquardt / GaussNewton use (update(bool), hessian().H() / b() /
// chi2() / maxAbsValBVect(), oplus(inc), backupSolution(), rollbackSolution(),
// computeRhoChi2Change(mu, inc, oldChi2)), so the reference's own
// LevenbergMarquardt<Solver>::solve(op) instantiates with them unchanged.
// The H and b a BASection hands out are handles of its device-resident
// Hessian (DeviceHessianMatrices / DeviceHessianVectors); a Hessian assembled
// on the host goes through SolverCholeskySchurCudaHost instead.
//
// LevenbergMarquardt::solve / GaussNewton::solve below are written against
// exactly those calls, in the reference's order (nelson/LevenbergMarquardt.hpp:
// 36-146, nelson/GaussNewton.hpp:32-127); solveOnDevice() runs the same loop
// entirely on the GPU (nl_lm_solve / nl_gn_solve) and is what a production
// caller uses.
//
// Errors: every failing C-ABI call throws nelson_b200::Error carrying the
// nl_status.  A Cholesky failure of the reduced system is not an error: it is
// the `false` return of computeIncrement, as in the reference.
#ifndef NELSON_B200_NELSON_HPP
#define NELSON_B200_NELSON_HPP

#include <algorithm>
#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../nelson_b200.h"

namespace nelson_b200 {

class Error : public std::runtime_error {
 public:
  Error(nl_status s, const std::string& what)
      : std::runtime_error(what + ": " + nl_status_string(s)), status_(s) {}
  nl_status status() const { return status_; }

 private:
  nl_status status_;
};

inline void check(nl_status s, const char* what) {
  if (s != NL_OK) throw Error(s, what);
}

// NodeType / NodeId (nelson/EdgeInterface.h:35-55): an id of a variable or of
// a fixed parameter block.
enum class NodeType { Variable, Fixed };
struct NodeId {
  int id = 0;
  NodeType type = NodeType::Variable;
  NodeId() = default;
  explicit NodeId(int i, NodeType t = NodeType::Variable) : id(i), type(t) {}
  static NodeId fixed(int i) { return NodeId(i, NodeType::Fixed); }
};

// nelson/LevenbergMarquardt.h:18-34, defaults nelson/LevenbergMarquardt.cpp:6-19.
struct LevenbergMarquardtSettings {
  int maxNumIt = 100;
  int maxNumSubIt = 10;
  int minNumIt = 0;
  double epsBVector = 1e-15;
  double epsIncSquare = 1e-30;
  double epsChi2 = 1e-15;
  double tau = 1e-3;
  double penaltyV = 2.0;
  double initV = 2.0;
  double maxScaleFactor = 2.0 / 3.0;
  double minScaleFactor = 1.0 / 3.0;
  nl_lm_settings c() const {
    return nl_lm_settings{maxNumIt, maxNumSubIt, minNumIt, epsBVector, epsIncSquare, epsChi2,
                          tau, penaltyV, initV, maxScaleFactor, minScaleFactor};
  }
};

// nelson/GaussNewton.h:18-30, defaults nelson/GaussNewton.cpp:12-22.
struct GaussNewtonSettings {
  int maxNumIt = 100;
  int minNumIt = 0;
  double epsBVector = 1e-15;
  double epsIncSquare = 1e-30;
  double epsChi2 = 1e-15;
  double absLambda = 0.0;
  double relLambda = 0.0;
  nl_gn_settings c() const {
    return nl_gn_settings{maxNumIt, minNumIt, epsBVector, epsIncSquare, epsChi2, absLambda,
                          relLambda};
  }
};

// nelson/LevenbergMarquardt.h:36-44 (GaussNewton uses the first six).
enum class TerminationReason {
  SuccessAtStart = NL_SUCCESS_AT_START,
  SuccessSmallIncrement = NL_SUCCESS_SMALL_INCREMENT,
  SuccessEpsB = NL_SUCCESS_EPS_B,
  SuccessSmallResiduals = NL_SUCCESS_SMALL_RESIDUALS,
  SolverFailure = NL_SOLVER_FAILURE,
  MaxIterationReached = NL_MAX_ITERATION_REACHED,
  MaxSubIterationReached = NL_MAX_SUBITERATION_REACHED
};

// One record per sub-iteration (the content of LevenbergMarquardtStats,
// nelson/LevenbergMarquardt.h:57-85, plus damping and gain ratio).
struct IterationRecord {
  int it, subit;
  double chi2, mu, rho, incSquaredNorm;
  bool solverOk, accepted;
};

// ---------------------------------------------------------------------------
// The Hessian blocks [U W; W' V], the gradient b and the increment of a
// BASection live on the device.  These handles stand where the reference
// passes DoubleSectionHessianMatrices and DoubleSectionHessianVectors
// (nelson/DoubleSectionHessian.h:37-141): a solver or a problem that receives
// one works on the device data of the handle's section.
struct DeviceHessianMatrices {
  nl_problem* h = nullptr;
};
struct DeviceHessianVectors {
  enum class Kind { Gradient, Increment };
  nl_problem* h = nullptr;
  Kind kind = Kind::Gradient;
  // Host copies, bU in internal camera order (the reference's bU() / bV()).
  void get(std::vector<double>& bU, std::vector<double>& bV, int numU, int numV, int bc) const {
    bU.resize(size_t(numU) * bc);
    bV.resize(size_t(numV) * 3);
    if (kind == Kind::Increment)
      check(nl_get_increment(h, bU.data(), bV.data()), "nl_get_increment");
    else
      check(nl_get_hessian(h, nullptr, nullptr, nullptr, bU.data(), bV.data()), "nl_get_hessian");
  }
};

// ---------------------------------------------------------------------------
// BASection: a DoubleSection of cameras (U, 6 or 9 parameters) and points
// (V, 3 parameters) joined by the projection EdgeBinaryUV, resident on one
// GPU.  Call order as in the reference: construct (parametersReady), addEdge
// ..., optionally setUser2InternalIndexesU, structureReady, then solve.
class BASection {
 public:
  BASection(int bc, int numCameras, int numPoints, int numFixedCameras = 0,
            int numFixedPoints = 0, int precision = NL_PREC_MIXED, double f = 500.0,
            double cx = 320.0, double cy = 240.0, int device = 0, int refineSweeps = -1) {
    nl_problem_desc d{};
    d.bc = bc;
    d.nc_var = numCameras;
    d.nc_fix = numFixedCameras;
    d.np_var = numPoints;
    d.np_fix = numFixedPoints;
    d.precision = precision;
    d.f = f;
    d.cx = cx;
    d.cy = cy;
    d.refine_sweeps = refineSweeps;
    d.device = device;
    check(nl_create(&d, &h_), "nl_create");
    desc_ = d;
    hessian_ = Hessian(h_);
  }
  ~BASection() {
    if (h_) nl_destroy(h_);
  }
  BASection(const BASection&) = delete;
  BASection& operator=(const BASection&) = delete;
  BASection(BASection&& o) noexcept : h_(std::exchange(o.h_, nullptr)), desc_(o.desc_), hessian_(h_) {}

  nl_problem* handle() const { return h_; }
  int cameraBlockSize() const { return desc_.bc; }
  int numParametersU() const { return desc_.nc_var; }
  int numParametersV() const { return desc_.np_var; }

  // Cameras: axis-angle[3], t[3] (, f, k1, k2), variable cameras then fixed;
  // points: xyz, variable then fixed.
  void setParameters(const std::vector<double>& cams, const std::vector<double>& pts) {
    const size_t nc = size_t(desc_.nc_var + desc_.nc_fix), np = size_t(desc_.np_var + desc_.np_fix);
    if (cams.size() != nc * desc_.bc || pts.size() != np * 3)
      throw Error(NL_ERR_ARG, "setParameters: sizes");
    check(nl_set_params(h_, cams.data(), pts.data()), "nl_set_params");
  }
  void getParameters(std::vector<double>& cams, std::vector<double>& pts) const {
    cams.resize(size_t(desc_.nc_var + desc_.nc_fix) * desc_.bc);
    pts.resize(size_t(desc_.np_var + desc_.np_fix) * 3);
    check(nl_get_params(h_, cams.data(), pts.data()), "nl_get_params");
  }
  // DoubleSection::parametersReady (nelson/DoubleSection.hpp:67-80): the
  // parameter counts are fixed by the constructor; kept for call-order parity.
  void parametersReady() {}

  // DoubleSection::addEdge(NodeId, NodeId, EdgeBinaryUV*) (DoubleSection.hpp:338-365),
  // with the projection edge given by its observation (and optional weight).
  void addEdge(NodeId cam, NodeId pt, double u, double v, double weight = 1.0) {
    cam_.push_back(cam.id);
    camFixed_.push_back(cam.type == NodeType::Fixed);
    pt_.push_back(pt.id);
    ptFixed_.push_back(pt.type == NodeType::Fixed);
    obs_.push_back(u);
    obs_.push_back(v);
    w_.push_back(weight);
  }
  // DoubleSection::setUser2InternalIndexesU (nelson/DoubleSection.hpp:23-27).
  void setUser2InternalIndexesU(const std::vector<int>& perm) {
    if (perm.size() != size_t(desc_.nc_var)) throw Error(NL_ERR_ARG, "setUser2InternalIndexesU");
    check(nl_set_user2internal_u(h_, perm.data()), "nl_set_user2internal_u");
  }
  // DoubleSection::permuteAMD_SchurU (nelson/DoubleSection.hpp:30-63): the
  // approximate minimum degree order of the camera graph (the pattern of
  // U + W W'), applied when the structure is built (structureReady).
  void permuteAMD_SchurU() { order_ = Order::Amd; }
  // Alternatively a reverse Cuthill-McKee order of the same graph: it narrows
  // the envelope that SolverEnvelopeSchurCuda factors.
  void permuteRCM_SchurU() { order_ = Order::Rcm; }
  // DoubleSection::structureReady (nelson/DoubleSection.hpp:83-246).
  void structureReady() {
    const bool weighted = std::any_of(w_.begin(), w_.end(), [](double x) { return x != 1.0; });
    check(nl_add_ba_edges(h_, int(cam_.size()), cam_.data(), camFixed_.data(), pt_.data(),
                          ptFixed_.data(), obs_.data(), weighted ? w_.data() : nullptr),
          "nl_add_ba_edges");
    if (order_ == Order::Rcm) check(nl_permute_rcm_u(h_), "nl_permute_rcm_u");
    if (order_ == Order::Amd) check(nl_permute_amd_u(h_), "nl_permute_amd_u");
    check(nl_structure_ready(h_), "nl_structure_ready");
    std::vector<int>().swap(cam_);
    std::vector<int>().swap(camFixed_);
    std::vector<int>().swap(pt_);
    std::vector<int>().swap(ptFixed_);
    std::vector<double>().swap(obs_);
    std::vector<double>().swap(w_);
  }

  // ---- the problem concept used by LevenbergMarquardt / GaussNewton ----
  // DoubleSection::update(bool) (nelson/DoubleSection.hpp:452-467).
  void update(bool computeHessian) {
    double c;
    check(nl_update(h_, computeHessian ? 1 : 0, &c), "nl_update");
  }
  // DoubleSection::hessian() (nelson/DoubleSection.h:265-272): H(), b(),
  // chi2(), maxAbsValBVect() of the section's device-resident Hessian.
  class Hessian {
   public:
    explicit Hessian(nl_problem* h = nullptr) : H_{h}, b_{h, DeviceHessianVectors::Kind::Gradient} {}
    DeviceHessianMatrices& H() { return H_; }
    const DeviceHessianMatrices& H() const { return H_; }
    const DeviceHessianVectors& b() const { return b_; }
    double chi2() const {
      double c;
      check(nl_chi2(H_.h, &c), "nl_chi2");
      return c;
    }
    double maxAbsValBVect() const {
      double b;
      check(nl_max_abs_b(H_.h, &b), "nl_max_abs_b");
      return b;
    }

   private:
    DeviceHessianMatrices H_;
    DeviceHessianVectors b_;
  };
  Hessian& hessian() { return hessian_; }
  const Hessian& hessian() const { return hessian_; }

  // oplus(inc) with the increment a solver computed on this section (the
  // increment stays on the device).
  void oplus(const DeviceHessianVectors& inc) {
    if (inc.h != h_ || inc.kind != DeviceHessianVectors::Kind::Increment)
      throw Error(NL_ERR_ARG, "oplus: not this section's increment");
    check(nl_oplus(h_), "nl_oplus");
  }
  void backupSolution() { check(nl_backup(h_), "nl_backup"); }
  void rollbackSolution() { check(nl_rollback(h_), "nl_rollback"); }
  // DoubleSection::computeRhoChi2Change (nelson/DoubleSection.h:300-311):
  // (oldChi2 - chi2) / (inc' (mu inc - b)).
  double computeRhoChi2Change(double mu, const DeviceHessianVectors& inc, double oldChi2) const {
    if (inc.h != h_ || inc.kind != DeviceHessianVectors::Kind::Increment)
      throw Error(NL_ERR_ARG, "computeRhoChi2Change: not this section's increment");
    double r;
    check(nl_rho(h_, mu, oldChi2, &r), "nl_rho");
    return r;
  }

 private:
  nl_problem* h_ = nullptr;
  nl_problem_desc desc_{};
  Hessian hessian_;
  std::vector<int> cam_, camFixed_, pt_, ptFixed_;
  enum class Order { User, Amd, Rcm };
  Order order_ = Order::User;
  std::vector<double> obs_, w_;
};

// ---------------------------------------------------------------------------
// SolverCholeskySchur's Solver concept (nelson/SolverCholeskySchur.h:71-115)
// on a BASection's device-resident Hessian: init(H, b) binds the section the
// handles name, computeIncrement(H, b, rel, abs) runs the whole Schur
// increment on the device, incrementVector() is the handle of the device
// increment that the section's oplus / computeRhoChi2Change accept.
class SolverCholeskySchurCuda {
 public:
  using Type = double;
  static constexpr bool hasSettings = false;
  class Settings {};

  // SolverCholeskySchur::init (nelson/SolverCholeskySchur.hpp:44-62).
  void init(DeviceHessianMatrices& H, const DeviceHessianVectors& b) {
    if (!H.h || b.h != H.h) throw Error(NL_ERR_ARG, "init: H and b of different sections");
    h_ = H.h;
    inc_ = DeviceHessianVectors{h_, DeviceHessianVectors::Kind::Increment};
    check(nl_solver_init(h_), "nl_solver_init");
    check(nl_set_solver_kind(h_, kind()), "nl_set_solver_kind");
  }
  // SolverCholeskySchur::maxAbsHDiag (nelson/SolverCholeskySchur.hpp:75-78).
  double maxAbsHDiag() const {
    double m;
    check(nl_max_abs_hdiag(h_, &m), "nl_max_abs_hdiag");
    return m;
  }
  // computeIncrement(H, b, relLambda, absLambda) (SolverCholeskySchur.hpp:91-157):
  // false when a damped block or the reduced system is not positive definite
  // (the increment is then zero).
  bool computeIncrement(DeviceHessianMatrices& H, const DeviceHessianVectors& b, double relLambda,
                        double absLambda) {
    if (H.h != h_ || b.h != h_) throw Error(NL_ERR_STATE, "computeIncrement: solver initialised on another section");
    int ok = 0;
    check(nl_compute_increment(h_, relLambda, absLambda, &ok), "nl_compute_increment");
    return ok != 0;
  }
  const DeviceHessianVectors& incrementVector() const { return inc_; }
  double incrementVectorSquaredNorm() const {
    double s;
    check(nl_inc_sqnorm(h_, &s), "nl_inc_sqnorm");
    return s;
  }
  // The phases of SolverCholeskySchurTimeStat (nelson/SolverCholeskySchur.h:25-38).
  nl_phase_times timingStats() const {
    nl_phase_times t{};
    check(nl_phase_timings(h_, &t), "nl_phase_timings");
    return t;
  }
  // the factorisation this solver stands for, on p's handle (solveOnDevice)
  void select(BASection& p) const { check(nl_set_solver_kind(p.handle(), kind()), "nl_set_solver_kind"); }

 protected:
  virtual int kind() const { return NL_SOLVER_DENSE; }

 private:
  nl_problem* h_ = nullptr;
  DeviceHessianVectors inc_;

 public:
  virtual ~SolverCholeskySchurCuda() = default;
};

// The solver that takes SolverDiagonalBlocksInverseWWtMultSchur's place in
// the solver choice (nelson/SolverDiagonalBlocksInverseWWtMultSchur.hpp:36-140):
// the same Schur complement, factored over its Cholesky envelope only
// (NL_SOLVER_ENVELOPE); its increments are SolverCholeskySchurCuda's.
class SolverEnvelopeSchurCuda : public SolverCholeskySchurCuda {
 protected:
  int kind() const override { return NL_SOLVER_ENVELOPE; }
};

// ---------------------------------------------------------------------------
// SolverCholeskySchur on a Hessian assembled on the host (any edge types the
// device does not evaluate): the Solver concept over the caller's own
// Hessian matrices / vectors types, read and written through an access
// traits class.  HostHessianAccess<Matrices, Vectors> provides
//   static int bu(const Matrices&)                      U block size
//   static int numU(const Matrices&), numV(const Matrices&)   parameter blocks
//   static void patterns(const Matrices&, std::vector<int>& u_rc,
//                        std::vector<int>& v_rc, std::vector<int>& w_rc)
//       (row, col) per block UID in the reference's storage order: U upper
//       CSC, V diagonal, W CSR (nelson/DoubleSection.hpp:157-191)
//   static void values(const Matrices&, std::vector<double>& U,
//                      std::vector<double>& V, std::vector<double>& W)
//       the blocks in UID order, each row-major
//   static void gradient(const Vectors&, std::vector<double>& bU, std::vector<double>& bV)
//   static void setIncrement(Vectors& inc, const Vectors& like, const std::vector<double>& incU,
//                            const std::vector<double>& incV)
// The reference's mat-based DoubleSectionHessianMatrices is read with its own
// block iterators (outerSize / begin(col) / row / col / block / blockUID) in a
// specialisation the integrating program writes; HostBlockHessian below is a
// self-contained stand-in that has one.
template <class Matrices, class Vectors>
struct HostHessianAccess;

template <class Matrices, class Vectors, class Access = HostHessianAccess<Matrices, Vectors>>
class SolverCholeskySchurCudaHost {
 public:
  using Type = double;
  static constexpr bool hasSettings = true;
  struct Settings {
    int precision = NL_PREC_FP64;
    int refineSweeps = -1;
    int device = 0;
    int kind = NL_SOLVER_DENSE;
  };
  Settings& settings() { return settings_; }
  const Settings& settings() const { return settings_; }

  SolverCholeskySchurCudaHost() = default;
  SolverCholeskySchurCudaHost(const SolverCholeskySchurCudaHost&) = delete;
  SolverCholeskySchurCudaHost& operator=(const SolverCholeskySchurCudaHost&) = delete;
  ~SolverCholeskySchurCudaHost() {
    if (s_) nl_solver_destroy(s_);
  }

  // init(H, b): the block pattern is fixed here (nelson/SolverCholeskySchur.hpp:44-62).
  void init(Matrices& H, const Vectors& b) {
    if (s_) nl_solver_destroy(s_);
    s_ = nullptr;
    std::vector<int> u_rc, v_rc, w_rc;
    Access::patterns(H, u_rc, v_rc, w_rc);
    nl_solver_desc d{};
    d.bu = Access::bu(H);
    d.nu = Access::numU(H);
    d.nv = Access::numV(H);
    d.nU = int(u_rc.size() / 2);
    d.nV = int(v_rc.size() / 2);
    d.nW = int(w_rc.size() / 2);
    d.precision = settings_.precision;
    d.refine_sweeps = settings_.refineSweeps;
    d.device = settings_.device;
    check(nl_solver_create(&d, u_rc.data(), v_rc.data(), w_rc.data(), &s_), "nl_solver_create");
    check(nl_solver_set_kind(s_, settings_.kind), "nl_solver_set_kind");
    bu_ = d.bu;
    nu_ = d.nu;
    nv_ = d.nv;
    upload(H, b);
    incU_.assign(size_t(nu_) * bu_, 0.0);
    incV_.assign(size_t(nv_) * 3, 0.0);
    Access::setIncrement(inc_, b, incU_, incV_);
  }
  double maxAbsHDiag() const {
    double m;
    check(nl_solver_max_abs_hdiag(s_, &m), "nl_solver_max_abs_hdiag");
    return m;
  }
  bool computeIncrement(Matrices& H, const Vectors& b, double relLambda, double absLambda) {
    upload(H, b);
    int ok = 0;
    check(nl_solver_compute_increment(s_, relLambda, absLambda, incU_.data(), incV_.data(), &ok),
          "nl_solver_compute_increment");
    Access::setIncrement(inc_, b, incU_, incV_);
    return ok != 0;
  }
  const Vectors& incrementVector() const { return inc_; }
  double incrementVectorSquaredNorm() const {
    double s = 0;
    for (double x : incU_) s += x * x;
    for (double x : incV_) s += x * x;
    return s;
  }

 private:
  void upload(const Matrices& H, const Vectors& b) {
    Access::values(H, U_, V_, W_);
    Access::gradient(b, bU_, bV_);
    check(nl_solver_set_hessian(s_, U_.data(), V_.data(), W_.data(), bU_.data(), bV_.data()),
          "nl_solver_set_hessian");
  }
  Settings settings_;
  nl_solver* s_ = nullptr;
  int bu_ = 0, nu_ = 0, nv_ = 0;
  std::vector<double> U_, V_, W_, bU_, bV_, incU_, incV_;
  Vectors inc_{};
};

// A self-contained host block Hessian in the reference's storage order, with
// its HostHessianAccess: U (bu x bu blocks, upper CSC), V (3 x 3 diagonal
// blocks), W (bu x 3, CSR), each block row-major, and the vectors bU (internal
// camera order) / bV.
struct HostBlockHessian {
  int bu = 0, numU = 0, numV = 0;
  std::vector<int> u_rc, v_rc, w_rc;  // (row, col) per UID
  std::vector<double> U, V, W;        // blocks in UID order
  void setZero() {
    std::fill(U.begin(), U.end(), 0.0);
    std::fill(V.begin(), V.end(), 0.0);
    std::fill(W.begin(), W.end(), 0.0);
  }
};
struct HostBlockVectors {
  std::vector<double> bU, bV;
  void setZero() {
    std::fill(bU.begin(), bU.end(), 0.0);
    std::fill(bV.begin(), bV.end(), 0.0);
  }
};
template <>
struct HostHessianAccess<HostBlockHessian, HostBlockVectors> {
  static int bu(const HostBlockHessian& H) { return H.bu; }
  static int numU(const HostBlockHessian& H) { return H.numU; }
  static int numV(const HostBlockHessian& H) { return H.numV; }
  static void patterns(const HostBlockHessian& H, std::vector<int>& u, std::vector<int>& v, std::vector<int>& w) {
    u = H.u_rc;
    v = H.v_rc;
    w = H.w_rc;
  }
  static void values(const HostBlockHessian& H, std::vector<double>& U, std::vector<double>& V,
                     std::vector<double>& W) {
    U = H.U;
    V = H.V;
    W = H.W;
  }
  static void gradient(const HostBlockVectors& b, std::vector<double>& bU, std::vector<double>& bV) {
    bU = b.bU;
    bV = b.bV;
  }
  static void setIncrement(HostBlockVectors& inc, const HostBlockVectors&, const std::vector<double>& incU,
                           const std::vector<double>& incV) {
    inc.bU = incU;
    inc.bV = incV;
  }
};

// ---------------------------------------------------------------------------
// LevenbergMarquardt<Solver> (nelson/LevenbergMarquardt.h:46-118).
template <class Solver = SolverCholeskySchurCuda>
class LevenbergMarquardt {
 public:
  LevenbergMarquardtSettings& settings() { return settings_; }
  const std::vector<IterationRecord>& stats() const { return stats_; }
  int numIterations() const { return iter_; }
  Solver& solver() { return solver_; }

  // nelson/LevenbergMarquardt.hpp:36-146: the reference's calls on the
  // problem and solver concepts, in its order (one C-ABI call per step for a
  // BASection).  Records one IterationRecord per sub-iteration.
  template <class OptimizationProblem>
  TerminationReason solve(OptimizationProblem& op) {
    const auto& s = settings_;
    using T = typename Solver::Type;
    stats_.clear();
    iter_ = -1;
    op.update(true);
    push(-1, -1, op.hessian().chi2(), 0, 0, 0, true, true);
    if (op.hessian().maxAbsValBVect() <= s.epsBVector) return TerminationReason::SuccessAtStart;
    op.backupSolution();
    T oldChi2 = op.hessian().chi2();
    solver_.init(op.hessian().H(), op.hessian().b());
    T mu = s.tau * solver_.maxAbsHDiag();
    T curV = s.initV;
    iter_ = 0;
    while (iter_ < s.maxNumIt) {
      int subiter = 0;
      bool toRepeat = false;
      do {
        const T muUsed = mu;
        const bool solveOk = solver_.computeIncrement(op.hessian().H(), op.hessian().b(), 0, mu);
        const T inc = solver_.incrementVectorSquaredNorm();
        if (solveOk && iter_ >= s.minNumIt && inc <= s.epsIncSquare) {
          push(iter_, subiter, op.hessian().chi2(), muUsed, 0, inc, true, false);
          return TerminationReason::SuccessSmallIncrement;
        }
        T rho = -1, chi2 = -1;
        if (solveOk) {
          op.oplus(solver_.incrementVector());
          op.update(false);
          chi2 = op.hessian().chi2();
          rho = op.computeRhoChi2Change(mu, solver_.incrementVector(), oldChi2);
        }
        const bool accepted = solveOk && rho > 0;
        push(iter_, subiter, chi2, muUsed, rho, inc, solveOk, accepted);
        if (accepted) {
          if (iter_ > s.minNumIt && op.hessian().maxAbsValBVect() <= s.epsBVector)
            return TerminationReason::SuccessEpsB;
          if (iter_ > s.minNumIt && op.hessian().chi2() < s.epsChi2) return TerminationReason::SuccessSmallResiduals;
          const T fc = 2 * rho - 1;
          T alpha = std::min(T(s.maxScaleFactor), 1 - fc * fc * fc);
          alpha = std::max(T(s.minScaleFactor), alpha);
          mu = mu * alpha;
          curV = s.initV;
        } else {
          op.rollbackSolution();
          mu = mu * curV;
          curV = curV * s.penaltyV;
        }
        ++subiter;
        if (subiter >= s.maxNumSubIt) return TerminationReason::MaxSubIterationReached;
        toRepeat = !accepted;
      } while (toRepeat);
      op.update(true);
      op.backupSolution();
      oldChi2 = op.hessian().chi2();
      ++iter_;
    }
    return TerminationReason::MaxIterationReached;
  }

  // The same loop with every step on the device (nl_lm_solve).
  TerminationReason solveOnDevice(BASection& P, nl_solve_report* report = nullptr) {
    solver_.select(P);
    const nl_lm_settings c = settings_.c();
    nl_solve_report rep{};
    std::vector<double> tr(size_t(settings_.maxNumIt + 1) * (settings_.maxNumSubIt + 1) *
                           NL_TRACE_STRIDE);
    check(nl_lm_solve(P.handle(), &c, &rep, tr.data(), int(tr.size() / NL_TRACE_STRIDE)),
          "nl_lm_solve");
    stats_.clear();
    for (int k = 0; k < rep.n_trace; k++) {
      const double* t = &tr[size_t(k) * NL_TRACE_STRIDE];
      stats_.push_back({int(t[0]), int(t[1]), t[2], t[3], t[4], t[5], t[6] != 0, t[7] != 0});
    }
    iter_ = rep.iterations;
    if (report) *report = rep;
    return TerminationReason(rep.reason);
  }

 private:
  void push(int it, int sub, double chi2, double mu, double rho, double inc, bool ok, bool acc) {
    stats_.push_back({it, sub, chi2, mu, rho, inc, ok, acc});
  }
  LevenbergMarquardtSettings settings_;
  Solver solver_;
  std::vector<IterationRecord> stats_;
  int iter_ = -1;
};

// GaussNewton<Solver> (nelson/GaussNewton.h:43-96).
template <class Solver = SolverCholeskySchurCuda>
class GaussNewton {
 public:
  GaussNewtonSettings& settings() { return settings_; }
  const std::vector<IterationRecord>& stats() const { return stats_; }
  int numIterations() const { return iter_; }
  Solver& solver() { return solver_; }

  // nelson/GaussNewton.hpp:32-127: the reference's calls, in its order.
  template <class OptimizationProblem>
  TerminationReason solve(OptimizationProblem& op) {
    const auto& s = settings_;
    stats_.clear();
    iter_ = -1;
    op.update(true);
    stats_.push_back({-1, 0, op.hessian().chi2(), 0, 0, 0, true, true});
    if (op.hessian().maxAbsValBVect() <= s.epsBVector) return TerminationReason::SuccessAtStart;
    solver_.init(op.hessian().H(), op.hessian().b());
    iter_ = 0;
    while (iter_ < s.maxNumIt) {
      const bool solveOk = solver_.computeIncrement(op.hessian().H(), op.hessian().b(), s.relLambda, s.absLambda);
      if (!solveOk) {
        stats_.push_back({iter_, 0, -1, 0, 0, 0, false, false});
        return TerminationReason::SolverFailure;
      }
      const double inc = solver_.incrementVectorSquaredNorm();
      if (iter_ >= s.minNumIt && inc <= s.epsIncSquare) {
        stats_.push_back({iter_, 0, op.hessian().chi2(), 0, 0, inc, true, false});
        return TerminationReason::SuccessSmallIncrement;
      }
      op.oplus(solver_.incrementVector());
      op.update(true);
      stats_.push_back({iter_, 0, op.hessian().chi2(), 0, 0, inc, true, true});
      if (iter_ > s.minNumIt && op.hessian().maxAbsValBVect() <= s.epsBVector)
        return TerminationReason::SuccessEpsB;
      if (iter_ > s.minNumIt && op.hessian().chi2() < s.epsChi2) return TerminationReason::SuccessSmallResiduals;
      ++iter_;
    }
    return TerminationReason::MaxIterationReached;
  }

  TerminationReason solveOnDevice(BASection& P, nl_solve_report* report = nullptr) {
    solver_.select(P);
    const nl_gn_settings c = settings_.c();
    nl_solve_report rep{};
    std::vector<double> tr(size_t(settings_.maxNumIt + 2) * NL_TRACE_STRIDE);
    check(nl_gn_solve(P.handle(), &c, &rep, tr.data(), int(tr.size() / NL_TRACE_STRIDE)),
          "nl_gn_solve");
    stats_.clear();
    for (int k = 0; k < rep.n_trace; k++) {
      const double* t = &tr[size_t(k) * NL_TRACE_STRIDE];
      stats_.push_back({int(t[0]), int(t[1]), t[2], t[3], t[4], t[5], t[6] != 0, t[7] != 0});
    }
    iter_ = rep.iterations;
    if (report) *report = rep;
    return TerminationReason(rep.reason);
  }

 private:
  GaussNewtonSettings settings_;
  Solver solver_;
  std::vector<IterationRecord> stats_;
  int iter_ = -1;
};

// ---------------------------------------------------------------------------
// ScanAlignSection: a SingleSection (nelson/SingleSection.hpp:26-139) of SE(2)
// poses (x, y, theta) joined by point-to-line edges, the problem of
// nelson/tests/testGaussNewton2DScansAlign.cpp:36-120, resident on one GPU.
// Call order as in the reference: construct, setPoses, addEdge ...,
// optionally permuteAMD / setUser2InternalIndexes, structureReady, then
// solveLM / solveGN (the loops of LevenbergMarquardt.hpp:36-146 and
// GaussNewton.hpp:32-127 on this section, with the tiled Cholesky of U).
class ScanAlignSection {
 public:
  ScanAlignSection(int numPoses, int numFixedPoses = 1, int precision = NL_PREC_FP64, int device = 0)
      : nv_(numPoses), nf_(numFixedPoses) {
    check(nl_pose2d_create(numPoses, numFixedPoses, precision, device, &h_), "nl_pose2d_create");
  }
  ~ScanAlignSection() {
    if (h_) nl_pose2d_destroy(h_);
  }
  ScanAlignSection(const ScanAlignSection&) = delete;
  ScanAlignSection& operator=(const ScanAlignSection&) = delete;

  int numParameters() const { return nv_; }
  // (x, y, theta) triples; either may be null
  void setPoses(const double* variable, const double* fixed) {
    check(nl_pose2d_set_poses(h_, variable, fixed), "nl_pose2d_set_poses");
  }
  std::vector<double> poses() const {
    std::vector<double> p(size_t(nv_) * 3);
    check(nl_pose2d_get_poses(h_, p.data()), "nl_pose2d_get_poses");
    return p;
  }
  // addEdge(NodeId a, NodeId b, new PointLineEdge(model, normals, target)):
  // npts (x, y) pairs each; model points and normals in a's frame, target
  // points in b's frame
  void addEdge(NodeId a, NodeId b, int npts, const double* model, const double* normals, const double* target) {
    check(nl_pose2d_add_edge(h_, a.id, a.type == NodeType::Fixed, b.id, b.type == NodeType::Fixed, npts, model,
                             normals, target),
          "nl_pose2d_add_edge");
  }
  void permuteAMD() { check(nl_pose2d_permute_amd(h_), "nl_pose2d_permute_amd"); }
  void permuteRCM() { check(nl_pose2d_permute_rcm(h_), "nl_pose2d_permute_rcm"); }
  void setUser2InternalIndexes(const std::vector<int>& perm) {
    if ((int)perm.size() != nv_) throw Error(NL_ERR_ARG, "setUser2InternalIndexes");
    check(nl_pose2d_set_user2internal(h_, perm.data()), "nl_pose2d_set_user2internal");
  }
  void structureReady() { check(nl_pose2d_structure_ready(h_), "nl_pose2d_structure_ready"); }
  void setSolverKind(int kind) { check(nl_pose2d_set_solver_kind(h_, kind), "nl_pose2d_set_solver_kind"); }
  // update(hessian): returns chi2 (hessian().chi2())
  double update(bool hessian) {
    double c = 0.0;
    check(nl_pose2d_update(h_, hessian ? 1 : 0, &c), "nl_pose2d_update");
    return c;
  }
  // hessian().H() (dense, symmetric, user pose order) and b()
  void hessian(std::vector<double>& H, std::vector<double>& b) const {
    const size_t n = size_t(nv_) * 3;
    H.resize(n * n);
    b.resize(n);
    check(nl_pose2d_get_hessian(h_, H.data(), b.data()), "nl_pose2d_get_hessian");
  }
  TerminationReason solveLM(const LevenbergMarquardtSettings& st = {}, std::vector<IterationRecord>* trace = nullptr) {
    const nl_lm_settings c = st.c();
    return solve([&](nl_solve_report* r, double* t, int cap) { return nl_pose2d_lm_solve(h_, &c, r, t, cap); },
                 trace, "nl_pose2d_lm_solve");
  }
  TerminationReason solveGN(const GaussNewtonSettings& st = {}, std::vector<IterationRecord>* trace = nullptr) {
    const nl_gn_settings c = st.c();
    return solve([&](nl_solve_report* r, double* t, int cap) { return nl_pose2d_gn_solve(h_, &c, r, t, cap); },
                 trace, "nl_pose2d_gn_solve");
  }
  const nl_solve_report& lastReport() const { return rep_; }

 private:
  template <class F>
  TerminationReason solve(F f, std::vector<IterationRecord>* trace, const char* what) {
    const int cap = trace ? 4096 : 0;
    std::vector<double> t(size_t(cap > 0 ? cap : 1) * 8);
    check(f(&rep_, cap ? t.data() : nullptr, cap), what);
    if (trace) {
      trace->clear();
      for (int i = 0; i < rep_.n_trace; i++) {
        const double* r = t.data() + size_t(i) * 8;
        trace->push_back(IterationRecord{int(r[0]), int(r[1]), r[2], r[3], r[4], r[5], r[6] != 0.0, r[7] != 0.0});
      }
    }
    return TerminationReason(rep_.reason);
  }
  nl_pose2d* h_ = nullptr;
  int nv_, nf_;
  nl_solve_report rep_{};
};


// ---------------------------------------------------------------------------
// DeviceEdgeSection: a DoubleSection with user-defined edges (the reference's
// DoubleSection subclass with EdgeBinary / EdgeUnary edges, nelson/
// DoubleSection.hpp:338-365), resident on one GPU.  Derive from it, keep the
// parameters on the device and implement:
//   evaluate(stream, jacobians, r, J): every edge's whitened residual into r
//     and, with jacobians, its Jacobian blocks into J (device arrays; edge e
//     at rOffsets()[e] / jOffsets()[e]: J_a (m x dim_a, row-major) then J_b);
//   oplus(stream, incU, incV): apply the increment (device, user order);
//   backupSolution / rollbackSolution(stream): keep / restore the parameters.
// Device work goes on `stream` (a cudaStream_t) or is finished on return; a
// non-zero return ends the solve with NL_ERR_CALLBACK.  Call order: addEdge
// ..., optionally permuteAMD_SchurU, structureReady, then solveLM / solveGN.
class DeviceEdgeSection {
 public:
  DeviceEdgeSection(int bu, int numU, int numV, int precision = NL_PREC_FP64, int device = 0)
      : bu_(bu), nu_(numU), nv_(numV) {
    check(nl_section_create(bu, numU, numV, precision, device, &h_), "nl_section_create");
  }
  virtual ~DeviceEdgeSection() {
    if (h_) nl_section_destroy(h_);
  }
  DeviceEdgeSection(const DeviceEdgeSection&) = delete;
  DeviceEdgeSection& operator=(const DeviceEdgeSection&) = delete;

  // kind NL_EDGE_UV (a: U block, b: V block), NL_EDGE_UU (two U blocks),
  // NL_EDGE_U / NL_EDGE_V (unary on block a); m residuals
  void addEdge(int kind, int a, int b, int m) {
    check(nl_section_add_edges(h_, 1, &kind, &a, &b, &m), "nl_section_add_edges");
    ++ne_;
  }
  void permuteAMD_SchurU() { check(nl_section_permute_amd_u(h_), "nl_section_permute_amd_u"); }
  void structureReady() {
    check(nl_section_structure_ready(h_), "nl_section_structure_ready");
    rOff_.resize(ne_ + 1);
    jOff_.resize(ne_ + 1);
    check(nl_section_layout(h_, rOff_.data(), jOff_.data()), "nl_section_layout");
    nl_section_callbacks cb{this, &DeviceEdgeSection::evalT, &DeviceEdgeSection::oplusT,
                            &DeviceEdgeSection::backupT, &DeviceEdgeSection::rollbackT};
    check(nl_section_set_callbacks(h_, &cb), "nl_section_set_callbacks");
  }
  const std::vector<long long>& rOffsets() const { return rOff_; }
  const std::vector<long long>& jOffsets() const { return jOff_; }
  int numEdges() const { return ne_; }
  void setSolverKind(int kind) { check(nl_section_set_solver_kind(h_, kind), "nl_section_set_solver_kind"); }
  double update(bool hessian) {
    double c = 0.0;
    check(nl_section_update(h_, hessian ? 1 : 0, &c), "nl_section_update");
    return c;
  }
  TerminationReason solveLM(const LevenbergMarquardtSettings& st = {}, std::vector<IterationRecord>* trace = nullptr) {
    const nl_lm_settings c = st.c();
    return run([&](nl_solve_report* r, double* t, int cap) { return nl_section_lm_solve(h_, &c, r, t, cap); }, trace,
               "nl_section_lm_solve");
  }
  TerminationReason solveGN(const GaussNewtonSettings& st = {}, std::vector<IterationRecord>* trace = nullptr) {
    const nl_gn_settings c = st.c();
    return run([&](nl_solve_report* r, double* t, int cap) { return nl_section_gn_solve(h_, &c, r, t, cap); }, trace,
               "nl_section_gn_solve");
  }
  const nl_solve_report& lastReport() const { return rep_; }

 protected:
  virtual int evaluate(void* stream, bool jacobians, double* r, double* J) = 0;
  virtual int oplus(void* stream, const double* incU, const double* incV) = 0;
  virtual int backupSolution(void*) { return 1; }
  virtual int rollbackSolution(void*) { return 1; }
  int bu_, nu_, nv_;

 private:
  static int evalT(void* u, void* st, int jac, double* r, double* J) {
    try {
      return static_cast<DeviceEdgeSection*>(u)->evaluate(st, jac != 0, r, J);
    } catch (...) {
      return 1;
    }
  }
  static int oplusT(void* u, void* st, const double* du, const double* dv) {
    try {
      return static_cast<DeviceEdgeSection*>(u)->oplus(st, du, dv);
    } catch (...) {
      return 1;
    }
  }
  static int backupT(void* u, void* st) {
    try {
      return static_cast<DeviceEdgeSection*>(u)->backupSolution(st);
    } catch (...) {
      return 1;
    }
  }
  static int rollbackT(void* u, void* st) {
    try {
      return static_cast<DeviceEdgeSection*>(u)->rollbackSolution(st);
    } catch (...) {
      return 1;
    }
  }
  template <class F>
  TerminationReason run(F f, std::vector<IterationRecord>* trace, const char* what) {
    const int cap = trace ? 4096 : 0;
    std::vector<double> t(size_t(cap > 0 ? cap : 1) * 8);
    check(f(&rep_, cap ? t.data() : nullptr, cap), what);
    if (trace) {
      trace->clear();
      for (int i = 0; i < rep_.n_trace; i++) {
        const double* r = t.data() + size_t(i) * 8;
        trace->push_back(IterationRecord{int(r[0]), int(r[1]), r[2], r[3], r[4], r[5], r[6] != 0.0, r[7] != 0.0});
      }
    }
    return TerminationReason(rep_.reason);
  }
  nl_section* h_ = nullptr;
  int ne_ = 0;
  std::vector<long long> rOff_, jOff_;
  nl_solve_report rep_{};
};


// ---------------------------------------------------------------------------
// Problem files.
// Problem / load: the visibility-list format of the reference's samples
// (nelson/samples/Problems.h:4-12, Problems.cpp:8-30): "nCameras nPoints
// nEdges" then nEdges (camera, point) pairs.  Returns false when the file
// cannot be read, is truncated or holds an index out of range.
struct Problem {
  int nCameras = 0;
  int nPoints = 0;
  std::vector<std::pair<int, int>> edges;

  bool load(const std::string& file) {
    std::ifstream f(file);
    if (!f.good()) return false;
    int ne = 0;
    if (!(f >> nCameras >> nPoints >> ne) || nCameras < 0 || nPoints < 0 || ne < 0) return false;
    edges.resize(ne);
    for (auto& e : edges) {
      if (!(f >> e.first >> e.second)) return false;
      if (e.first < 0 || e.first >= nCameras || e.second < 0 || e.second >= nPoints) return false;
    }
    return true;
  }
};

// A BAL-style file: "num_cameras num_points num_observations", one
// "camera point x y" line per observation, 9 parameters per camera (axis-angle,
// t, f, k1, k2) and 3 per point.  Its pixels are -f d (P.x, P.y) / P.z about the
// image centre; addToSection builds the equivalent BASection (9-parameter
// cameras, principal point (0, 0), observations negated).
struct BALData {
  int nCameras = 0, nPoints = 0;
  std::vector<int> cam, pt;
  std::vector<double> obs;            // as in the file, 2 per observation
  std::vector<double> cams, pts;      // 9 per camera, 3 per point

  bool load(const std::string& file) {
    std::ifstream f(file);
    if (!f.good()) return false;
    int ne = 0;
    if (!(f >> nCameras >> nPoints >> ne) || nCameras < 0 || nPoints < 0 || ne < 0) return false;
    cam.resize(ne);
    pt.resize(ne);
    obs.resize(2 * (size_t)ne);
    for (int e = 0; e < ne; e++) {
      if (!(f >> cam[e] >> pt[e] >> obs[2 * e] >> obs[2 * e + 1])) return false;
      if (cam[e] < 0 || cam[e] >= nCameras || pt[e] < 0 || pt[e] >= nPoints) return false;
    }
    cams.resize(9 * (size_t)nCameras);
    pts.resize(3 * (size_t)nPoints);
    for (auto& v : cams)
      if (!(f >> v)) return false;
    for (auto& v : pts)
      if (!(f >> v)) return false;
    return true;
  }

  BASection toSection(int precision = NL_PREC_MIXED, int device = 0) const {
    BASection ba(9, nCameras, nPoints, 0, 0, precision, 1.0, 0.0, 0.0, device);
    ba.setParameters(cams, pts);
    ba.parametersReady();
    for (size_t e = 0; e < cam.size(); e++)
      ba.addEdge(NodeId(cam[e]), NodeId(pt[e]), -obs[2 * e], -obs[2 * e + 1]);
    ba.structureReady();
    return ba;
  }
};

}  // namespace nelson_b200

#endif

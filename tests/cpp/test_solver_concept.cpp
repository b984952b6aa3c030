// The reference's Solver and problem concepts through the C++ header.
//
// nelson_b200::LevenbergMarquardt<Solver>::solve(op) and
// GaussNewton<Solver>::solve(op) make exactly the calls of
// nelson/LevenbergMarquardt.hpp:36-146 and nelson/GaussNewton.hpp:32-127:
//   op.update(bool), op.hessian().H() / b() / chi2() / maxAbsValBVect(),
//   op.backupSolution(), op.rollbackSolution(), op.oplus(inc),
//   op.computeRhoChi2Change(mu, inc, oldChi2),
//   solver.init(H, b), solver.maxAbsHDiag(), solver.computeIncrement(H, b, rel, abs),
//   solver.incrementVector(), solver.incrementVectorSquaredNorm(), Solver::Type.
// This program drives them with
//   1. a problem assembled on the host (the reference's 5 x 2D / 3 x 3D
//      identity-Jacobian fixture, nelson/tests/testDoubleSectionSchurCommon.h:
//      24-413, with unary, UU and UV edges) over the stand-in block types
//      HostBlockHessian / HostBlockVectors and SolverCholeskySchurCudaHost:
//      chi2 is 0 at the ground truth and LM / GN bring it below 1e-12 from
//      uniform noise of 0.5 (nelson/tests/testDoubleSectionCommon.hpp:58-130);
//   2. a BASection read from a BAL-style file (argv[1]) with
//      SolverCholeskySchurCuda: the per-sub-iteration records go to stdout as
//      "TRACE prec it subit chi2 mu rho" lines, which the Python harness
//      compares with the FP64 oracle's trace on the same file.
// Prints "ALL OK" when every check passed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "nelson_b200/nelson.hpp"

using nelson_b200::HostBlockHessian;
using nelson_b200::HostBlockVectors;

namespace {

int failures = 0;
void expect(bool ok, const std::string& what, double a, double b) {
  std::printf("%s %-58s %.6e %.6e\n", ok ? "ok  " : "FAIL", what.c_str(), a, b);
  if (!ok) failures++;
}

// ---------------------------------------------------------------------------
// The 5 x 2D / 3 x 3D fixture as a host problem with the reference's problem
// concept.  Edges (identity Jacobians): unary on every 2D point (r = x_i - z)
// and every 3D point (r = y_j - z), UU on every pair i < j
// (r = x_i - x_j - z), UV on every (i, j) (r = x_i - y_j.xy - z).
class Points2D3D {
 public:
  static constexpr int NU = 5, NV = 3;
  struct Edge {
    int type;  // 0 unary U, 1 unary V, 2 UU, 3 UV
    int i, j;
    double z[3];
  };

  explicit Points2D3D(unsigned seed) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> U(-1, 1);
    for (auto& v : xt_) v = U(g);
    for (auto& v : yt_) v = U(g);
    for (int i = 0; i < NU; i++) edges_.push_back({0, i, -1, {xt_[2 * i], xt_[2 * i + 1], 0}});
    for (int j = 0; j < NV; j++) edges_.push_back({1, j, -1, {yt_[3 * j], yt_[3 * j + 1], yt_[3 * j + 2]}});
    for (int i = 0; i < NU; i++)
      for (int k = i + 1; k < NU; k++)
        edges_.push_back({2, i, k, {xt_[2 * i] - xt_[2 * k], xt_[2 * i + 1] - xt_[2 * k + 1], 0}});
    for (int i = 0; i < NU; i++)
      for (int j = 0; j < NV; j++)
        edges_.push_back({3, i, j, {xt_[2 * i] - yt_[3 * j], xt_[2 * i + 1] - yt_[3 * j + 1], 0}});
    // structure in the reference's storage order (DoubleSection.hpp:157-191):
    // U upper CSC (column c: rows r <= c ascending), V diagonal, W CSR
    H_.bu = 2;
    H_.numU = NU;
    H_.numV = NV;
    for (int c = 0; c < NU; c++)
      for (int r = 0; r <= c; r++) {
        uid_u_[{r, c}] = int(H_.u_rc.size() / 2);
        H_.u_rc.push_back(r);
        H_.u_rc.push_back(c);
      }
    for (int j = 0; j < NV; j++) {
      H_.v_rc.push_back(j);
      H_.v_rc.push_back(j);
    }
    for (int i = 0; i < NU; i++)
      for (int j = 0; j < NV; j++) {
        uid_w_[{i, j}] = int(H_.w_rc.size() / 2);
        H_.w_rc.push_back(i);
        H_.w_rc.push_back(j);
      }
    H_.U.assign(H_.u_rc.size() / 2 * 4, 0.0);
    H_.V.assign(NV * 9, 0.0);
    H_.W.assign(H_.w_rc.size() / 2 * 6, 0.0);
    b_.bU.assign(NU * 2, 0.0);
    b_.bV.assign(NV * 3, 0.0);
    x_ = xt_;
    y_ = yt_;
  }
  // Points2d3dBase::addNoise (testDoubleSectionSchurCommon.h:347-354)
  void addNoise(double sigma, unsigned seed) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> U(-sigma, sigma);
    for (auto& v : x_) v += U(g);
    for (auto& v : y_) v += U(g);
  }

  // ---- the problem concept ----
  struct Hessian {
    HostBlockHessian* Hm;
    HostBlockVectors* bv;
    double* c2;
    double* mb;
    HostBlockHessian& H() { return *Hm; }
    const HostBlockVectors& b() const { return *bv; }
    double chi2() const { return *c2; }
    double maxAbsValBVect() const { return *mb; }
  };
  Hessian& hessian() { return view_; }

  void update(bool hessian) {
    chi2_ = 0;
    if (hessian) {
      H_.setZero();
      b_.setZero();
    }
    for (const Edge& e : edges_) {
      double r[3] = {0, 0, 0};
      const int dr = e.type == 1 ? 3 : 2;
      for (int k = 0; k < dr; k++) {
        double v = 0;
        if (e.type == 0) v = x_[2 * e.i + k];
        if (e.type == 1) v = y_[3 * e.i + k];
        if (e.type == 2) v = x_[2 * e.i + k] - x_[2 * e.j + k];
        if (e.type == 3) v = x_[2 * e.i + k] - y_[3 * e.j + k];
        r[k] = v - e.z[k];
        chi2_ += r[k] * r[k];
      }
      if (!hessian) continue;
      // H += J'J, b += J'r with J = identity / -identity / selection blocks
      if (e.type == 0 || e.type == 2 || e.type == 3) {
        double* Ui = &H_.U[size_t(uid_u_[{e.i, e.i}]) * 4];
        Ui[0] += 1;
        Ui[3] += 1;
        b_.bU[2 * e.i] += r[0];
        b_.bU[2 * e.i + 1] += r[1];
      }
      if (e.type == 2) {
        double* Uj = &H_.U[size_t(uid_u_[{e.j, e.j}]) * 4];
        Uj[0] += 1;
        Uj[3] += 1;
        double* Uij = &H_.U[size_t(uid_u_[{e.i, e.j}]) * 4];
        Uij[0] -= 1;
        Uij[3] -= 1;
        b_.bU[2 * e.j] -= r[0];
        b_.bU[2 * e.j + 1] -= r[1];
      }
      if (e.type == 1 || e.type == 3) {
        const int j = e.type == 1 ? e.i : e.j;
        double* Vj = &H_.V[size_t(j) * 9];
        const double sgn = e.type == 1 ? 1.0 : -1.0;
        for (int k = 0; k < dr; k++) {
          Vj[k * 3 + k] += 1;
          b_.bV[3 * j + k] += sgn * r[k];
        }
      }
      if (e.type == 3) {
        double* Wij = &H_.W[size_t(uid_w_[{e.i, e.j}]) * 6];  // 2 x 3, J_x' J_y = -[I2 0]
        Wij[0] -= 1;
        Wij[4] -= 1;
      }
    }
    maxb_ = 0;
    for (double v : b_.bU) maxb_ = std::max(maxb_, std::fabs(v));
    for (double v : b_.bV) maxb_ = std::max(maxb_, std::fabs(v));
  }
  void oplus(const HostBlockVectors& inc) {
    for (size_t k = 0; k < x_.size(); k++) x_[k] += inc.bU[k];
    for (size_t k = 0; k < y_.size(); k++) y_[k] += inc.bV[k];
  }
  void backupSolution() {
    xb_ = x_;
    yb_ = y_;
  }
  void rollbackSolution() {
    x_ = xb_;
    y_ = yb_;
  }
  // DoubleSection::computeRhoChi2Change (nelson/DoubleSection.h:300-311)
  double computeRhoChi2Change(double mu, const HostBlockVectors& inc, double oldChi2) const {
    double den = 0;
    for (size_t k = 0; k < inc.bU.size(); k++) den += inc.bU[k] * (mu * inc.bU[k] - b_.bU[k]);
    for (size_t k = 0; k < inc.bV.size(); k++) den += inc.bV[k] * (mu * inc.bV[k] - b_.bV[k]);
    return (oldChi2 - chi2_) / den;
  }

 private:
  std::vector<double> xt_ = std::vector<double>(2 * NU), yt_ = std::vector<double>(3 * NV);
  std::vector<double> x_, y_, xb_, yb_;
  std::vector<Edge> edges_;
  std::map<std::pair<int, int>, int> uid_u_, uid_w_;
  HostBlockHessian H_;
  HostBlockVectors b_;
  double chi2_ = 0, maxb_ = 0;
  Hessian view_{&H_, &b_, &chi2_, &maxb_};
};

using HostSolver = nelson_b200::SolverCholeskySchurCudaHost<HostBlockHessian, HostBlockVectors>;

void fixture_checks(int prec) {
  const char* pn = prec == NL_PREC_FP64 ? "fp64" : "mixed";
  {
    Points2D3D p(11);
    p.update(true);
    expect(p.hessian().chi2() == 0.0, std::string(pn) + " fixture chi2 at ground truth", p.hessian().chi2(), 0);
  }
  for (int algo = 0; algo < 2; algo++) {
    Points2D3D p(11);
    p.addNoise(0.5, 5);
    p.update(true);
    const double c0 = p.hessian().chi2();
    double c1 = -1;
    if (algo == 0) {
      nelson_b200::LevenbergMarquardt<HostSolver> lm;
      lm.solver().settings().precision = prec;
      const auto r = lm.solve(p);
      (void)r;
      c1 = p.hessian().chi2();
      expect(c1 < 1e-12, std::string(pn) + " fixture LM final chi2 < 1e-12", c0, c1);
    } else {
      nelson_b200::GaussNewton<HostSolver> gn;
      gn.solver().settings().precision = prec;
      gn.settings().maxNumIt = 10;
      gn.solve(p);
      c1 = p.hessian().chi2();
      expect(c1 < 1e-12, std::string(pn) + " fixture GN final chi2 < 1e-12", c0, c1);
    }
  }
}

void ba_trace(const char* bal, int prec, int its) {
  nelson_b200::BALData d;
  if (!d.load(bal)) {
    expect(false, "BAL file readable", 0, 0);
    return;
  }
  nelson_b200::BASection ba = d.toSection(prec, 0);
  nelson_b200::LevenbergMarquardt<nelson_b200::SolverCholeskySchurCuda> lm;
  lm.settings().maxNumIt = its;
  const auto r = lm.solve(ba);
  for (const auto& s : lm.stats())
    std::printf("TRACE %d %d %d %.17g %.17g %.17g\n", prec, s.it, s.subit, s.chi2, s.mu, s.rho);
  std::printf("REASON %d %d\n", prec, int(r));
  // the same section, the device loop: the same trace
  nelson_b200::BASection bb = d.toSection(prec, 0);
  nelson_b200::LevenbergMarquardt<nelson_b200::SolverCholeskySchurCuda> lm2;
  lm2.settings().maxNumIt = its;
  const auto r2 = lm2.solveOnDevice(bb);
  double worst = 0;
  const size_t n = std::min(lm.stats().size(), lm2.stats().size());
  for (size_t k = 0; k < n; k++)
    if (lm.stats()[k].chi2 > 0 && lm2.stats()[k].chi2 > 0)
      worst = std::max(worst, std::fabs(lm.stats()[k].chi2 - lm2.stats()[k].chi2) / lm.stats()[k].chi2);
  expect(r == r2 && lm.stats().size() == lm2.stats().size(), std::string(prec ? "mixed" : "fp64") +
         " BA concept loop: reason / records == device loop", double(lm.stats().size()), double(lm2.stats().size()));
  expect(worst <= (prec == NL_PREC_FP64 ? 1e-9 : 1e-6), std::string(prec ? "mixed" : "fp64") +
         " BA concept loop: cost trace vs device loop (rel)", worst, 0);
}

}  // namespace

int main(int argc, char** argv) {
  try {
    for (int prec : {NL_PREC_FP64, NL_PREC_MIXED}) fixture_checks(prec);
    if (argc > 1)
      for (int prec : {NL_PREC_FP64, NL_PREC_MIXED}) ba_trace(argv[1], prec, argc > 2 ? std::atoi(argv[2]) : 8);
  } catch (const nelson_b200::Error& e) {
    std::printf("FAIL exception: %s\n", e.what());
    return 2;
  }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}

// C++ API test: drives nelson_b200::BASection through the header-only
// LevenbergMarquardt / GaussNewton classes (include/nelson_b200/nelson.hpp).
//
// Checks, on a small seeded scene (cameras in a plane looking along +z at a
// slab of points, all points seen by all cameras, pixel noise):
//   1. LevenbergMarquardt::solve (host loop, one C-ABI call per step) and
//      solveOnDevice (nl_lm_solve) give the same per-iteration cost trace;
//   2. the same for GaussNewton (damped by absLambda);
//   3. a fixed camera and a fixed point do not move;
//   4. the cost decreases at least tenfold.
// Prints one line per check and exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "nelson_b200/nelson.hpp"

using nelson_b200::BASection;
using nelson_b200::NodeId;

namespace {

struct Scene {
  int nc = 8, np = 300, ncFix = 1, npFix = 2;
  std::vector<double> cams, pts;  // true values, variable then fixed
  std::vector<int> cam, camFixed, pt, ptFixed;
  std::vector<double> obs;
};

void rodrigues(const double w[3], double R[9]) {
  const double th = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  const double k[3] = {th > 0 ? w[0] / th : 1, th > 0 ? w[1] / th : 0, th > 0 ? w[2] / th : 0};
  const double c = std::cos(th), s = std::sin(th), v = 1 - c;
  R[0] = c + k[0] * k[0] * v;        R[1] = k[0] * k[1] * v - k[2] * s; R[2] = k[0] * k[2] * v + k[1] * s;
  R[3] = k[1] * k[0] * v + k[2] * s; R[4] = c + k[1] * k[1] * v;        R[5] = k[1] * k[2] * v - k[0] * s;
  R[6] = k[2] * k[0] * v - k[1] * s; R[7] = k[2] * k[1] * v + k[0] * s; R[8] = c + k[2] * k[2] * v;
}

void project(const double* cam, const double* X, double cx, double cy, double out[2]) {
  double R[9];
  rodrigues(cam, R);
  double P[3];
  for (int i = 0; i < 3; i++) P[i] = R[3 * i] * X[0] + R[3 * i + 1] * X[1] + R[3 * i + 2] * X[2] + cam[3 + i];
  const double x = P[0] / P[2], y = P[1] / P[2], r2 = x * x + y * y;
  const double d = 1 + cam[7] * r2 + cam[8] * r2 * r2;
  out[0] = cam[6] * d * x + cx;
  out[1] = cam[6] * d * y + cy;
}

Scene make_scene(unsigned seed) {
  Scene s;
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> U(-1, 1);
  const int nct = s.nc + s.ncFix, npt = s.np + s.npFix;
  for (int c = 0; c < nct; c++) {
    const double p[9] = {0.05 * U(g), 0.05 * U(g), 0.05 * U(g), 0.8 * U(g), 0.8 * U(g), 0.1 * U(g),
                         500 + 20 * U(g), 0.01 * U(g), 0.0};
    s.cams.insert(s.cams.end(), p, p + 9);
  }
  for (int q = 0; q < npt; q++) {
    const double X[3] = {2 * U(g), 2 * U(g), 6 + 2 * U(g)};
    s.pts.insert(s.pts.end(), X, X + 3);
  }
  std::normal_distribution<double> N(0, 0.5);
  for (int c = 0; c < nct; c++)
    for (int q = 0; q < npt; q++) {
      double uv[2];
      project(&s.cams[9 * c], &s.pts[3 * q], 320, 240, uv);
      const bool cf = c >= s.nc, pf = q >= s.np;
      s.cam.push_back(cf ? c - s.nc : c);
      s.camFixed.push_back(cf);
      s.pt.push_back(pf ? q - s.np : q);
      s.ptFixed.push_back(pf);
      s.obs.push_back(uv[0] + N(g));
      s.obs.push_back(uv[1] + N(g));
    }
  return s;
}

BASection make_section(const Scene& s, int precision, unsigned seed, int order = 0) {  // order: 0 user, 1 RCM, 2 AMD
  BASection ba(9, s.nc, s.np, s.ncFix, s.npFix, precision, 500.0, 320.0, 240.0, 0);
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> U(-1, 1);
  std::vector<double> cams = s.cams, pts = s.pts;
  for (int c = 0; c < s.nc; c++) {  // perturb the variable blocks only
    for (int k = 0; k < 3; k++) cams[9 * c + k] += 0.01 * U(g);
    for (int k = 3; k < 6; k++) cams[9 * c + k] += 0.05 * U(g);
    cams[9 * c + 6] += 5 * U(g);
  }
  for (int q = 0; q < s.np; q++)
    for (int k = 0; k < 3; k++) pts[3 * q + k] += 0.05 * U(g);
  ba.setParameters(cams, pts);
  ba.parametersReady();
  for (size_t e = 0; e < s.cam.size(); e++)
    ba.addEdge(NodeId(s.cam[e], s.camFixed[e] ? nelson_b200::NodeType::Fixed : nelson_b200::NodeType::Variable),
               NodeId(s.pt[e], s.ptFixed[e] ? nelson_b200::NodeType::Fixed : nelson_b200::NodeType::Variable),
               s.obs[2 * e], s.obs[2 * e + 1]);
  if (order == 1) ba.permuteRCM_SchurU();
  if (order == 2) ba.permuteAMD_SchurU();
  ba.structureReady();
  return ba;
}

int failures = 0;
void expect(bool ok, const char* what, double a, double b) {
  std::printf("%s %-48s %.6e %.6e\n", ok ? "ok  " : "FAIL", what, a, b);
  if (!ok) failures++;
}

template <class Stats>
double trace_diff(const Stats& a, const Stats& b, size_t* n) {
  *n = std::min(a.size(), b.size());
  double worst = 0;
  for (size_t k = 0; k < *n; k++) {
    if (a[k].chi2 < 0 || b[k].chi2 < 0) continue;
    worst = std::max(worst, std::fabs(a[k].chi2 - b[k].chi2) / a[k].chi2);
  }
  return worst;
}

// The 2D scan alignment of nelson/tests/testGaussNewton2DScansAlign.cpp:
// scans of common world points and normals seen from random SE(2) poses;
// pose 0 fixed, the others started from a perturbed truth.
struct Scans {
  int n = 0, k = 0;
  std::vector<double> truth;                   // (n + 1) x 3
  std::vector<std::vector<double>> pts, nrm;   // per scan, k x 2
};

Scans make_scans(int n, int k, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  Scans sc;
  sc.n = n;
  sc.k = k;
  std::vector<double> wp(2 * k), wn(2 * k);
  for (int i = 0; i < k; i++) {
    wp[2 * i] = 100 * u(rng);
    wp[2 * i + 1] = 100 * u(rng);
    const double a = 3.14159265358979 * u(rng);
    wn[2 * i] = std::cos(a);
    wn[2 * i + 1] = std::sin(a);
  }
  for (int p = 0; p <= n; p++) {
    const double x = 10 * u(rng), y = 10 * u(rng), th = 3.14159265358979 * u(rng);
    sc.truth.insert(sc.truth.end(), {x, y, th});
    const double c = std::cos(th), s_ = std::sin(th);
    std::vector<double> q(2 * k), m(2 * k);
    for (int i = 0; i < k; i++) {  // R' (X - t), R' n
      const double dx = wp[2 * i] - x, dy = wp[2 * i + 1] - y;
      q[2 * i] = c * dx + s_ * dy;
      q[2 * i + 1] = -s_ * dx + c * dy;
      m[2 * i] = c * wn[2 * i] + s_ * wn[2 * i + 1];
      m[2 * i + 1] = -s_ * wn[2 * i] + c * wn[2 * i + 1];
    }
    sc.pts.push_back(q);
    sc.nrm.push_back(m);
  }
  return sc;
}

}  // namespace

int main() {
  const Scene s = make_scene(7);
  try {
    for (int prec : {NL_PREC_FP64, NL_PREC_MIXED}) {
      const double tol = prec == NL_PREC_FP64 ? 1e-9 : 1e-6;
      std::printf("precision %s\n", prec == NL_PREC_FP64 ? "fp64" : "mixed");
      // 1. LM host loop vs device loop
      BASection a = make_section(s, prec, 11), b = make_section(s, prec, 11);
      nelson_b200::LevenbergMarquardt<> lmA, lmB;
      lmA.settings().maxNumIt = 10;
      lmB.settings().maxNumIt = 10;
      const auto rA = lmA.solve(a);
      const auto rB = lmB.solveOnDevice(b);
      size_t n;
      const double d = trace_diff(lmA.stats(), lmB.stats(), &n);
      expect(rA == rB, "LM termination reason host == device", double(rA), double(rB));
      expect(lmA.stats().size() == lmB.stats().size(), "LM sub-iteration count host == device",
             double(lmA.stats().size()), double(lmB.stats().size()));
      expect(d <= tol, "LM per-iteration cost host vs device (rel)", d, tol);
      const double c0 = lmA.stats().front().chi2, c1 = a.hessian().chi2();
      expect(c1 < 0.1 * c0, "LM cost reduced 10x", c0, c1);

      // 3. fixed nodes do not move
      std::vector<double> cams, pts;
      a.getParameters(cams, pts);
      double moved = 0;
      for (int k = 0; k < 9 * s.ncFix; k++) moved = std::max(moved, std::fabs(cams[9 * s.nc + k] - s.cams[9 * s.nc + k]));
      for (int k = 0; k < 3 * s.npFix; k++) moved = std::max(moved, std::fabs(pts[3 * s.np + k] - s.pts[3 * s.np + k]));
      expect(moved <= 1e-12, "fixed camera / points unchanged", moved, 1e-12);

      // 2. GN host loop vs device loop
      BASection g1 = make_section(s, prec, 13), g2 = make_section(s, prec, 13);
      nelson_b200::GaussNewton<> gnA, gnB;
      gnA.settings().maxNumIt = 5;
      gnA.settings().absLambda = 1e-3;
      gnB.settings() = gnA.settings();
      const auto gA = gnA.solve(g1);
      const auto gB = gnB.solveOnDevice(g2);
      const double dg = trace_diff(gnA.stats(), gnB.stats(), &n);
      expect(gA == gB, "GN termination reason host == device", double(gA), double(gB));
      expect(dg <= tol, "GN per-iteration cost host vs device (rel)", dg, tol);

      // 4. the envelope solver (SolverEnvelopeSchurCuda) gives the dense solver's trace
      BASection e1 = make_section(s, prec, 11), e2 = make_section(s, prec, 11);
      nelson_b200::LevenbergMarquardt<> lmD;
      nelson_b200::LevenbergMarquardt<nelson_b200::SolverEnvelopeSchurCuda> lmE;
      lmD.settings().maxNumIt = 10;
      lmE.settings().maxNumIt = 10;
      const auto rD = lmD.solveOnDevice(e1);
      const auto rE = lmE.solveOnDevice(e2);
      const double de = trace_diff(lmD.stats(), lmE.stats(), &n);
      expect(rD == rE, "envelope solver termination reason == dense", double(rD), double(rE));
      expect(de <= 1e-12, "envelope solver per-iteration cost vs dense (rel)", de, 1e-12);

      // 5. the reverse Cuthill-McKee camera order (permuteRCM_SchurU): the same
      //    trace up to rounding (another elimination order)
      BASection r1 = make_section(s, prec, 11, 1);
      nelson_b200::LevenbergMarquardt<nelson_b200::SolverEnvelopeSchurCuda> lmR;
      lmR.settings().maxNumIt = 10;
      const auto rR = lmR.solveOnDevice(r1);
      const double dr = trace_diff(lmD.stats(), lmR.stats(), &n);
      (void)rR;
      expect(dr <= tol, "RCM order per-iteration cost vs user order (rel)", dr, tol);

      // 6. the approximate minimum degree order (permuteAMD_SchurU): the same
      //    trace up to rounding
      BASection am = make_section(s, prec, 11, 2);
      nelson_b200::LevenbergMarquardt<nelson_b200::SolverCholeskySchurCuda> lmAmd;
      lmAmd.settings().maxNumIt = 10;
      const auto rAmd = lmAmd.solveOnDevice(am);
      const double da = trace_diff(lmD.stats(), lmAmd.stats(), &n);
      (void)rAmd;
      expect(da <= tol, "AMD order per-iteration cost vs user order (rel)", da, tol);
    }
    // 7. ScanAlignSection (SingleSection with point-to-line edges): LM and GN
    //    reach the reference test's criterion chi2 < 1e-12, natural and AMD order
    const Scans sc = make_scans(8, 500, 3);
    for (int order = 0; order < 2; order++)
      for (int solver = 0; solver < 2; solver++) {
        nelson_b200::ScanAlignSection sa(sc.n, 1, NL_PREC_FP64);
        std::vector<double> start(sc.truth.begin() + 3, sc.truth.end());
        for (int p = 0; p < sc.n; p++) {
          start[3 * p] += 0.01 * ((p % 3) - 1);
          start[3 * p + 1] -= 0.01 * ((p % 2) ? 1 : -1);
          start[3 * p + 2] += 0.003 * ((p % 5) - 2);
        }
        sa.setPoses(start.data(), sc.truth.data());
        for (int i = 0; i <= sc.n; i++)
          for (int j = i + 1; j <= sc.n; j++) {
            const NodeId a = i == 0 ? NodeId::fixed(0) : NodeId(i - 1);
            sa.addEdge(a, NodeId(j - 1), sc.k, sc.pts[i].data(), sc.nrm[i].data(), sc.pts[j].data());
          }
        if (order == 1) sa.permuteAMD();
        sa.structureReady();
        const double c0 = sa.update(true);
        std::vector<nelson_b200::IterationRecord> tr;
        const auto reason = solver == 0 ? sa.solveLM({}, &tr) : sa.solveGN({}, &tr);
        const double c1 = sa.update(true);
        const std::vector<double> p = sa.poses();
        double err = 0;
        for (int q = 0; q < 3 * sc.n; q++) err = std::max(err, std::fabs(p[q] - sc.truth[3 + q]));
        std::printf("scan align %s %s: reason %d, %zu records\n", order ? "amd" : "natural",
                    solver ? "GN" : "LM", int(reason), tr.size());
        expect(c1 < 1e-12 && c0 > 1.0, "scan alignment chi2 below 1e-12 after the solve", c0, c1);
        expect(err < 1e-6, "scan alignment poses equal the truth", err, 1e-6);
      }
  } catch (const nelson_b200::Error& e) {
    std::printf("FAIL exception: %s\n", e.what());
    return 2;
  }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}

// nelson_oracle.cpp -- FP64 CPU oracle for the Schur-complement LM/GN path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++17 + OpenMP with
// no Eigen and no `mat`, the algorithms of nelson's DoubleSection problem
// (structure + UID assignment + Hessian accumulation), SolverCholeskySchur and
// LevenbergMarquardt / GaussNewton.  It is the checker the CUDA library is
// compared against and the CPU baseline bench.py times; the nelson_b200
// product never links or calls it.
//
// Parity pinning: the reference ships no golden vectors.  The oracle is pinned
// against the reference's own known-answer tests (tests/test_oracle.py): the
// 5x2D/3x3D identity-Jacobian fixture of
// nelson/tests/testDoubleSectionSchurCommon.h:24-413 that GN and LM must
// drive to chi2 < 1e-12 (nelson/tests/testDoubleSectionCommon.hpp:58-130),
// the 3x5 W pattern and its expected S pattern
// (nelson/tests/testMatrixWWtMultiplier.cpp:36-59), the permutation sections
// (nelson/tests/testDoubleSectionSchurDiagBlockWWtFFFF.cpp:482-504), and the
// multiplier identities at 1e-12 (testMatrixWWtMultiplier.cpp:90-102,
// testMatrixWtXMultiplier.cpp:87-91, testMatrixVinv.cpp:58-62).
//
// The BA camera model (axis-angle pose, pinhole with optional focal + 2-term
// radial distortion) is this project's own; the reference's BA sample uses the
// absent `lie`/`camera` libraries (nelson/samples/BASchurPerfomances.cpp:195-232)
// so only its structure (a projection EdgeBinaryUV with analytic Jacobians,
// H11 += Jc'Jc, H22 += Jp'Jp, H12 += Jc'Jp) is restated.

#include "nelson_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kCamState = 16;  // R[9], t[3], f, k1, k2, pad

// ---------------------------------------------------------------------------
// SO(3) helpers (Rodrigues' formula and its inverse).
void so3_exp(const double* w, double* R) {
  const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double A, B;
  if (th2 < 1e-8) {
    A = 1.0 - th2 / 6.0 + th2 * th2 / 120.0;
    B = 0.5 - th2 / 24.0 + th2 * th2 / 720.0;
  } else {
    const double th = std::sqrt(th2);
    A = std::sin(th) / th;
    B = (1.0 - std::cos(th)) / th2;
  }
  const double K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
  double K2[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += K[i * 3 + k] * K[k * 3 + j];
      K2[i * 3 + j] = s;
    }
  for (int i = 0; i < 9; i++) R[i] = A * K[i] + B * K2[i];
  R[0] += 1.0;
  R[4] += 1.0;
  R[8] += 1.0;
}

void so3_log(const double* R, double* w) {
  const double tr = R[0] + R[4] + R[8];
  double c = 0.5 * (tr - 1.0);
  c = std::max(-1.0, std::min(1.0, c));
  const double th = std::acos(c);
  const double v[3] = {R[7] - R[5], R[2] - R[6], R[3] - R[1]};
  if (th < 1e-6) {
    for (int i = 0; i < 3; i++) w[i] = 0.5 * v[i];
    return;
  }
  if (M_PI - th < 1e-4) {
    // Near pi: axis from the diagonal of (R + I) / 2.
    int k = 0;
    if (R[4] > R[k * 4]) k = 1;
    if (R[8] > R[k * 4]) k = 2;
    double a[3];
    const double d = std::sqrt(std::max(0.0, 0.5 * (R[k * 4] + 1.0)));
    a[k] = d;
    for (int i = 0; i < 3; i++)
      if (i != k) a[i] = (0.5 * (R[i * 3 + k] + R[k * 3 + i]) * 0.5) / d;
    const double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double s = (v[0] * a[0] + v[1] * a[1] + v[2] * a[2]) < 0 ? -1.0 : 1.0;
    for (int i = 0; i < 3; i++) w[i] = s * th * a[i] / n;
    return;
  }
  const double f = th / (2.0 * std::sin(th));
  for (int i = 0; i < 3; i++) w[i] = f * v[i];
}

// ---------------------------------------------------------------------------
// BA projection edge: P = R X + t, (x, y) = P.xy / P.z,
// d = 1 + k1 r^2 + k2 r^4, pixel = f d (x, y) + (cx, cy).
// Camera tangent: [dw(3) (left SO3 increment), dt(3) [, df, dk1, dk2]].
// Residual r = pixel - z.  Jc is 2 x bc, Jp is 2 x 3 (row-major).
inline void ba_eval(const double* cam, const double* X, const double* z,
                    double f_fixed, double cx, double cy, int bc, bool jac,
                    double* r, double* Jc, double* Jp) {
  const double* R = cam;
  const double* t = cam + 9;
  const double a0 = R[0] * X[0] + R[1] * X[1] + R[2] * X[2];
  const double a1 = R[3] * X[0] + R[4] * X[1] + R[5] * X[2];
  const double a2 = R[6] * X[0] + R[7] * X[1] + R[8] * X[2];
  const double P0 = a0 + t[0], P1 = a1 + t[1], P2 = a2 + t[2];
  const double iz = 1.0 / P2;
  const double x = P0 * iz, y = P1 * iz;
  const double f = bc == 9 ? cam[12] : f_fixed;
  const double k1 = bc == 9 ? cam[13] : 0.0;
  const double k2 = bc == 9 ? cam[14] : 0.0;
  const double r2 = x * x + y * y;
  const double d = 1.0 + r2 * (k1 + k2 * r2);
  r[0] = f * d * x + cx - z[0];
  r[1] = f * d * y + cy - z[1];
  if (!jac) return;
  const double g = 2.0 * (k1 + 2.0 * k2 * r2);
  const double m00 = f * (d + g * x * x), m01 = f * g * x * y;
  const double m11 = f * (d + g * y * y);
  // M = d(pixel)/dP = [[m00, m01], [m01, m11]] * [[iz, 0, -x iz], [0, iz, -y iz]]
  double M[6];
  M[0] = m00 * iz;
  M[1] = m01 * iz;
  M[2] = -(m00 * x + m01 * y) * iz;
  M[3] = m01 * iz;
  M[4] = m11 * iz;
  M[5] = -(m01 * x + m11 * y) * iz;
  for (int i = 0; i < 2; i++) {
    const double* m = M + 3 * i;
    // Jp = M R
    for (int j = 0; j < 3; j++) Jp[i * 3 + j] = m[0] * R[j] + m[1] * R[3 + j] + m[2] * R[6 + j];
    // d P / d dw = -[a]x = [[0, a2, -a1], [-a2, 0, a0], [a1, -a0, 0]]
    double* jc = Jc + i * bc;
    jc[0] = -m[1] * a2 + m[2] * a1;
    jc[1] = m[0] * a2 - m[2] * a0;
    jc[2] = -m[0] * a1 + m[1] * a0;
    jc[3] = m[0];
    jc[4] = m[1];
    jc[5] = m[2];
  }
  if (bc == 9) {
    Jc[6] = d * x;
    Jc[7] = f * x * r2;
    Jc[8] = f * x * r2 * r2;
    Jc[9 + 6] = d * y;
    Jc[9 + 7] = f * y * r2;
    Jc[9 + 8] = f * y * r2 * r2;
  }
}

// ---------------------------------------------------------------------------
// Dense blocked Cholesky (lower, row-major).  Right-looking, 128-wide panels,
// OpenMP over panel rows and trailing tiles, 4x4 register-blocked dot
// products for the trailing update.
inline double dotn(const double* a, const double* b, int n) {
  double s = 0;
#pragma omp simd reduction(+ : s)
  for (int p = 0; p < n; p++) s += a[p] * b[p];
  return s;
}

void trailing_tile(double* A, int lda, int k0, int kb, int i0, int i1, int j0,
                   int j1) {
  // A[i][j] -= sum_p A[i][k0+p] A[j][k0+p] for i in [i0,i1), j in [j0,j1), j <= i
  int i = i0;
  for (; i + 4 <= i1; i += 4) {
    const double* a0 = A + (size_t)i * lda + k0;
    const double* a1 = a0 + lda;
    const double* a2 = a1 + lda;
    const double* a3 = a2 + lda;
    int jmax = std::min(j1, i + 4);
    int j = j0;
    for (; j + 4 <= jmax; j += 4) {
      const double* b0 = A + (size_t)j * lda + k0;
      const double* b1 = b0 + lda;
      const double* b2 = b1 + lda;
      const double* b3 = b2 + lda;
      double c00 = 0, c01 = 0, c02 = 0, c03 = 0, c10 = 0, c11 = 0, c12 = 0, c13 = 0;
      double c20 = 0, c21 = 0, c22 = 0, c23 = 0, c30 = 0, c31 = 0, c32 = 0, c33 = 0;
#pragma omp simd reduction(+ : c00, c01, c02, c03, c10, c11, c12, c13, c20, c21, c22, c23, c30, c31, c32, c33)
      for (int p = 0; p < kb; p++) {
        const double x0 = a0[p], x1 = a1[p], x2 = a2[p], x3 = a3[p];
        const double y0 = b0[p], y1 = b1[p], y2 = b2[p], y3 = b3[p];
        c00 += x0 * y0; c01 += x0 * y1; c02 += x0 * y2; c03 += x0 * y3;
        c10 += x1 * y0; c11 += x1 * y1; c12 += x1 * y2; c13 += x1 * y3;
        c20 += x2 * y0; c21 += x2 * y1; c22 += x2 * y2; c23 += x2 * y3;
        c30 += x3 * y0; c31 += x3 * y1; c32 += x3 * y2; c33 += x3 * y3;
      }
      const double c[4][4] = {{c00, c01, c02, c03}, {c10, c11, c12, c13},
                              {c20, c21, c22, c23}, {c30, c31, c32, c33}};
      for (int u = 0; u < 4; u++)
        for (int v = 0; v < 4; v++)
          if (j + v <= i + u) A[(size_t)(i + u) * lda + j + v] -= c[u][v];
    }
    for (; j < jmax; j++) {
      const double* b0 = A + (size_t)j * lda + k0;
      for (int u = 0; u < 4; u++)
        if (j <= i + u) A[(size_t)(i + u) * lda + j] -= dotn(A + (size_t)(i + u) * lda + k0, b0, kb);
    }
  }
  for (; i < i1; i++) {
    const double* a0 = A + (size_t)i * lda + k0;
    int jmax = std::min(j1, i + 1);
    for (int j = j0; j < jmax; j++) A[(size_t)i * lda + j] -= dotn(a0, A + (size_t)j * lda + k0, kb);
  }
}

bool chol_blocked(double* A, int n, int lda, int nthreads) {
  const int nb = 128;
  const int tile = 64;
  for (int k0 = 0; k0 < n; k0 += nb) {
    const int kb = std::min(nb, n - k0);
    // (1) diagonal block.
    for (int j = k0; j < k0 + kb; j++) {
      double* aj = A + (size_t)j * lda;
      double d = aj[j] - dotn(aj + k0, aj + k0, j - k0);
      if (!(d > 0.0) || !std::isfinite(d)) return false;
      d = std::sqrt(d);
      aj[j] = d;
      for (int i = j + 1; i < k0 + kb; i++) {
        double* ai = A + (size_t)i * lda;
        ai[j] = (ai[j] - dotn(ai + k0, aj + k0, j - k0)) / d;
      }
    }
    // (2) panel below the diagonal block: row-wise forward substitution.
    const int r0 = k0 + kb;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = r0; i < n; i++) {
      double* ai = A + (size_t)i * lda;
      for (int j = k0; j < k0 + kb; j++) {
        const double* aj = A + (size_t)j * lda;
        ai[j] = (ai[j] - dotn(ai + k0, aj + k0, j - k0)) / aj[j];
      }
    }
    // (3) trailing update of the lower triangle.
    const int nt = (n - r0 + tile - 1) / tile;
    const int npairs = nt * (nt + 1) / 2;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int q = 0; q < npairs; q++) {
      // decode q -> (I, J) with J <= I
      int I = (int)((std::sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
      while ((I + 1) * (I + 2) / 2 <= q) I++;
      while (I * (I + 1) / 2 > q) I--;
      const int J = q - I * (I + 1) / 2;
      const int i0 = r0 + I * tile, i1 = std::min(n, i0 + tile);
      const int j0 = r0 + J * tile, j1 = std::min(n, j0 + tile);
      trailing_tile(A, lda, k0, kb, i0, i1, j0, j1);
    }
  }
  return true;
}

// L y = b then L' x = y, in place, L lower row-major.
void chol_solve(const double* L, int n, int lda, double* x) {
  for (int i = 0; i < n; i++) {
    const double* li = L + (size_t)i * lda;
    double s = x[i];
    for (int j = 0; j < i; j++) s -= li[j] * x[j];
    x[i] = s / li[i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int j = i + 1; j < n; j++) s -= L[(size_t)j * lda + i] * x[j];
    x[i] = s / L[(size_t)i * lda + i];
  }
}

// Small SPD inverse by Cholesky (B <= 9).  Returns false on a non-positive pivot.
bool small_spd_inverse(const double* A, int B, double* Ainv) {
  double L[81];
  for (int i = 0; i < B; i++)
    for (int j = 0; j <= i; j++) {
      double s = A[i * B + j];
      for (int k = 0; k < j; k++) s -= L[i * B + k] * L[j * B + k];
      if (i == j) {
        if (!(s > 0.0) || !std::isfinite(s)) return false;
        L[i * B + i] = std::sqrt(s);
      } else {
        L[i * B + j] = s / L[j * B + j];
      }
    }
  for (int c = 0; c < B; c++) {
    double x[9];
    for (int i = 0; i < B; i++) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; k++) s -= L[i * B + k] * x[k];
      x[i] = s / L[i * B + i];
    }
    for (int i = B - 1; i >= 0; i--) {
      double s = x[i];
      for (int k = i + 1; k < B; k++) s -= L[k * B + i] * x[k];
      x[i] = s / L[i * B + i];
    }
    for (int i = 0; i < B; i++) Ainv[i * B + c] = x[i];
  }
  return true;
}


// ---------------------------------------------------------------------------
struct Edge {
  int type;  // ORC_EDGE_*; BA projection edges are ORC_EDGE_BINARY_UV
  int id1, id2;
  bool fixed1, fixed2;
  int dr;
  double z[3];
  double w;
};

struct Problem {
  int kind, bu, bv, nu_var, nu_fix, nv_var, nv_fix, nthreads;
  double f_fixed = 500.0, cx = 320.0, cy = 240.0;
  std::vector<double> u, v, u_bck, v_bck;  // parameter state
  std::vector<Edge> edges;
  int dr_max = 2;
  int s1 = 0, s2 = 0;                       // per-edge Jacobian strides
  std::vector<double> er, eJ1, eJ2, echi2;  // per-edge cache (the edge objects' members)
  std::vector<int> perm;                    // user -> internal camera index
  bool ready = false;

  // structure
  int nU = 0, nV = 0, nW = 0;
  std::vector<int> u_r, u_c, v_r, v_c, w_r, w_c;
  std::vector<char> u_tr;                           // transpose flag per U block
  std::vector<int> unit_ptr, unit_edge, unit_slot;  // computation units (U, V, W)
  std::vector<int> h11, h12, h22;
  std::vector<int> w_row_ptr;             // CSR rows (internal camera) of W uids
  std::vector<int> w_col_ptr, w_col_uid;  // CSC columns (point) -> W uids
  std::vector<int> v_diag_uid;            // per point -> V uid or -1
  std::vector<int> u_diag_uid;            // per internal camera -> U uid or -1

  // Hessian
  std::vector<double> U, V, W, bU, bV;
  double chi2 = 0;

  // solver
  int n = 0;
  std::vector<double> Vinv, xV0, S, bS, incU, incV;
};

// ---------------------------------------------------------------------------
// Structure (DoubleSection::parametersReady/addEdge/structureReady,
// nelson/DoubleSection.hpp:67-80, 338-365, 83-246).
struct Contrib {
  int64_t key;  // storage-order key of the target block inside its matrix
  int edge;
  int slot;     // 11, 12, 22
  int r, c;     // internal block coordinates
  int tr;       // transpose flag (U off-diagonal only)
};

int build_structure(Problem& P) {
  const int ne = (int)P.edges.size();
  std::vector<Contrib> cu, cv, cw;
  cu.reserve(ne);
  cv.reserve(ne);
  cw.reserve(ne);
  const int64_t NU = std::max(1, P.nu_var), NV = std::max(1, P.nv_var);
  // U setters live at _edgeSetterComputerU[uj][ui] (user ids, ui <= uj) and
  // are re-keyed to (min, max) of the permuted indices with a transpose flag
  // (DoubleSection.hpp:129-151); UIDs follow CSC order of the upper pattern.
  auto add_u = [&](int e, int slot, int ui, int uj) {
    const int ni = P.perm[ui], nj = P.perm[uj];
    Contrib c;
    c.edge = e;
    c.slot = slot;
    c.tr = (nj < ni) ? 1 : 0;
    c.r = std::min(ni, nj);
    c.c = std::max(ni, nj);
    c.key = (int64_t)c.c * NU + c.r;
    cu.push_back(c);
  };
  auto add_v = [&](int e, int slot, int vi, int vj) {
    Contrib c;
    c.edge = e;
    c.slot = slot;
    c.tr = 0;
    c.r = vi;
    c.c = vj;
    c.key = (int64_t)vj * NV + vi;  // CSC
    cv.push_back(c);
  };
  auto add_w = [&](int e, int ui, int vj) {
    Contrib c;
    c.edge = e;
    c.slot = 12;
    c.tr = 0;
    c.r = P.perm[ui];
    c.c = vj;
    c.key = (int64_t)c.r * NV + vj;  // CSR, row = permuted camera
    cw.push_back(c);
  };
  for (int e = 0; e < ne; e++) {
    const Edge& E = P.edges[e];
    switch (E.type) {
      case ORC_EDGE_UNARY_U:
        if (!E.fixed1) add_u(e, 11, E.id1, E.id1);
        break;
      case ORC_EDGE_UNARY_V:
        if (!E.fixed1) add_v(e, 11, E.id1, E.id1);
        break;
      case ORC_EDGE_BINARY_UU:
        if (!E.fixed1) add_u(e, 11, E.id1, E.id1);
        if (!E.fixed1 && !E.fixed2) {
          if (!(E.id1 < E.id2)) return -2;  // DoubleSection.hpp:355
          add_u(e, 12, E.id1, E.id2);
        }
        if (!E.fixed2) add_u(e, 22, E.id2, E.id2);
        break;
      case ORC_EDGE_BINARY_UV:
        if (!E.fixed1) add_u(e, 11, E.id1, E.id1);
        if (!E.fixed1 && !E.fixed2) add_w(e, E.id1, E.id2);
        if (!E.fixed2) add_v(e, 22, E.id2, E.id2);
        break;
      default:
        return -2;
    }
  }
  // Inside a block the updater list holds edges newest-first
  // (std::forward_list::emplace_front, DoubleSection.hpp:349-363).
  auto cmp = [](const Contrib& a, const Contrib& b) {
    return a.key != b.key ? a.key < b.key : a.edge > b.edge;
  };
  std::sort(cu.begin(), cu.end(), cmp);
  std::sort(cv.begin(), cv.end(), cmp);
  std::sort(cw.begin(), cw.end(), cmp);

  P.h11.assign(ne, -1);
  P.h12.assign(ne, -1);
  P.h22.assign(ne, -1);
  P.u_r.clear(); P.u_c.clear(); P.u_tr.clear();
  P.v_r.clear(); P.v_c.clear(); P.w_r.clear(); P.w_c.clear();
  P.unit_ptr.assign(1, 0);
  P.unit_edge.clear();
  P.unit_slot.clear();
  auto emit = [&](std::vector<Contrib>& cs, std::vector<int>& br, std::vector<int>& bc,
                  std::vector<char>* btr) {
    int uid = -1;
    int64_t last = -1;
    for (size_t q = 0; q < cs.size(); q++) {
      const Contrib& c = cs[q];
      if (c.key != last) {
        if (uid >= 0) P.unit_ptr.push_back((int)P.unit_edge.size());
        uid++;
        last = c.key;
        br.push_back(c.r);
        bc.push_back(c.c);
        if (btr) btr->push_back((char)c.tr);
      }
      P.unit_edge.push_back(c.edge);
      P.unit_slot.push_back(c.slot);
      if (c.slot == 11) P.h11[c.edge] = uid;
      if (c.slot == 12) P.h12[c.edge] = uid;
      if (c.slot == 22) P.h22[c.edge] = uid;
    }
    if (uid >= 0) P.unit_ptr.push_back((int)P.unit_edge.size());
    return uid + 1;
  };
  P.nU = emit(cu, P.u_r, P.u_c, &P.u_tr);
  P.nV = emit(cv, P.v_r, P.v_c, nullptr);
  P.nW = emit(cw, P.w_r, P.w_c, nullptr);

  P.v_diag_uid.assign(P.nv_var, -1);
  for (int q = 0; q < P.nV; q++) {
    if (P.v_r[q] != P.v_c[q]) return -3;  // the V solve needs a block-diagonal V
    P.v_diag_uid[P.v_c[q]] = q;
  }
  P.u_diag_uid.assign(P.nu_var, -1);
  for (int q = 0; q < P.nU; q++)
    if (P.u_r[q] == P.u_c[q]) P.u_diag_uid[P.u_c[q]] = q;
  P.w_row_ptr.assign(P.nu_var + 1, 0);
  for (int q = 0; q < P.nW; q++) P.w_row_ptr[P.w_r[q] + 1]++;
  for (int i = 0; i < P.nu_var; i++) P.w_row_ptr[i + 1] += P.w_row_ptr[i];
  P.w_col_ptr.assign(P.nv_var + 1, 0);
  for (int q = 0; q < P.nW; q++) P.w_col_ptr[P.w_c[q] + 1]++;
  for (int j = 0; j < P.nv_var; j++) P.w_col_ptr[j + 1] += P.w_col_ptr[j];
  P.w_col_uid.assign(P.nW, 0);
  {
    std::vector<int> fill(P.w_col_ptr.begin(), P.w_col_ptr.end() - 1);
    for (int q = 0; q < P.nW; q++) P.w_col_uid[fill[P.w_c[q]]++] = q;  // rows ascending
  }
  const int bu = P.bu, bv = P.bv;
  P.U.assign((size_t)P.nU * bu * bu, 0.0);
  P.V.assign((size_t)P.nV * bv * bv, 0.0);
  P.W.assign((size_t)P.nW * bu * bv, 0.0);
  P.bU.assign((size_t)P.nu_var * bu, 0.0);
  P.bV.assign((size_t)P.nv_var * bv, 0.0);
  P.ready = true;
  return 0;
}

// ---------------------------------------------------------------------------
// Edge evaluation (BaseSection::evaluateEdges, nelson/BaseSection.cpp:88-169).
const double* param_u(const Problem& P, int id, bool fixed) {
  const int stride = P.kind == ORC_KIND_BA ? kCamState : P.bu;
  return P.u.data() + (size_t)(fixed ? P.nu_var + id : id) * stride;
}
const double* param_v(const Problem& P, int id, bool fixed) {
  return P.v.data() + (size_t)(fixed ? P.nv_var + id : id) * P.bv;
}
// Dimension of the first / second parameter of an edge.
inline int dim1(const Problem& P, const Edge& E) { return E.type == ORC_EDGE_UNARY_V ? P.bv : P.bu; }
inline int dim2(const Problem& P, const Edge& E) { return E.type == ORC_EDGE_BINARY_UU ? P.bu : P.bv; }

void evaluate_edges(Problem& P, bool hessian) {
  const int ne = (int)P.edges.size();
  const int dr = P.dr_max;
#pragma omp parallel for num_threads(P.nthreads) schedule(static)
  for (int e = 0; e < ne; e++) {
    const Edge& E = P.edges[e];
    double* r = P.er.data() + (size_t)e * dr;
    double* J1 = P.eJ1.data() + (size_t)e * P.s1;
    double* J2 = P.eJ2.data() + (size_t)e * P.s2;
    if (P.kind == ORC_KIND_BA) {
      ba_eval(param_u(P, E.id1, E.fixed1), param_v(P, E.id2, E.fixed2), E.z,
              P.f_fixed, P.cx, P.cy, P.bu, hessian, r, J1, J2);
    } else {
      const int b1 = dim1(P, E), b2 = dim2(P, E);
      const double* x1 = E.type == ORC_EDGE_UNARY_V ? param_v(P, E.id1, E.fixed1)
                                                    : param_u(P, E.id1, E.fixed1);
      const double* x2 = nullptr;
      if (E.type == ORC_EDGE_BINARY_UU) x2 = param_u(P, E.id2, E.fixed2);
      if (E.type == ORC_EDGE_BINARY_UV) x2 = param_v(P, E.id2, E.fixed2);
      for (int i = 0; i < E.dr; i++) {
        double s = 0;
        for (int k = 0; k < b1; k++) s += J1[i * b1 + k] * x1[k];
        if (x2)
          for (int k = 0; k < b2; k++) s += J2[i * b2 + k] * x2[k];
        r[i] = s - E.z[i];
      }
    }
    double c = 0;
    for (int i = 0; i < E.dr; i++) c += r[i] * r[i];
    P.echi2[e] = E.w * c;
  }
  // chi2 summed in insertion order (the reference's single-thread loop).
  double chi2 = 0;
  for (int e = 0; e < ne; e++) chi2 += P.echi2[e];
  P.chi2 = chi2;
}

// Hessian block accumulation (BaseSection::updateHessianBlocks,
// nelson/BaseSection.cpp:5-86 -> EdgeBinarySectionBaseCRPT::updateH_11/12/22,
// nelson/EdgeBinary.h:133-157): one computation unit per H block, updaters
// applied in list order.  Edge e adds w J1'J1 / w J1'r to its first
// parameter's blocks, w J2'J2 / w J2'r to its second's, and w J1'J2 to the
// coupling block (w J2'J1 when the permuted U block is stored transposed).
void update_hessian_blocks(Problem& P) {
  std::fill(P.U.begin(), P.U.end(), 0.0);
  std::fill(P.V.begin(), P.V.end(), 0.0);
  std::fill(P.W.begin(), P.W.end(), 0.0);
  std::fill(P.bU.begin(), P.bU.end(), 0.0);
  std::fill(P.bV.begin(), P.bV.end(), 0.0);
  const int nunits = P.nU + P.nV + P.nW;
  const int bu = P.bu, bv = P.bv;
#pragma omp parallel for num_threads(P.nthreads) schedule(dynamic, 64)
  for (int q = 0; q < nunits; q++) {
    int mat, uid;  // 0 = U, 1 = V, 2 = W
    if (q < P.nU) { mat = 0; uid = q; }
    else if (q < P.nU + P.nV) { mat = 1; uid = q - P.nU; }
    else { mat = 2; uid = q - P.nU - P.nV; }
    for (int t = P.unit_ptr[q]; t < P.unit_ptr[q + 1]; t++) {
      const int e = P.unit_edge[t];
      const int slot = P.unit_slot[t];
      const Edge& E = P.edges[e];
      const double w = E.w;
      const double* r = P.er.data() + (size_t)e * P.dr_max;
      const double* J1 = P.eJ1.data() + (size_t)e * P.s1;
      const double* J2 = P.eJ2.data() + (size_t)e * P.s2;
      const int dr = E.dr;
      const int b1 = dim1(P, E), b2 = dim2(P, E);
      if (slot == 12) {
        const int rows = mat == 2 ? bu : bu;
        const int cols = mat == 2 ? bv : bu;
        double* H = (mat == 2 ? P.W.data() + (size_t)uid * bu * bv : P.U.data() + (size_t)uid * bu * bu);
        const bool tr = mat == 0 && P.u_tr[uid] != 0;
        for (int i = 0; i < rows; i++)
          for (int j = 0; j < cols; j++) {
            double s = 0;
            for (int k = 0; k < dr; k++)
              s += tr ? J2[k * b2 + i] * J1[k * b1 + j] : J1[k * b1 + i] * J2[k * b2 + j];
            H[i * cols + j] += w * s;
          }
        continue;
      }
      const int B = mat == 0 ? bu : bv;
      double* H = (mat == 0 ? P.U.data() : P.V.data()) + (size_t)uid * B * B;
      const double* J = slot == 11 ? J1 : J2;
      const int Bj = slot == 11 ? b1 : b2;  // == B
      const int pid = slot == 11 ? E.id1 : E.id2;
      double* b = mat == 0 ? P.bU.data() + (size_t)P.perm[pid] * bu : P.bV.data() + (size_t)pid * bv;
      for (int i = 0; i < B; i++) {
        for (int j = 0; j < B; j++) {
          double s = 0;
          for (int k = 0; k < dr; k++) s += J[k * Bj + i] * J[k * Bj + j];
          H[i * B + j] += w * s;
        }
        double s = 0;
        for (int k = 0; k < dr; k++) s += J[k * Bj + i] * r[k];
        b[i] += w * s;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// SolverCholeskySchur (nelson/SolverCholeskySchur.hpp:44-157) with the V
// solve done block by block (MatrixDiagInv, nelson/MatrixDiagInv.hpp:32-43).
double max_abs_hdiag(const Problem& P) {
  // SolverCholeskySchur::maxAbsHDiag (SolverCholeskySchur.hpp:75-78)
  double m = std::numeric_limits<double>::lowest();
  for (int p = 0; p < P.nv_var; p++) {
    const int q = P.v_diag_uid[p];
    for (int i = 0; i < P.bv; i++)
      m = std::max(m, q >= 0 ? std::fabs(P.V[(size_t)q * P.bv * P.bv + i * P.bv + i]) : 0.0);
  }
  for (int c = 0; c < P.nu_var; c++) {
    const int q = P.u_diag_uid[c];
    for (int i = 0; i < P.bu; i++)
      m = std::max(m, q >= 0 ? std::fabs(P.U[(size_t)q * P.bu * P.bu + i * P.bu + i]) : 0.0);
  }
  return m;
}

bool compute_increment(Problem& P, double rel, double abs) {
  const int bu = P.bu, bv = P.bv;
  const int nc = P.nu_var, np = P.nv_var;
  const int n = nc * bu;
  P.n = n;
  P.Vinv.assign((size_t)np * bv * bv, 0.0);
  P.xV0.assign((size_t)np * bv, 0.0);
  P.incU.assign((size_t)n, 0.0);
  P.incV.assign((size_t)np * bv, 0.0);
  int bad = 0;
  // (1) V_mu^-1 and xV0 = V_mu^-1 (-bV)   (SolverCholeskySchur.hpp:100)
#pragma omp parallel for num_threads(P.nthreads) schedule(static) reduction(+ : bad)
  for (int p = 0; p < np; p++) {
    double A[81] = {0};
    const int q = P.v_diag_uid[p];
    if (q >= 0) {
      const double* Vb = P.V.data() + (size_t)q * bv * bv;
      for (int i = 0; i < bv; i++)
        for (int j = 0; j < bv; j++) A[i * bv + j] = (i <= j) ? Vb[i * bv + j] : Vb[j * bv + i];
    }
    if (rel != 0 || abs != 0)
      for (int i = 0; i < bv; i++) A[i * bv + i] = A[i * bv + i] * (1 + rel) + abs;
    double* Vi = P.Vinv.data() + (size_t)p * bv * bv;
    if (!small_spd_inverse(A, bv, Vi)) { bad++; continue; }
    const double* b = P.bV.data() + (size_t)p * bv;
    for (int i = 0; i < bv; i++) {
      double s = 0;
      for (int j = 0; j < bv; j++) s -= Vi[i * bv + j] * b[j];
      P.xV0[(size_t)p * bv + i] = s;
    }
  }
  bool ok = bad == 0;
  if (ok) {
    // (2) bS = -bU - W xV0   (SolverCholeskySchur.hpp:114)
    P.bS.assign((size_t)n, 0.0);
#pragma omp parallel for num_threads(P.nthreads) schedule(static)
    for (int c = 0; c < nc; c++) {
      for (int i = 0; i < bu; i++) {
        double s = -P.bU[(size_t)c * bu + i];
        for (int q = P.w_row_ptr[c]; q < P.w_row_ptr[c + 1]; q++) {
          const double* Wb = P.W.data() + (size_t)q * bu * bv;
          const double* x = P.xV0.data() + (size_t)P.w_c[q] * bv;
          for (int j = 0; j < bv; j++) s -= Wb[i * bv + j] * x[j];
        }
        P.bS[(size_t)c * bu + i] = s;
      }
    }
    // (3) S = triu(U - W V_mu^-1 W')   (SolverCholeskySchur.hpp:118)
    P.S.assign((size_t)n * n, 0.0);
    for (int q = 0; q < P.nU; q++) {
      const int r = P.u_r[q], c = P.u_c[q];
      const double* Ub = P.U.data() + (size_t)q * bu * bu;
      for (int i = 0; i < bu; i++)
        for (int j = 0; j < bu; j++) P.S[(size_t)(r * bu + i) * n + c * bu + j] = Ub[i * bu + j];
    }
#pragma omp parallel for num_threads(P.nthreads) schedule(dynamic, 1)
    for (int ci = 0; ci < nc; ci++) {
      double Y[81];
      for (int qa = P.w_row_ptr[ci]; qa < P.w_row_ptr[ci + 1]; qa++) {
        const int p = P.w_c[qa];
        const double* Wa = P.W.data() + (size_t)qa * bu * bv;
        const double* Vi = P.Vinv.data() + (size_t)p * bv * bv;
        for (int i = 0; i < bu; i++)
          for (int j = 0; j < bv; j++) {
            double s = 0;
            for (int k = 0; k < bv; k++) s += Wa[i * bv + k] * Vi[k * bv + j];
            Y[i * bv + j] = s;
          }
        for (int t = P.w_col_ptr[p]; t < P.w_col_ptr[p + 1]; t++) {
          const int qb = P.w_col_uid[t];
          const int cj = P.w_r[qb];
          if (cj < ci) continue;
          const double* Wb = P.W.data() + (size_t)qb * bu * bv;
          for (int i = 0; i < bu; i++)
            for (int j = 0; j < bu; j++) {
              double s = 0;
              for (int k = 0; k < bv; k++) s += Y[i * bv + k] * Wb[j * bv + k];
              P.S[(size_t)(ci * bu + i) * n + cj * bu + j] -= s;
            }
        }
      }
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < i; j++) P.S[(size_t)i * n + j] = 0.0;  // triangularView<Upper>
    // (4) diag(S) += rel diag(U) + abs   (SolverCholeskySchur.hpp:121-124)
    if (rel != 0 || abs != 0) {
      for (int c = 0; c < nc; c++) {
        const int q = P.u_diag_uid[c];
        for (int i = 0; i < bu; i++) {
          const double ud = q >= 0 ? P.U[(size_t)q * bu * bu + i * bu + i] : 0.0;
          double& s = P.S[(size_t)(c * bu + i) * n + c * bu + i];
          s += rel * ud;
          s += abs;
        }
      }
    }
    // (5) factorize S, solve for xU   (SolverCholeskySchur.hpp:136-140)
    std::vector<double> L(P.S);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < i; j++) L[(size_t)i * n + j] = L[(size_t)j * n + i];
    ok = chol_blocked(L.data(), n, n, P.nthreads);
    if (ok) {
      std::copy(P.bS.begin(), P.bS.end(), P.incU.begin());
      chol_solve(L.data(), n, n, P.incU.data());
      // (6) bVt = -bV - W' xU; xV = V_mu^-1 bVt   (SolverCholeskySchur.hpp:144-147)
#pragma omp parallel for num_threads(P.nthreads) schedule(static)
      for (int p = 0; p < np; p++) {
        double t[9];
        for (int j = 0; j < bv; j++) t[j] = -P.bV[(size_t)p * bv + j];
        for (int s = P.w_col_ptr[p]; s < P.w_col_ptr[p + 1]; s++) {
          const int q = P.w_col_uid[s];
          const double* Wb = P.W.data() + (size_t)q * bu * bv;
          const double* x = P.incU.data() + (size_t)P.w_r[q] * bu;
          for (int j = 0; j < bv; j++)
            for (int i = 0; i < bu; i++) t[j] -= Wb[i * bv + j] * x[i];
        }
        const double* Vi = P.Vinv.data() + (size_t)p * bv * bv;
        for (int i = 0; i < bv; i++) {
          double s = 0;
          for (int j = 0; j < bv; j++) s += Vi[i * bv + j] * t[j];
          P.incV[(size_t)p * bv + i] = s;
        }
      }
    }
  }
  if (!ok) {  // SolverCholeskySchur.hpp:151-154
    std::fill(P.incU.begin(), P.incU.end(), 0.0);
    std::fill(P.incV.begin(), P.incV.end(), 0.0);
  }
  return ok;
}

double inc_sqnorm(const Problem& P) {
  double s = 0;
  for (double x : P.incU) s += x * x;
  for (double x : P.incV) s += x * x;
  return s;
}

double max_abs_b(const Problem& P) {
  // DoubleSectionHessian::maxAbsValBVect (DoubleSectionHessian.hpp:61-63)
  double mu = 0, mv = 0;
  for (double x : P.bU) mu = std::max(mu, std::fabs(x));
  for (double x : P.bV) mv = std::max(mv, std::fabs(x));
  return std::max(mu, mv);
}

// DoubleSection::computeRhoChi2Change (nelson/DoubleSection.h:300-311).
double rho(const Problem& P, double mu, double old_chi2) {
  const double num = old_chi2 - P.chi2;
  double den = 0;
  for (size_t i = 0; i < P.incU.size(); i++) den += P.incU[i] * (mu * P.incU[i] - P.bU[i]);
  for (size_t i = 0; i < P.incV.size(); i++) den += P.incV[i] * (mu * P.incV[i] - P.bV[i]);
  return num / den;
}

// Problem::oplus: cameras R <- exp(dw) R, t += dt, intrinsics += d; the
// camera increment is read at its internal (permuted) position, as the
// reference's problems do (testDoubleSectionSchurDiagBlockWWtFFFF.cpp:401).
void oplus(Problem& P) {
  const int bu = P.bu, bv = P.bv;
  if (P.kind == ORC_KIND_BA) {
#pragma omp parallel for num_threads(P.nthreads) schedule(static)
    for (int c = 0; c < P.nu_var; c++) {
      const double* d = P.incU.data() + (size_t)P.perm[c] * bu;
      double* s = P.u.data() + (size_t)c * kCamState;
      double dR[9], R[9];
      so3_exp(d, dR);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          R[i * 3 + j] = dR[i * 3] * s[j] + dR[i * 3 + 1] * s[3 + j] + dR[i * 3 + 2] * s[6 + j];
      for (int i = 0; i < 9; i++) s[i] = R[i];
      for (int i = 0; i < 3; i++) s[9 + i] += d[3 + i];
      if (bu == 9)
        for (int i = 0; i < 3; i++) s[12 + i] += d[6 + i];
    }
  } else {
    for (int c = 0; c < P.nu_var; c++)
      for (int i = 0; i < bu; i++) P.u[(size_t)c * bu + i] += P.incU[(size_t)P.perm[c] * bu + i];
  }
#pragma omp parallel for num_threads(P.nthreads) schedule(static)
  for (int p = 0; p < P.nv_var; p++)
    for (int i = 0; i < bv; i++) P.v[(size_t)p * bv + i] += P.incV[(size_t)p * bv + i];
}

void backup(Problem& P) {
  P.u_bck = P.u;
  P.v_bck = P.v;
}
void rollback(Problem& P) {
  P.u = P.u_bck;
  P.v = P.v_bck;
}

void update(Problem& P, bool hessian) {
  // DoubleSection::update (DoubleSection.hpp:452-467)
  evaluate_edges(P, hessian);
  if (hessian) update_hessian_blocks(P);
}

void trace_push(double* trace, int cap, int* n, double it, double sub, double chi2,
                double mu, double rh, double inc, double ok, double acc) {
  if (trace && *n < cap) {
    double* t = trace + (size_t)(*n) * ORC_TRACE_STRIDE;
    t[0] = it; t[1] = sub; t[2] = chi2; t[3] = mu; t[4] = rh; t[5] = inc; t[6] = ok; t[7] = acc;
  }
  (*n)++;
}

// LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146).
int lm_solve(Problem& P, const orc_lm_settings& s, double* trace, int cap, int* ntr,
             int* its) {
  enum { SuccessAtStart, SuccessSmallIncrement, SuccessEpsB, SuccessSmallResiduals,
         SolverFailure, MaxIterationReached, MaxSubIterationReached };
  int n = 0;
  int iter = -1, subiter = -1;
  auto finish = [&](int reason) {
    if (ntr) *ntr = std::min(n, cap);
    if (its) { its[0] = iter; its[1] = subiter; }
    return reason;
  };
  update(P, true);
  trace_push(trace, cap, &n, iter, subiter, P.chi2, 0, 0, 0, 1, 1);
  if (max_abs_b(P) <= s.epsBVector) return finish(SuccessAtStart);
  backup(P);
  double oldChi2 = P.chi2;
  double mu = s.tau * max_abs_hdiag(P);
  double curV = s.initV;
  iter = 0;
  while (iter < s.maxNumIt) {
    subiter = 0;
    bool toRepeat = false;
    do {
      const double mu_used = mu;
      const bool solveOk = compute_increment(P, 0.0, mu);
      const double inc = inc_sqnorm(P);
      if (solveOk && iter >= s.minNumIt && inc <= s.epsIncSquare) {
        trace_push(trace, cap, &n, iter, subiter, P.chi2, mu_used, 0, inc, 1, 0);
        return finish(SuccessSmallIncrement);
      }
      double rh = -1;
      double chi2_rec = -1;
      if (solveOk) {
        oplus(P);
        update(P, false);
        chi2_rec = P.chi2;
        rh = rho(P, mu, oldChi2);
      }
      const bool accepted = solveOk && rh > 0;
      trace_push(trace, cap, &n, iter, subiter, chi2_rec, mu_used, rh, inc, solveOk ? 1 : 0,
                 accepted ? 1 : 0);
      if (accepted) {
        if (iter > s.minNumIt && max_abs_b(P) <= s.epsBVector) return finish(SuccessEpsB);
        if (iter > s.minNumIt && P.chi2 < s.epsChi2) return finish(SuccessSmallResiduals);
        const double fc = 2 * rh - 1;
        double alpha = std::min(s.maxScaleFactor, 1 - fc * fc * fc);
        alpha = std::max(s.minScaleFactor, alpha);
        mu = mu * alpha;
        curV = s.initV;
      } else {
        rollback(P);
        mu = mu * curV;
        curV = curV * s.penaltyV;
      }
      subiter++;
      if (subiter >= s.maxNumSubIt) return finish(MaxSubIterationReached);
      toRepeat = (rh <= 0 || !solveOk);
    } while (toRepeat);
    update(P, true);
    backup(P);
    oldChi2 = P.chi2;
    iter++;
  }
  return finish(MaxIterationReached);
}

// GaussNewton::solve (nelson/GaussNewton.hpp:32-127).
int gn_solve(Problem& P, const orc_gn_settings& s, double* trace, int cap, int* ntr,
             int* its) {
  enum { SuccessAtStart, SuccessSmallIncrement, SuccessEpsB, SuccessSmallResiduals,
         SolverFailure, MaxIterationReached };
  int n = 0;
  int iter = -1;
  auto finish = [&](int reason) {
    if (ntr) *ntr = std::min(n, cap);
    if (its) { its[0] = iter; its[1] = 0; }
    return reason;
  };
  update(P, true);
  trace_push(trace, cap, &n, iter, 0, P.chi2, 0, 0, 0, 1, 1);
  if (max_abs_b(P) <= s.epsBVector) return finish(SuccessAtStart);
  iter = 0;
  while (iter < s.maxNumIt) {
    const bool ok = compute_increment(P, s.relLambda, s.absLambda);
    const double inc = inc_sqnorm(P);
    if (!ok) {
      trace_push(trace, cap, &n, iter, 0, -1, 0, 0, inc, 0, 0);
      return finish(SolverFailure);
    }
    if (iter >= s.minNumIt && inc <= s.epsIncSquare) {
      trace_push(trace, cap, &n, iter, 0, P.chi2, 0, 0, inc, 1, 0);
      return finish(SuccessSmallIncrement);
    }
    oplus(P);
    update(P, true);
    trace_push(trace, cap, &n, iter, 0, P.chi2, 0, 0, inc, 1, 1);
    if (iter > s.minNumIt && max_abs_b(P) <= s.epsBVector) return finish(SuccessEpsB);
    if (iter > s.minNumIt && P.chi2 < s.epsChi2) return finish(SuccessSmallResiduals);
    iter++;
  }
  return finish(MaxIterationReached);
}

Problem* as(void* h) { return static_cast<Problem*>(h); }

// ---------------------------------------------------------------------------
// Implicit-function adjoint of a converged BA solve, in FP64 (no counterpart
// in the reference, which has no differentiation; it is the CPU reference
// gradient the CUDA adjoint is checked against).
//
// At x* the local gradient b = sum_e w_e J_e' r_e vanishes; for a loss with
// gradient dL/dx, H' mu = dL/dx with H = db/dx (derivative along the
// retraction: R <- exp(dw) R, the rest additive), and
//   dL/dz_e = w_e J_e mu_e,   dL/dw_e = -(J_e mu_e) . r_e.
// H is assembled edge by edge from the derivative of the edge's own gradient
// g_e = w_e J_e' r_e, taken by complex-step differentiation (the projection
// and its analytic Jacobian evaluated in complex arithmetic at x* + i h v,
// Im(g_e) / h, h = 1e-20: exact to rounding, no cancellation), so it is
// independent of the forward-mode dual numbers the CUDA kernels use.  Its
// blocks have the Gauss-Newton Hessian's pattern; each is symmetrised (the
// antisymmetric part is proportional to b and vanishes at x*) and H mu =
// dL/dx is solved with the oracle's own Schur solve at zero damping.
template <typename T>
void ba_resjac_t(const T* R, const T* t, T f, T k1, T k2, const T* X, const double* z, double cx,
                 double cy, int bc, T* r, T* Jc, T* Jp) {
  const T a0 = R[0] * X[0] + R[1] * X[1] + R[2] * X[2];
  const T a1 = R[3] * X[0] + R[4] * X[1] + R[5] * X[2];
  const T a2 = R[6] * X[0] + R[7] * X[1] + R[8] * X[2];
  const T P0 = a0 + t[0], P1 = a1 + t[1], P2 = a2 + t[2];
  const T iz = T(1.0) / P2;
  const T x = P0 * iz, y = P1 * iz;
  const T r2 = x * x + y * y;
  const T d = T(1.0) + r2 * (k1 + k2 * r2);
  r[0] = f * d * x + T(cx - z[0]);
  r[1] = f * d * y + T(cy - z[1]);
  const T g = T(2.0) * (k1 + T(2.0) * k2 * r2);
  const T m00 = f * (d + g * x * x), m01 = f * g * x * y, m11 = f * (d + g * y * y);
  const T M[6] = {m00 * iz, m01 * iz, -(m00 * x + m01 * y) * iz,
                  m01 * iz, m11 * iz, -(m01 * x + m11 * y) * iz};
  for (int i = 0; i < 2; i++) {
    const T* m = M + 3 * i;
    for (int j = 0; j < 3; j++) Jp[i * 3 + j] = m[0] * R[j] + m[1] * R[3 + j] + m[2] * R[6 + j];
    T* jc = Jc + i * bc;
    jc[0] = m[2] * a1 - m[1] * a2;
    jc[1] = m[0] * a2 - m[2] * a0;
    jc[2] = m[1] * a0 - m[0] * a1;
    jc[3] = m[0];
    jc[4] = m[1];
    jc[5] = m[2];
  }
  if (bc == 9) {
    Jc[6] = d * x;
    Jc[7] = f * x * r2;
    Jc[8] = f * x * r2 * r2;
    Jc[9 + 6] = d * y;
    Jc[9 + 7] = f * y * r2;
    Jc[9 + 8] = f * y * r2 * r2;
  }
}

// Edge gradient g = w [Jc' r; Jp' r] at the camera state `cs` and point X,
// perturbed by i h along local direction k (k < bc: camera tangent, else
// point coordinate k - bc); returns Im(g) / h in col (bc + 3 entries).
void edge_hessian_column(const double* cs, const double* X, const double* z, double w, double f_fixed,
                         double cx, double cy, int bc, int k, double* col) {
  using Z = std::complex<double>;
  const double h = 1e-20;
  Z R[9], t[3], Xc[3], f, k1, k2;
  for (int i = 0; i < 9; i++) R[i] = cs[i];
  if (k < 3) {
    // exp(i h [e_k]x) R = R + i h [e_k]x R  (the h^2 term is below rounding)
    double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (k == 0) { K[5] = -1; K[7] = 1; }
    if (k == 1) { K[2] = 1; K[6] = -1; }
    if (k == 2) { K[1] = -1; K[3] = 1; }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double s = 0;
        for (int q = 0; q < 3; q++) s += K[i * 3 + q] * cs[q * 3 + j];
        R[i * 3 + j] += Z(0.0, h * s);
      }
  }
  for (int i = 0; i < 3; i++) t[i] = cs[9 + i];
  f = bc == 9 ? cs[12] : f_fixed;
  k1 = bc == 9 ? cs[13] : 0.0;
  k2 = bc == 9 ? cs[14] : 0.0;
  for (int i = 0; i < 3; i++) Xc[i] = X[i];
  if (k >= 3 && k < 6) t[k - 3] += Z(0.0, h);
  if (bc == 9 && k == 6) f += Z(0.0, h);
  if (bc == 9 && k == 7) k1 += Z(0.0, h);
  if (bc == 9 && k == 8) k2 += Z(0.0, h);
  if (k >= bc) Xc[k - bc] += Z(0.0, h);
  Z r[2], Jc[18], Jp[6];
  ba_resjac_t<Z>(R, t, f, k1, k2, Xc, z, cx, cy, bc, r, Jc, Jp);
  for (int i = 0; i < bc; i++) col[i] = w * (Jc[i] * r[0] + Jc[bc + i] * r[1]).imag() / h;
  for (int i = 0; i < 3; i++) col[bc + i] = w * (Jp[i] * r[0] + Jp[3 + i] * r[1]).imag() / h;
}

// Returns 1 when the solve succeeded.
int adjoint_ba(Problem& P, const double* dL_dcams, const double* dL_dpts, double* g_obs, double* g_w,
               double* mu_cams, double* mu_pts) {
  const int bc = P.bu, nc = P.nu_var, np = P.nv_var, ne = (int)P.edges.size();
  const int nl = bc + 3;
  update(P, true);  // r, J and the Gauss-Newton blocks at x* (the pattern and UIDs)
  std::vector<double> U(P.U.size(), 0.0), V(P.V.size(), 0.0), W(P.W.size(), 0.0);
  std::vector<double> He((size_t)nl * nl), col(nl);
  for (int e = 0; e < ne; e++) {  // insertion order: a fixed summation order
    const Edge& E = P.edges[e];
    const double* cs = param_u(P, E.id1, E.fixed1);
    const double* X = param_v(P, E.id2, E.fixed2);
    for (int k = 0; k < nl; k++) {
      if ((k < bc && E.fixed1) || (k >= bc && E.fixed2)) continue;
      edge_hessian_column(cs, X, E.z, E.w, P.f_fixed, P.cx, P.cy, bc, k, col.data());
      for (int i = 0; i < nl; i++) He[(size_t)i * nl + k] = col[i];
    }
    if (!E.fixed1) {
      double* Ub = U.data() + (size_t)P.h11[e] * bc * bc;
      for (int i = 0; i < bc; i++)
        for (int j = 0; j < bc; j++) Ub[i * bc + j] += 0.5 * (He[(size_t)i * nl + j] + He[(size_t)j * nl + i]);
    }
    if (!E.fixed2) {
      double* Vb = V.data() + (size_t)P.h22[e] * 9;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          Vb[i * 3 + j] += 0.5 * (He[(size_t)(bc + i) * nl + bc + j] + He[(size_t)(bc + j) * nl + bc + i]);
    }
    if (!E.fixed1 && !E.fixed2) {
      double* Wb = W.data() + (size_t)P.h12[e] * bc * 3;
      for (int i = 0; i < bc; i++)
        for (int j = 0; j < 3; j++)
          Wb[i * 3 + j] += 0.5 * (He[(size_t)i * nl + bc + j] + He[(size_t)(bc + j) * nl + i]);
    }
  }
  // H mu = dL/dx through the Schur solve: b := -dL/dx, zero damping
  std::vector<double> U0, V0, W0, bU0, bV0;
  U0.swap(P.U);
  V0.swap(P.V);
  W0.swap(P.W);
  bU0 = P.bU;
  bV0 = P.bV;
  P.U.swap(U);
  P.V.swap(V);
  P.W.swap(W);
  for (int c = 0; c < nc; c++)
    for (int i = 0; i < bc; i++) P.bU[(size_t)P.perm[c] * bc + i] = dL_dcams ? -dL_dcams[(size_t)c * bc + i] : 0.0;
  for (int i = 0; i < 3 * np; i++) P.bV[i] = dL_dpts ? -dL_dpts[i] : 0.0;
  const bool ok = compute_increment(P, 0.0, 0.0);
  const std::vector<double> muU = P.incU, muV = P.incV;  // internal camera order
  P.U.swap(U0);
  P.V.swap(V0);
  P.W.swap(W0);
  P.bU = bU0;
  P.bV = bV0;
  // per-edge VJP (insertion order)
  for (int e = 0; e < ne; e++) {
    const Edge& E = P.edges[e];
    const double* r = P.er.data() + (size_t)e * P.dr_max;
    const double* Jc = P.eJ1.data() + (size_t)e * P.s1;
    const double* Jp = P.eJ2.data() + (size_t)e * P.s2;
    double Jm[2] = {0.0, 0.0};
    if (!E.fixed1) {
      const double* m = muU.data() + (size_t)P.perm[E.id1] * bc;
      for (int i = 0; i < 2; i++)
        for (int k = 0; k < bc; k++) Jm[i] += Jc[i * bc + k] * m[k];
    }
    if (!E.fixed2) {
      const double* m = muV.data() + (size_t)E.id2 * 3;
      for (int i = 0; i < 2; i++)
        for (int k = 0; k < 3; k++) Jm[i] += Jp[i * 3 + k] * m[k];
    }
    if (g_obs) {
      g_obs[2 * (size_t)e] = E.w * Jm[0];
      g_obs[2 * (size_t)e + 1] = E.w * Jm[1];
    }
    if (g_w) g_w[e] = -(Jm[0] * r[0] + Jm[1] * r[1]);
  }
  if (mu_cams)
    for (int c = 0; c < nc; c++)
      for (int i = 0; i < bc; i++) mu_cams[(size_t)c * bc + i] = muU[(size_t)P.perm[c] * bc + i];
  if (mu_pts) std::copy(muV.begin(), muV.end(), mu_pts);
  return ok ? 1 : 0;
}

}  // namespace

// ===========================================================================
// C ABI
extern "C" {

void* orc_create(int kind, int bu, int bv, int nu_var, int nu_fix, int nv_var, int nv_fix,
                 int num_threads) {
  if (bu < 1 || bu > 9 || bv < 1 || bv > 9 || nu_var < 0 || nv_var < 0) return nullptr;
  if (kind == ORC_KIND_BA && !((bu == 6 || bu == 9) && bv == 3)) return nullptr;
  Problem* P = new Problem();
  P->kind = kind;
  P->bu = bu;
  P->bv = bv;
  P->nu_var = nu_var;
  P->nu_fix = nu_fix;
  P->nv_var = nv_var;
  P->nv_fix = nv_fix;
#ifdef _OPENMP
  P->nthreads = num_threads > 0 ? num_threads : omp_get_max_threads();
#else
  P->nthreads = 1;
#endif
  P->dr_max = kind == ORC_KIND_BA ? 2 : 3;
  if (kind == ORC_KIND_BA) {
    P->s1 = 2 * bu;
    P->s2 = 2 * bv;
  } else {
    P->s1 = P->s2 = 3 * std::max(bu, bv);
  }
  const int us = kind == ORC_KIND_BA ? kCamState : bu;
  P->u.assign((size_t)(nu_var + nu_fix) * us, 0.0);
  P->v.assign((size_t)(nv_var + nv_fix) * bv, 0.0);
  P->perm.resize(nu_var);
  std::iota(P->perm.begin(), P->perm.end(), 0);
  return P;
}

void orc_destroy(void* h) { delete as(h); }

int orc_set_intrinsics(void* h, double f, double cx, double cy) {
  as(h)->f_fixed = f;
  as(h)->cx = cx;
  as(h)->cy = cy;
  return 0;
}

int orc_set_params(void* h, const double* u, const double* v) {
  Problem& P = *as(h);
  const int nu = P.nu_var + P.nu_fix, nv = P.nv_var + P.nv_fix;
  if (P.kind == ORC_KIND_BA) {
    for (int c = 0; c < nu; c++) {
      const double* in = u + (size_t)c * P.bu;
      double* s = P.u.data() + (size_t)c * kCamState;
      so3_exp(in, s);
      for (int i = 0; i < 3; i++) s[9 + i] = in[3 + i];
      if (P.bu == 9) {
        s[12] = in[6]; s[13] = in[7]; s[14] = in[8];
      } else {
        s[12] = P.f_fixed; s[13] = 0; s[14] = 0;
      }
      s[15] = 0;
    }
  } else {
    std::copy(u, u + (size_t)nu * P.bu, P.u.begin());
  }
  std::copy(v, v + (size_t)nv * P.bv, P.v.begin());
  return 0;
}

int orc_get_params(void* h, double* u, double* v) {
  Problem& P = *as(h);
  const int nu = P.nu_var + P.nu_fix;
  if (P.kind == ORC_KIND_BA) {
    for (int c = 0; c < nu; c++) {
      const double* s = P.u.data() + (size_t)c * kCamState;
      double* o = u + (size_t)c * P.bu;
      so3_log(s, o);
      for (int i = 0; i < 3; i++) o[3 + i] = s[9 + i];
      if (P.bu == 9) { o[6] = s[12]; o[7] = s[13]; o[8] = s[14]; }
    }
  } else {
    std::copy(P.u.begin(), P.u.end(), u);
  }
  std::copy(P.v.begin(), P.v.end(), v);
  return 0;
}

int orc_get_camera_state(void* h, double* states) {
  Problem& P = *as(h);
  if (P.kind != ORC_KIND_BA) return -1;
  std::copy(P.u.begin(), P.u.end(), states);
  return 0;
}

int orc_add_ba_edges(void* h, int ne, const int* cam, const int* cam_fixed, const int* pt,
                     const int* pt_fixed, const double* obs, const double* weight) {
  Problem& P = *as(h);
  if (P.kind != ORC_KIND_BA || P.ready) return -1;
  P.edges.reserve(P.edges.size() + ne);
  for (int e = 0; e < ne; e++) {
    Edge E;
    E.type = ORC_EDGE_BINARY_UV;
    E.id1 = cam[e];
    E.fixed1 = cam_fixed && cam_fixed[e];
    E.id2 = pt[e];
    E.fixed2 = pt_fixed && pt_fixed[e];
    const int lim1 = E.fixed1 ? P.nu_fix : P.nu_var;
    const int lim2 = E.fixed2 ? P.nv_fix : P.nv_var;
    if (E.id1 < 0 || E.id1 >= lim1 || E.id2 < 0 || E.id2 >= lim2) return -2;
    E.dr = 2;
    E.z[0] = obs[2 * e];
    E.z[1] = obs[2 * e + 1];
    E.z[2] = 0;
    E.w = weight ? weight[e] : 1.0;
    P.edges.push_back(E);
  }
  return 0;
}

int orc_add_linear_edge(void* h, int type, int id1, int fixed1, int id2, int fixed2, int dr,
                        const double* A1, const double* A2, const double* z) {
  Problem& P = *as(h);
  if (P.kind != ORC_KIND_LINEAR || P.ready || dr < 1 || dr > 3) return -1;
  Edge E;
  E.type = type;
  E.id1 = id1;
  E.fixed1 = fixed1 != 0;
  E.id2 = id2;
  E.fixed2 = fixed2 != 0;
  E.dr = dr;
  for (int i = 0; i < 3; i++) E.z[i] = i < dr ? z[i] : 0.0;
  E.w = 1.0;
  const size_t e = P.edges.size();
  P.edges.push_back(E);
  // constant Jacobians live in the per-edge cache from the start
  P.eJ1.resize((e + 1) * P.s1, 0.0);
  P.eJ2.resize((e + 1) * P.s2, 0.0);
  const int b1 = dim1(P, E), b2 = dim2(P, E);
  for (int i = 0; i < dr * b1; i++) P.eJ1[e * P.s1 + i] = A1[i];
  if (type == ORC_EDGE_BINARY_UU || type == ORC_EDGE_BINARY_UV)
    for (int i = 0; i < dr * b2; i++) P.eJ2[e * P.s2 + i] = A2[i];
  return 0;
}

int orc_set_user2internal_u(void* h, const int* perm) {
  Problem& P = *as(h);
  if (P.ready) return -1;
  std::vector<int> seen(P.nu_var, 0);
  for (int i = 0; i < P.nu_var; i++) {
    if (perm[i] < 0 || perm[i] >= P.nu_var || seen[perm[i]]) return -2;
    seen[perm[i]] = 1;
  }
  std::copy(perm, perm + P.nu_var, P.perm.begin());
  return 0;
}

int orc_structure_ready(void* h) {
  Problem& P = *as(h);
  if (P.ready) return -1;
  const size_t ne = P.edges.size();
  P.er.assign(ne * P.dr_max, 0.0);
  P.echi2.assign(ne, 0.0);
  if (P.kind == ORC_KIND_BA) {
    P.eJ1.assign(ne * P.s1, 0.0);
    P.eJ2.assign(ne * P.s2, 0.0);
  }
  return build_structure(P);
}

int orc_get_counts(void* h, int* counts) {
  Problem& P = *as(h);
  counts[0] = P.nU;
  counts[1] = P.nV;
  counts[2] = P.nW;
  counts[3] = (int)P.edges.size();
  return 0;
}

int orc_get_patterns(void* h, int* u_rc, int* v_rc, int* w_rc) {
  Problem& P = *as(h);
  for (int q = 0; q < P.nU; q++) { u_rc[2 * q] = P.u_r[q]; u_rc[2 * q + 1] = P.u_c[q]; }
  for (int q = 0; q < P.nV; q++) { v_rc[2 * q] = P.v_r[q]; v_rc[2 * q + 1] = P.v_c[q]; }
  for (int q = 0; q < P.nW; q++) { w_rc[2 * q] = P.w_r[q]; w_rc[2 * q + 1] = P.w_c[q]; }
  return 0;
}

int orc_get_edge_uids(void* h, int* h11, int* h12, int* h22) {
  Problem& P = *as(h);
  std::copy(P.h11.begin(), P.h11.end(), h11);
  std::copy(P.h12.begin(), P.h12.end(), h12);
  std::copy(P.h22.begin(), P.h22.end(), h22);
  return 0;
}

int orc_update(void* h, int hessian, double* chi2) {
  Problem& P = *as(h);
  if (!P.ready) return -1;
  update(P, hessian != 0);
  if (chi2) *chi2 = P.chi2;
  return 0;
}

int orc_get_hessian(void* h, double* U, double* V, double* W, double* bU, double* bV) {
  Problem& P = *as(h);
  if (U) std::copy(P.U.begin(), P.U.end(), U);
  if (V) std::copy(P.V.begin(), P.V.end(), V);
  if (W) std::copy(P.W.begin(), P.W.end(), W);
  if (bU) std::copy(P.bU.begin(), P.bU.end(), bU);
  if (bV) std::copy(P.bV.begin(), P.bV.end(), bV);
  return 0;
}

int orc_get_residuals(void* h, double* r) {
  Problem& P = *as(h);
  for (size_t e = 0; e < P.edges.size(); e++)
    for (int i = 0; i < P.edges[e].dr; i++) r[e * P.edges[e].dr + i] = P.er[e * P.dr_max + i];
  return 0;
}

int orc_adjoint_ba(void* h, const double* dL_dcams, const double* dL_dpts, double* g_obs, double* g_w,
                   double* mu_cams, double* mu_pts) {
  Problem& P = *as(h);
  if (!P.ready || P.kind != ORC_KIND_BA) return -1;
  return adjoint_ba(P, dL_dcams, dL_dpts, g_obs, g_w, mu_cams, mu_pts);
}

int orc_solver_init(void* h) { return as(h)->ready ? 0 : -1; }
double orc_max_abs_hdiag(void* h) { return max_abs_hdiag(*as(h)); }
int orc_compute_increment(void* h, double rel, double abs) {
  return compute_increment(*as(h), rel, abs) ? 1 : 0;
}
int orc_get_increment(void* h, double* incU, double* incV) {
  Problem& P = *as(h);
  std::copy(P.incU.begin(), P.incU.end(), incU);
  std::copy(P.incV.begin(), P.incV.end(), incV);
  return 0;
}
double orc_inc_sqnorm(void* h) { return inc_sqnorm(*as(h)); }
int orc_get_schur(void* h, double* S, double* bS, int* n) {
  Problem& P = *as(h);
  if (n) *n = P.n;
  if (S) std::copy(P.S.begin(), P.S.end(), S);
  if (bS) std::copy(P.bS.begin(), P.bS.end(), bS);
  return 0;
}
int orc_oplus(void* h) { oplus(*as(h)); return 0; }
int orc_backup(void* h) { backup(*as(h)); return 0; }
int orc_rollback(void* h) { rollback(*as(h)); return 0; }
double orc_max_abs_b(void* h) { return max_abs_b(*as(h)); }
double orc_chi2(void* h) { return as(h)->chi2; }
double orc_rho(void* h, double mu, double old_chi2) { return rho(*as(h), mu, old_chi2); }

int orc_lm_solve(void* h, const orc_lm_settings* s, double* trace, int trace_cap, int* n_trace,
                 int* its) {
  Problem& P = *as(h);
  if (!P.ready) return -1;
  return lm_solve(P, *s, trace, trace_cap, n_trace, its);
}

int orc_gn_solve(void* h, const orc_gn_settings* s, double* trace, int trace_cap, int* n_trace,
                 int* its) {
  Problem& P = *as(h);
  if (!P.ready) return -1;
  return gn_solve(P, *s, trace, trace_cap, n_trace, its);
}

int orc_dense_cholesky(double* A, int n, int lda, int num_threads) {
#ifdef _OPENMP
  if (num_threads <= 0) num_threads = omp_get_max_threads();
#endif
  return chol_blocked(A, n, lda, num_threads) ? 1 : 0;
}

}  // extern "C"

// A DoubleSection with user-defined edges written as CUDA code: the
// DeviceEdgeSection of include/nelson_b200/nelson.hpp subclassed the way a
// reference user subclasses DoubleSection with EdgeBinary / EdgeUnary edges.
//
// U blocks: 3D sensor positions x_u; V blocks: 3D points p_v.
//   U-V edge (2 residuals): |x_u - p_v| - d,  a . (x_u - p_v) - e
//   U unary (3): w (x_u - prior_u);  V unary (3): w (p_v - prior_v)
//   U-U edge (3): x_a - x_b - delta
// Measurements are exact, so the optimum is the truth with chi2 = 0: LM and
// GN, natural and AMD order, must reach chi2 < 1e-12 and the true parameters.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "nelson_b200/nelson.hpp"

using nelson_b200::DeviceEdgeSection;

namespace {

struct EdgeData {
  int kind, a, b;
  long long ro, jo;
  double d, e, w;
  double v[3];  // unit direction (U-V), prior (unary) or delta (U-U)
};

__global__ void range_edges_kernel(const EdgeData* __restrict__ ed, int ne, const double* __restrict__ x,
                                   const double* __restrict__ p, int jac, double* __restrict__ r,
                                   double* __restrict__ J) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const EdgeData E = ed[k];
  double* rr = r + E.ro;
  double* jj = J + E.jo;
  if (E.kind == NL_EDGE_UV) {
    double diff[3];
    for (int i = 0; i < 3; i++) diff[i] = x[3 * E.a + i] - p[3 * E.b + i];
    const double n = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
    rr[0] = n - E.d;
    rr[1] = E.v[0] * diff[0] + E.v[1] * diff[1] + E.v[2] * diff[2] - E.e;
    if (jac)
      for (int i = 0; i < 3; i++) {
        jj[i] = diff[i] / n;  // J_a row 0
        jj[3 + i] = E.v[i];   // J_a row 1
        jj[6 + i] = -diff[i] / n;
        jj[9 + i] = -E.v[i];
      }
  } else if (E.kind == NL_EDGE_UU) {
    for (int i = 0; i < 3; i++) rr[i] = x[3 * E.a + i] - x[3 * E.b + i] - E.v[i];
    if (jac)
      for (int i = 0; i < 9; i++) {
        jj[i] = (i % 4 == 0) ? 1.0 : 0.0;
        jj[9 + i] = (i % 4 == 0) ? -1.0 : 0.0;
      }
  } else {
    const double* q = E.kind == NL_EDGE_U ? x : p;
    for (int i = 0; i < 3; i++) rr[i] = E.w * (q[3 * E.a + i] - E.v[i]);
    if (jac)
      for (int i = 0; i < 9; i++) jj[i] = (i % 4 == 0) ? E.w : 0.0;
  }
}

__global__ void add_kernel(double* __restrict__ x, const double* __restrict__ d, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

struct Scene {
  int nu = 0, nv = 0;
  std::vector<double> x, p, x0, p0;
  std::vector<EdgeData> edges;
};

Scene make_scene(int nu, int nv, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(-10.0, 10.0);
  std::normal_distribution<double> g(0.0, 1.0);
  Scene s;
  s.nu = nu;
  s.nv = nv;
  for (int i = 0; i < 3 * nu; i++) s.x.push_back(u(rng));
  for (int i = 0; i < nv; i++) s.p.insert(s.p.end(), {u(rng), u(rng), 25.0 + u(rng)});
  for (int v = 0; v < nv; v++)
    for (int t = 0; t < 3; t++) {
      EdgeData E{};
      E.kind = NL_EDGE_UV;
      E.a = (v * 7 + t * 5) % nu;
      E.b = v;
      double a[3] = {g(rng), g(rng), g(rng)}, n = 0, diff[3], dn = 0;
      for (int i = 0; i < 3; i++) n += a[i] * a[i];
      for (int i = 0; i < 3; i++) {
        E.v[i] = a[i] / std::sqrt(n);
        diff[i] = s.x[3 * E.a + i] - s.p[3 * v + i];
        dn += diff[i] * diff[i];
      }
      E.d = std::sqrt(dn);
      E.e = E.v[0] * diff[0] + E.v[1] * diff[1] + E.v[2] * diff[2];
      s.edges.push_back(E);
    }
  for (int i = 0; i + 1 < nu; i += 3) {
    EdgeData E{};
    E.kind = NL_EDGE_UU;
    E.a = i;
    E.b = i + 1;
    for (int c = 0; c < 3; c++) E.v[c] = s.x[3 * i + c] - s.x[3 * (i + 1) + c];
    s.edges.push_back(E);
  }
  for (int i = 0; i < nu; i++) {
    EdgeData E{};
    E.kind = NL_EDGE_U;
    E.a = i;
    E.w = 0.1;
    for (int c = 0; c < 3; c++) E.v[c] = s.x[3 * i + c];
    s.edges.push_back(E);
  }
  for (int v = 0; v < nv; v += 10) {
    EdgeData E{};
    E.kind = NL_EDGE_V;
    E.a = v;
    E.w = 0.5;
    for (int c = 0; c < 3; c++) E.v[c] = s.p[3 * v + c];
    s.edges.push_back(E);
  }
  s.x0 = s.x;
  s.p0 = s.p;
  for (auto& q : s.x0) q += 0.05 * g(rng);
  for (auto& q : s.p0) q += 0.05 * g(rng);
  return s;
}

// The user's section: parameters and edge data on the device.
class RangeSection : public DeviceEdgeSection {
 public:
  RangeSection(const Scene& s, bool amd) : DeviceEdgeSection(3, s.nu, s.nv), s_(s) {
    for (const auto& E : s.edges) addEdge(E.kind, E.a, E.kind == NL_EDGE_UV || E.kind == NL_EDGE_UU ? E.b : -1,
                                          E.kind == NL_EDGE_UV ? 2 : 3);
    if (amd) permuteAMD_SchurU();
    structureReady();
    std::vector<EdgeData> ed = s.edges;
    for (size_t k = 0; k < ed.size(); k++) {
      ed[k].ro = rOffsets()[k];
      ed[k].jo = jOffsets()[k];
    }
    ne_ = (int)ed.size();
    cudaMalloc(&ed_, sizeof(EdgeData) * ed.size());
    cudaMemcpy(ed_, ed.data(), sizeof(EdgeData) * ed.size(), cudaMemcpyHostToDevice);
    for (double** q : {&x_, &xb_}) cudaMalloc(q, sizeof(double) * s.x0.size());
    for (double** q : {&p_, &pb_}) cudaMalloc(q, sizeof(double) * s.p0.size());
    cudaMemcpy(x_, s.x0.data(), sizeof(double) * s.x0.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p_, s.p0.data(), sizeof(double) * s.p0.size(), cudaMemcpyHostToDevice);
  }
  ~RangeSection() override {
    for (void* q : {(void*)ed_, (void*)x_, (void*)xb_, (void*)p_, (void*)pb_}) cudaFree(q);
  }
  double maxError() const {
    std::vector<double> x(s_.x.size()), p(s_.p.size());
    cudaMemcpy(x.data(), x_, sizeof(double) * x.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(p.data(), p_, sizeof(double) * p.size(), cudaMemcpyDeviceToHost);
    double e = 0;
    for (size_t i = 0; i < x.size(); i++) e = std::max(e, std::fabs(x[i] - s_.x[i]));
    for (size_t i = 0; i < p.size(); i++) e = std::max(e, std::fabs(p[i] - s_.p[i]));
    return e;
  }

 protected:
  int evaluate(void* stream, bool jacobians, double* r, double* J) override {
    range_edges_kernel<<<(ne_ + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ed_, ne_, x_, p_, jacobians ? 1 : 0, r,
                                                                             J);
    return cudaGetLastError() != cudaSuccess;
  }
  int oplus(void* stream, const double* du, const double* dv) override {
    const int nx = 3 * s_.nu, np = 3 * s_.nv;
    add_kernel<<<(nx + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x_, du, nx);
    add_kernel<<<(np + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p_, dv, np);
    return cudaGetLastError() != cudaSuccess;
  }
  int backupSolution(void* stream) override {
    cudaMemcpyAsync(xb_, x_, sizeof(double) * 3 * s_.nu, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    cudaMemcpyAsync(pb_, p_, sizeof(double) * 3 * s_.nv, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    return cudaGetLastError() != cudaSuccess;
  }
  int rollbackSolution(void* stream) override {
    cudaMemcpyAsync(x_, xb_, sizeof(double) * 3 * s_.nu, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    cudaMemcpyAsync(p_, pb_, sizeof(double) * 3 * s_.nv, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    return cudaGetLastError() != cudaSuccess;
  }

 private:
  const Scene& s_;
  int ne_ = 0;
  EdgeData* ed_ = nullptr;
  double *x_ = nullptr, *xb_ = nullptr, *p_ = nullptr, *pb_ = nullptr;
};

int failures = 0;
void expect(bool ok, const char* what, double a, double b) {
  std::printf("%s %-52s %.6e %.6e\n", ok ? "ok  " : "FAIL", what, a, b);
  if (!ok) failures++;
}

}  // namespace

int main() {
  const Scene s = make_scene(24, 240, 5);
  try {
    for (int amd = 0; amd < 2; amd++)
      for (int gn = 0; gn < 2; gn++) {
        RangeSection sec(s, amd != 0);
        const double c0 = sec.update(true);
        std::vector<nelson_b200::IterationRecord> tr;
        nelson_b200::LevenbergMarquardtSettings lm;
        nelson_b200::GaussNewtonSettings g;
        g.maxNumIt = 20;
        const auto reason = gn ? sec.solveGN(g, &tr) : sec.solveLM(lm, &tr);
        const double c1 = sec.update(true);
        std::printf("%s %s: reason %d, %zu records, chi2 %.3e -> %.3e\n", amd ? "amd" : "natural", gn ? "GN" : "LM",
                    int(reason), tr.size(), c0, c1);
        expect(c0 > 1.0 && c1 < 1e-12, "user-edge section chi2 below 1e-12", c0, c1);
        expect(sec.maxError() < 1e-7, "user-edge section reaches the true parameters", sec.maxError(), 1e-7);
      }
  } catch (const nelson_b200::Error& e) {
    std::printf("FAIL exception: %s\n", e.what());
    return 2;
  }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}

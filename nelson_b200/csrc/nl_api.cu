// nl_api.cu -- the C ABI of include/nelson_b200.h: device-resident BA section
// (DoubleSection), SolverCholeskySchur core, and LM / GN drivers.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

#include "ba_kernels.cuh"
#include "adjoint.cuh"
#include "problem_view.h"
#include "schur_core.cuh"
#include "unroll.cuh"

using namespace nl;

namespace {

constexpr int kCostNT = 256;
constexpr int kCostCTAs = 592;  // 4 x 148 SMs, fixed -> fixed summation order
constexpr int kCamNT = 128;
// refinement sweeps of the mixed handle's step adjoints u = A^-1 a in the
// unrolled reverse pass (each sweep divides the error by about the FP32
// factor's relative error times the condition of A)
constexpr int kUnrollRefineSweeps = 3;

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace

// ===========================================================================
struct nl_problem {
  nl_problem_desc desc{};
  int device = 0;
  int timing_detail = 0;
  cudaStream_t st = nullptr;
  cublasHandle_t cublas = nullptr;
  DevBuf cublas_ws;
  bool ready = false;
  // host copies
  std::vector<double> cam_state;  // nc_all x 16
  std::vector<double> pts;        // np_all x 3
  std::vector<int> e_cam, e_camfix, e_pt, e_ptfix;
  std::vector<double> e_obs, e_w;
  std::vector<int> perm;  // user -> internal
  // structure
  int nU = 0, nV = 0, nW = 0, nci = 0, ngrp = 0;
  std::vector<int> u_rc, v_rc, w_rc, h11, h12, h22;
  std::vector<int> eorder;   // device E-order -> insertion index
  std::vector<int> porder;   // device P-order -> insertion index
  // device
  DevBuf cam, pt, cam_bck, pt_bck;
  DevBuf d_e_cam, d_e_pt, d_e_obs, d_e_w, d_cam_grp_ptr, d_grp_edge_ptr, d_grp_wuid, d_cam_uid, d_cam_slot;
  DevBuf d_pt_edge_ptr, d_p_cam, d_p_obs, d_p_w, d_pt_vuid;
  DevBuf d_part, d_scal, d_lm, d_trace;
  DevBuf d_eorder, d_porder, stage_cams, stage_obs, stage_w;  // parameter / observation exchange
  std::unique_ptr<SchurCore> core;
  BaDev ba{};
  // scalars on the device: [0] chi2, [1] maxAbsB, [2] maxAbsHDiag, [3] rho
  double* scal = nullptr;
  LmDev* lm = nullptr;
  int* status = nullptr;  // solver status (inside LmDev)
  double* host_pin = nullptr;
  double lam_host[2] = {0, 0};
  DevBuf d_lam;
  long long launches = 0;
  DevBuf adj_vec, adj_slot2int, adj_out;  // adjoint work (allocated on first nl_adjoint)
  DevBuf unr_ckpt, unr_work;               // unrolled steps: per-step checkpoints, backward work
  std::vector<double> unr_mu;              // damping of the recorded steps
  int unr_n = -1;                          // recorded steps (-1: none)
  cudaGraphExec_t sub_exec = nullptr;       // captured LM sub-iteration without trace (batched solves)
  cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
  float eval_ms = 0;
  int have_jac = 0;

  ~nl_problem() {
    if (sub_exec) cudaGraphExecDestroy(sub_exec);
    if (cublas) cublasDestroy(cublas);
    if (host_pin) cudaFreeHost(host_pin);
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
    if (ev_t0) cudaEventDestroy(ev_t0);
    if (ev_t1) cudaEventDestroy(ev_t1);
    core.reset();
    if (st) cudaStreamDestroy(st);
  }
  int nc_all() const { return desc.nc_var + desc.nc_fix; }
  int np_all() const { return desc.np_var + desc.np_fix; }
};

namespace {

nl_status select_device(nl_problem* h) {
  NL_CUDA(cudaSetDevice(h->device));
  return NL_OK;
}

// ---------------------------------------------------------------------------
// structureReady for BA edges (nelson/DoubleSection.hpp:83-246): U, V blocks
// on the diagonal of every camera / point with an edge; W blocks on the
// distinct (internal camera, point) pairs; UIDs in CSC (U, V) / CSR (W) order.
nl_status build_structure(nl_problem* h) {
  const int ne = (int)h->e_cam.size();
  const int ncv = h->desc.nc_var, npv = h->desc.np_var, bc = h->desc.bc;
  h->nci = ncv;
  std::vector<int> has_u(ncv, 0), has_v(npv, 0);
  for (int e = 0; e < ne; e++) {
    if (!h->e_camfix[e]) has_u[h->perm[h->e_cam[e]]] = 1;
    if (!h->e_ptfix[e]) has_v[h->e_pt[e]] = 1;
  }
  std::vector<int> u_uid(ncv, -1), v_uid(npv, -1);
  int q = 0;
  for (int c = 0; c < ncv; c++)
    if (has_u[c]) u_uid[c] = q++;
  h->nU = q;
  q = 0;
  for (int p = 0; p < npv; p++)
    if (has_v[p]) v_uid[p] = q++;
  h->nV = q;
  // E-order: variable-camera edges sorted by (internal cam, fixed point last,
  // point id, insertion); fixed-camera edges after.
  std::vector<int> ord(ne);
  std::iota(ord.begin(), ord.end(), 0);
  auto key = [&](int e) -> long long {
    if (h->e_camfix[e]) return (long long)(ncv + 1) << 32;
    const long long c = h->perm[h->e_cam[e]];
    const long long p = h->e_ptfix[e] ? (long long)npv + h->e_pt[e] : h->e_pt[e];
    return (c << 32) | p;
  };
  std::vector<long long> keys(ne);
  for (int e = 0; e < ne; e++) keys[e] = key(e);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return keys[a] < keys[b]; });
  h->eorder = ord;
  // groups + W uids
  std::vector<int> cam_grp_ptr(ncv + 1, 0), grp_edge_ptr(1, 0), grp_wuid;
  h->h11.assign(ne, -1);
  h->h12.assign(ne, -1);
  h->h22.assign(ne, -1);
  h->w_rc.clear();
  int wq = 0;
  for (int t = 0; t < ne;) {
    const int e = ord[t];
    if (h->e_camfix[e]) break;  // fixed-camera edges close the E-order
    const int c = h->perm[h->e_cam[e]];
    int t1 = t + 1;
    if (!h->e_ptfix[e])
      while (t1 < ne && keys[ord[t1]] == keys[e]) t1++;
    int wuid = -1;
    if (!h->e_ptfix[e]) {
      wuid = wq++;
      h->w_rc.push_back(c);
      h->w_rc.push_back(h->e_pt[e]);
    }
    for (int s = t; s < t1; s++) h->h12[ord[s]] = wuid;
    grp_wuid.push_back(wuid);
    grp_edge_ptr.push_back(t1);
    cam_grp_ptr[c + 1]++;
    t = t1;
  }
  for (int c = 0; c < ncv; c++) cam_grp_ptr[c + 1] += cam_grp_ptr[c];
  h->nW = wq;
  h->ngrp = (int)grp_wuid.size();
  for (int e = 0; e < ne; e++) {
    if (!h->e_camfix[e]) h->h11[e] = u_uid[h->perm[h->e_cam[e]]];
    if (!h->e_ptfix[e]) h->h22[e] = v_uid[h->e_pt[e]];
  }
  h->u_rc.clear();
  for (int c = 0; c < ncv; c++)
    if (u_uid[c] >= 0) {
      h->u_rc.push_back(c);
      h->u_rc.push_back(c);
    }
  h->v_rc.clear();
  for (int p = 0; p < npv; p++)
    if (v_uid[p] >= 0) {
      h->v_rc.push_back(p);
      h->v_rc.push_back(p);
    }
  // P-order: variable-point edges by (point, insertion)
  std::vector<int> pord;
  pord.reserve(ne);
  for (int e = 0; e < ne; e++)
    if (!h->e_ptfix[e]) pord.push_back(e);
  std::stable_sort(pord.begin(), pord.end(), [&](int a, int b) { return h->e_pt[a] < h->e_pt[b]; });
  h->porder = pord;
  std::vector<int> pt_edge_ptr(npv + 1, 0);
  for (int e : pord) pt_edge_ptr[h->e_pt[e] + 1]++;
  for (int p = 0; p < npv; p++) pt_edge_ptr[p + 1] += pt_edge_ptr[p];
  // device edge arrays
  const int ncv_ = ncv;
  auto cam_slot = [&](int e) { return h->e_camfix[e] ? ncv_ + h->e_cam[e] : h->e_cam[e]; };
  auto pt_slot = [&](int e) { return h->e_ptfix[e] ? npv + h->e_pt[e] : h->e_pt[e]; };
  std::vector<int> ecam(ne), ept(ne), pcam(pord.size());
  std::vector<double> eobs(2 * (size_t)ne), ew(ne), pobs(2 * pord.size()), pw(pord.size());
  for (int t = 0; t < ne; t++) {
    const int e = ord[t];
    ecam[t] = cam_slot(e);
    ept[t] = pt_slot(e);
    eobs[2 * t] = h->e_obs[2 * (size_t)e];
    eobs[2 * t + 1] = h->e_obs[2 * (size_t)e + 1];
    ew[t] = h->e_w[e];
  }
  for (size_t t = 0; t < pord.size(); t++) {
    const int e = pord[t];
    pcam[t] = cam_slot(e);
    pobs[2 * t] = h->e_obs[2 * (size_t)e];
    pobs[2 * t + 1] = h->e_obs[2 * (size_t)e + 1];
    pw[t] = h->e_w[e];
  }
  std::vector<int> slot_of_internal(ncv);
  for (int u = 0; u < ncv; u++) slot_of_internal[h->perm[u]] = u;
  nl_status s;
#define NL_TRY(x)             \
  do {                        \
    if ((s = (x)) != NL_OK) { \
      return s;               \
    }                         \
  } while (0)
  NL_TRY(upload(h->d_e_cam, ecam, h->st));
  NL_TRY(upload(h->d_e_pt, ept, h->st));
  NL_TRY(upload(h->d_e_obs, eobs, h->st));
  NL_TRY(upload(h->d_e_w, ew, h->st));
  NL_TRY(upload(h->d_cam_grp_ptr, cam_grp_ptr, h->st));
  NL_TRY(upload(h->d_grp_edge_ptr, grp_edge_ptr, h->st));
  NL_TRY(upload(h->d_grp_wuid, grp_wuid, h->st));
  NL_TRY(upload(h->d_cam_uid, u_uid, h->st));
  NL_TRY(upload(h->d_cam_slot, slot_of_internal, h->st));
  NL_TRY(upload(h->d_pt_edge_ptr, pt_edge_ptr, h->st));
  NL_TRY(upload(h->d_p_cam, pcam, h->st));
  NL_TRY(upload(h->d_p_obs, pobs, h->st));
  NL_TRY(upload(h->d_p_w, pw, h->st));
  NL_TRY(upload(h->d_pt_vuid, v_uid, h->st));
  NL_TRY(upload(h->d_eorder, ord, h->st));
  NL_TRY(upload(h->d_porder, pord, h->st));
  NL_TRY(upload(h->stage_obs, h->e_obs, h->st));
  NL_TRY(upload(h->stage_w, h->e_w, h->st));
  // Schur core
  SchurStructure ss;
  ss.bc = bc;
  ss.nci = ncv;
  ss.np = npv;
  for (size_t i = 0; i < h->u_rc.size(); i += 2) {
    ss.u_r.push_back(h->u_rc[i]);
    ss.u_c.push_back(h->u_rc[i + 1]);
  }
  ss.v_uid = v_uid;
  for (size_t i = 0; i < h->w_rc.size(); i += 2) {
    ss.w_r.push_back(h->w_rc[i]);
    ss.w_c.push_back(h->w_rc[i + 1]);
  }
  NL_TRY(h->core->setup(ss, h->st));
  BaDev& d = h->ba;
  d.bc = bc;
  d.nci = ncv;
  d.nc_all = h->nc_all();
  d.np_var = npv;
  d.np_all = h->np_all();
  d.ne = ne;
  d.ngrp = h->ngrp;
  d.f_fixed = h->desc.f;
  d.cx = h->desc.cx;
  d.cy = h->desc.cy;
  d.cam = h->cam.as<double>();
  d.pt = h->pt.as<double>();
  d.e_cam = h->d_e_cam.as<int>();
  d.e_pt = h->d_e_pt.as<int>();
  d.e_obs = h->d_e_obs.as<double>();
  d.e_w = h->d_e_w.as<double>();
  d.cam_grp_ptr = h->d_cam_grp_ptr.as<int>();
  d.grp_edge_ptr = h->d_grp_edge_ptr.as<int>();
  d.grp_wuid = h->d_grp_wuid.as<int>();
  d.cam_uid = h->d_cam_uid.as<int>();
  d.cam_slot = h->d_cam_slot.as<int>();
  d.pt_edge_ptr = h->d_pt_edge_ptr.as<int>();
  d.p_cam = h->d_p_cam.as<int>();
  d.p_obs = h->d_p_obs.as<double>();
  d.p_w = h->d_p_w.as<double>();
  d.pt_vuid = h->d_pt_vuid.as<int>();
#undef NL_TRY
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

// ---------------------------------------------------------------------------
// update(hessian): cost always (FP64), Hessian blocks when asked.
template <typename T, int BC>
nl_status enqueue_eval_t(nl_problem* h, bool hessian, double* chi2_out, double* maxb_out, const int* active) {
  cost_kernel<BC, kCostNT><<<kCostCTAs, kCostNT, 0, h->st>>>(h->ba, h->d_part.as<double>(), active);
  sum_partials_kernel<256><<<1, 256, 0, h->st>>>(h->d_part.as<double>(), kCostCTAs, chi2_out, active);
  h->launches += 2;
  if (hessian) {
    if (h->nci > 0)
      cam_pass_kernel<T, BC, kCamNT><<<h->nci, kCamNT, 0, h->st>>>(h->ba, (T*)h->core->dU(), (T*)h->core->dW(),
                                                                   (T*)h->core->dbU(), active);
    if (h->desc.np_var > 0)
      pt_pass_kernel<T, BC, 128><<<cdiv(h->desc.np_var, 128), 128, 0, h->st>>>(h->ba, (T*)h->core->dV(),
                                                                                (T*)h->core->dbV(), active);
    h->launches += 2;
    nl_status s = h->core->enqueue_maxabs_b(maxb_out, active);
    if (s != NL_OK) return s;
  }
  NL_CUDA(cudaGetLastError());
  return NL_OK;
}

nl_status enqueue_eval(nl_problem* h, bool hessian, double* chi2_out, double* maxb_out, const int* active) {
  NvtxRange rg(hessian ? "nl:update(true)" : "nl:update(false)");
  const bool f64 = h->desc.precision == NL_PREC_FP64;
  if (h->desc.bc == 9)
    return f64 ? enqueue_eval_t<double, 9>(h, hessian, chi2_out, maxb_out, active)
               : enqueue_eval_t<float, 9>(h, hessian, chi2_out, maxb_out, active);
  return f64 ? enqueue_eval_t<double, 6>(h, hessian, chi2_out, maxb_out, active)
             : enqueue_eval_t<float, 6>(h, hessian, chi2_out, maxb_out, active);
}

nl_status enqueue_oplus(nl_problem* h, const int* active) {
  const int nci = h->nci;
  if (nci > 0) {
    if (h->desc.bc == 9)
      oplus_cam_kernel<9><<<cdiv(nci, 128), 128, 0, h->st>>>(h->cam.as<double>(), h->ba.cam_slot, nci,
                                                              h->core->incU, active);
    else
      oplus_cam_kernel<6><<<cdiv(nci, 128), 128, 0, h->st>>>(h->cam.as<double>(), h->ba.cam_slot, nci,
                                                              h->core->incU, active);
  }
  if (h->desc.np_var > 0)
    oplus_pt_kernel<<<cdiv(3LL * h->desc.np_var, 256), 256, 0, h->st>>>(h->pt.as<double>(), h->desc.np_var,
                                                                         h->core->incV, active);
  h->launches += 2;
  NL_CUDA(cudaGetLastError());
  return NL_OK;
}

nl_status enqueue_copy_params(nl_problem* h, bool to_backup, const int* flag) {
  const size_t nc = (size_t)h->nc_all() * 16, np = (size_t)h->np_all() * 3;
  double* c_dst = to_backup ? h->cam_bck.as<double>() : h->cam.as<double>();
  const double* c_src = to_backup ? h->cam.as<double>() : h->cam_bck.as<double>();
  double* p_dst = to_backup ? h->pt_bck.as<double>() : h->pt.as<double>();
  const double* p_src = to_backup ? h->pt.as<double>() : h->pt_bck.as<double>();
  copy_if_kernel<<<std::max(1, std::min(296, cdiv(nc, 256))), 256, 0, h->st>>>(c_dst, c_src, nc, flag);
  copy_if_kernel<<<std::max(1, std::min(296, cdiv(np, 256))), 256, 0, h->st>>>(p_dst, p_src, np, flag);
  h->launches += 2;
  NL_CUDA(cudaGetLastError());
  return NL_OK;
}

// One sub-iteration of LM / one iteration of GN (see lm_kernels.cuh).
nl_status enqueue_subiteration(nl_problem* h, double* trace) {
  LmDev* s = h->lm;
  lm_begin_kernel<<<1, 1, 0, h->st>>>(s);
  nl_status r = h->core->enqueue_increment(s->lam, &s->status, &s->active);
  if (r != NL_OK) return r;
  int nparts = 0;
  if ((r = h->core->enqueue_inc_dot(s, h->d_part.as<double>() + 4096, &nparts)) != NL_OK) return r;
  lm_inc_kernel<<<1, 1, 0, h->st>>>(s, h->d_part.as<double>() + 4096, nparts, trace);
  if ((r = enqueue_oplus(h, &s->apply)) != NL_OK) return r;
  if ((r = enqueue_eval(h, false, &s->chi2_new, nullptr, &s->apply)) != NL_OK) return r;
  lm_decide_kernel<<<1, 1, 0, h->st>>>(s, trace);
  if ((r = enqueue_copy_params(h, false, &s->rollback)) != NL_OK) return r;
  // update(true) at the accepted point (GN: after every step), then backup
  if ((r = enqueue_eval(h, true, h->scal, &s->maxAbsB, &s->do_jac)) != NL_OK) return r;
  if ((r = enqueue_copy_params(h, true, &s->do_jac)) != NL_OK) return r;
  lm_after_jac_kernel<<<1, 1, 0, h->st>>>(s, h->scal, trace);
  h->launches += 4;
  NL_CUDA(cudaGetLastError());
  return NL_OK;
}

}  // namespace

// ===========================================================================
// C ABI
#define NL_CHECK_H(h)          \
  do {                         \
    if (!(h)) return NL_ERR_ARG; \
  } while (0)
#define NL_CHECK_READY(h)                    \
  do {                                       \
    if (!(h) || !(h)->ready) return NL_ERR_STATE; \
  } while (0)

namespace {

nl_status sync_read(nl_problem* h, const double* dev, double* out, int n) {
  NL_CUDA(cudaMemcpyAsync(h->host_pin, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  for (int i = 0; i < n; i++) out[i] = h->host_pin[i];
  return NL_OK;
}

nl_status upload_params(nl_problem* h) {
  NL_CUDA(cudaMemcpyAsync(h->cam.p, h->cam_state.data(), h->cam_state.size() * sizeof(double),
                          cudaMemcpyHostToDevice, h->st));
  if (!h->pts.empty())
    NL_CUDA(cudaMemcpyAsync(h->pt.p, h->pts.data(), h->pts.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

// One LM / GN sub-iteration captured as a CUDA graph on the handle's streams
// (the kernels are predicated on device flags, so the same graph serves every
// sub-iteration); `trace` is baked into the graph.
nl_status capture_subiteration(nl_problem* h, double* trace, cudaGraphExec_t* out) {
  NL_CUDA(cudaStreamSynchronize(h->st));
  NL_CUDA(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed));
  nl_status r = enqueue_subiteration(h, trace);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->st, &g);
  if (r != NL_OK) {
    if (g) cudaGraphDestroy(g);
    return r;
  }
  NL_CUDA(ce);
  const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  NL_CUDA(ie);
  return NL_OK;
}

// Solve driver shared by LM and GN (the host only relaunches the fixed
// sub-iteration sequence and watches the `done` flag one launch behind).
nl_status run_solver(nl_problem* h, LmDev& init, nl_solve_report* rep, double* trace, int trace_cap, int max_launch) {
  NL_CUDA(cudaEventRecord(h->ev_t0, h->st));
  // update(true) at the start (LevenbergMarquardt.hpp:41 / GaussNewton.hpp:40)
  nl_status r = enqueue_eval(h, true, h->scal, h->scal + 1, nullptr);
  if (r != NL_OK) return r;
  double v[2];
  if ((r = sync_read(h, h->scal, v, 2)) != NL_OK) return r;
  init.chi2 = init.oldChi2 = v[0];
  init.maxAbsB = v[1];
  const int cap = std::max(0, trace_cap);
  if (h->d_trace.bytes < sizeof(double) * NL_TRACE_STRIDE * (size_t)std::max(cap, 1))
    if ((r = h->d_trace.alloc(sizeof(double) * NL_TRACE_STRIDE * (size_t)std::max(cap, 1))) != NL_OK) return r;
  double* dtrace = cap > 0 ? h->d_trace.as<double>() : nullptr;
  init.trace_cap = cap;
  init.trace_n = 1;
  double first[NL_TRACE_STRIDE] = {-1, init.gn ? 0.0 : -1.0, v[0], 0, 0, 0, 1, 1};
  if (trace && cap > 0) memcpy(trace, first, sizeof(first));
  if (v[1] <= init.epsBVector) {
    NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
    NL_CUDA(cudaEventSynchronize(h->ev_t1));
    if (rep) {
      float ms = 0;
      cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
      rep->reason = NL_SUCCESS_AT_START;
      rep->iterations = -1;
      rep->subiterations = 0;
      rep->n_trace = cap > 0 ? 1 : 0;
      rep->chi2 = v[0];
      rep->mu = 0;
      rep->device_ms = ms;
    }
    return NL_OK;
  }
  if ((r = enqueue_copy_params(h, true, nullptr)) != NL_OK) return r;  // backupSolution
  if ((r = h->core->enqueue_hdiag(h->scal + 2)) != NL_OK) return r;
  double hd;
  if ((r = sync_read(h, h->scal + 2, &hd, 1)) != NL_OK) return r;
  init.maxAbsHDiag = hd;
  init.mu = init.tau * hd;  // LevenbergMarquardt.hpp:58
  init.curV = init.initV;
  init.iter = 0;
  init.subiter = 0;
  init.nsub = 0;
  init.done = init.gn && init.maxNumIt <= 0 ? 1 : 0;
  if (!init.gn && init.maxNumIt <= 0) init.done = 1;
  init.reason = NL_MAX_ITERATION_REACHED;
  NL_CUDA(cudaMemcpyAsync(h->lm, &init, sizeof(LmDev), cudaMemcpyHostToDevice, h->st));
  // launch loop: watch `done` one launch behind
  int* done_pin = reinterpret_cast<int*>(h->host_pin + 8);
  done_pin[0] = done_pin[1] = init.done;
  int launched = 0;
  // stream launches, not a captured graph: graph nodes do not keep the
  // streams' priorities, and the factorisation's critical path relies on them
  while (!init.done && launched < max_launch) {
    if ((r = enqueue_subiteration(h, dtrace)) != NL_OK) return r;
    NL_CUDA(cudaMemcpyAsync(done_pin + (launched & 1), &h->lm->done, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    NL_CUDA(cudaEventRecord(launched & 1 ? h->ev_b : h->ev_a, h->st));
    if (launched > 0) {
      cudaEvent_t prev = (launched & 1) ? h->ev_a : h->ev_b;
      NL_CUDA(cudaEventSynchronize(prev));
      if (done_pin[(launched - 1) & 1]) break;
    }
    launched++;
  }
  NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  float dev_ms = 0;
  cudaEventElapsedTime(&dev_ms, h->ev_t0, h->ev_t1);
  LmDev fin;
  NL_CUDA(cudaMemcpy(&fin, h->lm, sizeof(LmDev), cudaMemcpyDeviceToHost));
  const int nt = std::min(fin.trace_n, cap);
  if (trace && nt > 1)
    NL_CUDA(cudaMemcpy(trace + NL_TRACE_STRIDE, dtrace + NL_TRACE_STRIDE, sizeof(double) * NL_TRACE_STRIDE * (nt - 1),
                       cudaMemcpyDeviceToHost));
  if (rep) {
    rep->reason = fin.done ? fin.reason : NL_MAX_ITERATION_REACHED;
    rep->iterations = fin.iter;
    rep->subiterations = fin.nsub;
    rep->n_trace = nt;
    rep->chi2 = fin.chi2;
    rep->mu = fin.mu;
    rep->device_ms = dev_ms;
  }
  return NL_OK;
}

}  // namespace

extern "C" {

const char* nl_version(void) { return "nelson_b200 0.1 sm_100a"; }

const char* nl_status_string(int s) {
  switch (s) {
    case NL_OK: return "ok";
    case NL_ERR_ARG: return "bad argument";
    case NL_ERR_STATE: return "call out of order";
    case NL_ERR_CUDA: return "CUDA error";
    case NL_ERR_UNSUPPORTED: return "unsupported structure";
    case NL_ERR_NOT_SPD: return "not positive definite";
    case NL_ERR_NONFINITE: return "non-finite value";
    case NL_ERR_TIMEOUT: return "device wait timed out";
    case NL_ERR_NOMEM: return "device allocation failed";
    case NL_ERR_CALLBACK: return "a user callback failed";
    default: return "unknown status";
  }
}

nl_status nl_create(const nl_problem_desc* d, nl_problem** out) {
  if (!d || !out) return NL_ERR_ARG;
  *out = nullptr;
  if ((d->bc != 6 && d->bc != 9) || d->nc_var < 0 || d->nc_fix < 0 || d->np_var < 0 || d->np_fix < 0 ||
      (d->precision != NL_PREC_FP64 && d->precision != NL_PREC_MIXED))
    return NL_ERR_ARG;
  std::unique_ptr<nl_problem> h(new nl_problem());
  h->desc = *d;
  h->device = d->device;
  nl_status s;
  if ((s = select_device(h.get())) != NL_OK) return s;
  {
    // the main stream carries the factorisation's critical path: highest priority
    int lo = 0, hi = 0;
    NL_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    NL_CUDA(cudaStreamCreateWithPriority(&h->st, cudaStreamNonBlocking, hi));
  }
  NL_CUDA(cudaEventCreateWithFlags(&h->ev_a, cudaEventDisableTiming));
  NL_CUDA(cudaEventCreateWithFlags(&h->ev_b, cudaEventDisableTiming));
  NL_CUDA(cudaEventCreate(&h->ev_t0));
  NL_CUDA(cudaEventCreate(&h->ev_t1));
  if (d->precision == NL_PREC_FP64) {
    if (cublasCreate(&h->cublas) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
    cublasSetStream(h->cublas, h->st);
    if ((s = h->cublas_ws.alloc(64u << 20)) != NL_OK) return s;
    cublasSetWorkspace(h->cublas, h->cublas_ws.p, h->cublas_ws.bytes);
  }
  h->core = make_schur_core(d->precision, d->bc, h->cublas);
  if (!h->core) return NL_ERR_UNSUPPORTED;
  h->core->refine_sweeps = d->refine_sweeps >= 0 ? d->refine_sweeps : (d->precision == NL_PREC_MIXED ? 1 : 0);
  h->core->keep_schur = (long long)d->nc_var * d->bc <= 4096 ? 1 : 0;
  h->core->use_tc = d->precision == NL_PREC_MIXED ? 1 : 0;
  const int nc_all = d->nc_var + d->nc_fix, np_all = d->np_var + d->np_fix;
  h->cam_state.assign((size_t)nc_all * 16, 0.0);
  h->pts.assign((size_t)np_all * 3, 0.0);
  for (int c = 0; c < nc_all; c++) {
    double* st = h->cam_state.data() + (size_t)c * 16;
    st[0] = st[4] = st[8] = 1.0;
    st[11] = 1.0;
    st[12] = d->f;
  }
  h->perm.resize(d->nc_var);
  std::iota(h->perm.begin(), h->perm.end(), 0);
  if ((s = h->cam.alloc(sizeof(double) * std::max<size_t>(h->cam_state.size(), 16))) != NL_OK) return s;
  if ((s = h->cam_bck.alloc(h->cam.bytes)) != NL_OK) return s;
  if ((s = h->pt.alloc(sizeof(double) * std::max<size_t>(h->pts.size(), 3))) != NL_OK) return s;
  if ((s = h->pt_bck.alloc(h->pt.bytes)) != NL_OK) return s;
  if ((s = h->d_part.alloc(sizeof(double) * 8192)) != NL_OK) return s;
  if ((s = h->stage_cams.alloc(sizeof(double) * std::max<size_t>((size_t)nc_all * 9, 9))) != NL_OK) return s;
  if ((s = h->d_scal.alloc(sizeof(double) * 16)) != NL_OK) return s;
  if ((s = h->d_lm.alloc(sizeof(LmDev))) != NL_OK) return s;
  if ((s = h->d_lam.alloc(sizeof(double) * 2 + sizeof(int) * 2)) != NL_OK) return s;
  NL_CUDA(cudaMemsetAsync(h->d_scal.p, 0, h->d_scal.bytes, h->st));
  NL_CUDA(cudaMemsetAsync(h->d_lm.p, 0, h->d_lm.bytes, h->st));
  h->scal = h->d_scal.as<double>();
  h->lm = h->d_lm.as<LmDev>();
  h->status = reinterpret_cast<int*>(h->d_lam.as<double>() + 2);
  NL_CUDA(cudaMallocHost(&h->host_pin, 4096));
  if ((s = upload_params(h.get())) != NL_OK) return s;  // identity cameras, origin points
  *out = h.release();
  return NL_OK;
}

nl_status nl_destroy(nl_problem* h) {
  if (!h) return NL_ERR_ARG;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->st);
  delete h;
  return NL_OK;
}

nl_status nl_set_params(nl_problem* h, const double* cams, const double* pts) {
  NL_CHECK_H(h);
  NL_CUDA(cudaSetDevice(h->device));
  const int nc = h->nc_all(), bc = h->desc.bc;
  if (cams && nc > 0) {
    NL_CUDA(cudaMemcpyAsync(h->stage_cams.p, cams, sizeof(double) * (size_t)nc * bc, cudaMemcpyHostToDevice, h->st));
    cams_in_kernel<<<cdiv(nc, 128), 128, 0, h->st>>>(h->stage_cams.as<double>(), h->cam.as<double>(), nc, bc,
                                                     h->desc.f);
    h->launches++;
  }
  if (pts && h->np_all() > 0)
    NL_CUDA(cudaMemcpyAsync(h->pt.p, pts, sizeof(double) * 3 * (size_t)h->np_all(), cudaMemcpyHostToDevice, h->st));
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

nl_status nl_get_camera_state(nl_problem* h, double* states) {
  NL_CHECK_H(h);
  NL_CUDA(cudaSetDevice(h->device));
  NL_CUDA(cudaStreamSynchronize(h->st));
  NL_CUDA(cudaMemcpy(states, h->cam.p, sizeof(double) * h->cam_state.size(), cudaMemcpyDeviceToHost));
  return NL_OK;
}

nl_status nl_get_params(nl_problem* h, double* cams, double* pts) {
  NL_CHECK_H(h);
  NL_CUDA(cudaSetDevice(h->device));
  const int nc = h->nc_all(), bc = h->desc.bc;
  if (cams && nc > 0) {
    cams_out_kernel<<<cdiv(nc, 128), 128, 0, h->st>>>(h->cam.as<double>(), h->stage_cams.as<double>(), nc, bc);
    h->launches++;
    NL_CUDA(cudaMemcpyAsync(cams, h->stage_cams.p, sizeof(double) * (size_t)nc * bc, cudaMemcpyDeviceToHost, h->st));
  }
  if (pts && h->np_all() > 0)
    NL_CUDA(cudaMemcpyAsync(pts, h->pt.p, sizeof(double) * 3 * (size_t)h->np_all(), cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

nl_status nl_add_ba_edges(nl_problem* h, int ne, const int* cam, const int* cam_fixed, const int* pt,
                          const int* pt_fixed, const double* obs, const double* weight) {
  NL_CHECK_H(h);
  if (h->ready) return NL_ERR_STATE;
  if (ne < 0 || (ne > 0 && (!cam || !pt || !obs))) return NL_ERR_ARG;
  for (int e = 0; e < ne; e++) {
    const int cf = cam_fixed ? (cam_fixed[e] != 0) : 0, pf = pt_fixed ? (pt_fixed[e] != 0) : 0;
    const int lc = cf ? h->desc.nc_fix : h->desc.nc_var, lp = pf ? h->desc.np_fix : h->desc.np_var;
    if (cam[e] < 0 || cam[e] >= lc || pt[e] < 0 || pt[e] >= lp) return NL_ERR_ARG;
    if (weight && !(weight[e] >= 0.0)) return NL_ERR_ARG;
  }
  for (int e = 0; e < ne; e++) {
    h->e_cam.push_back(cam[e]);
    h->e_camfix.push_back(cam_fixed ? (cam_fixed[e] != 0) : 0);
    h->e_pt.push_back(pt[e]);
    h->e_ptfix.push_back(pt_fixed ? (pt_fixed[e] != 0) : 0);
    h->e_obs.push_back(obs[2 * (size_t)e]);
    h->e_obs.push_back(obs[2 * (size_t)e + 1]);
    h->e_w.push_back(weight ? weight[e] : 1.0);
  }
  return NL_OK;
}

nl_status nl_set_user2internal_u(nl_problem* h, const int* perm) {
  NL_CHECK_H(h);
  if (h->ready) return NL_ERR_STATE;
  if (!perm) return NL_ERR_ARG;
  std::vector<int> seen(h->desc.nc_var, 0);
  for (int i = 0; i < h->desc.nc_var; i++) {
    if (perm[i] < 0 || perm[i] >= h->desc.nc_var || seen[perm[i]]) return NL_ERR_ARG;
    seen[perm[i]] = 1;
  }
  memcpy(h->perm.data(), perm, sizeof(int) * h->desc.nc_var);
  return NL_OK;
}

nl_status nl_get_user2internal_u(nl_problem* h, int* perm) {
  NL_CHECK_H(h);
  if (!perm) return NL_ERR_ARG;
  memcpy(perm, h->perm.data(), sizeof(int) * h->desc.nc_var);
  return NL_OK;
}

nl_status nl_rcm_order(int nc, int np, int ne, const int* cam, const int* pt, int* perm) {
  if (nc < 0 || np < 0 || ne < 0 || !perm || (ne > 0 && (!cam || !pt))) return NL_ERR_ARG;
  for (int e = 0; e < ne; e++)
    if (cam[e] < 0 || cam[e] >= nc || pt[e] < 0 || pt[e] >= np) return NL_ERR_ARG;
  if (nc == 0) return NL_OK;
  // camera graph: cameras that observe a common point
  std::vector<std::vector<int>> by_pt(np);
  for (int e = 0; e < ne; e++) by_pt[pt[e]].push_back(cam[e]);
  std::vector<std::vector<int>> adj(nc);
  for (auto& cams : by_pt)
    for (size_t a = 0; a < cams.size(); a++)
      for (size_t b = 0; b < cams.size(); b++)
        if (cams[a] != cams[b]) adj[cams[a]].push_back(cams[b]);
  std::vector<int> deg(nc);
  for (int c = 0; c < nc; c++) {
    std::sort(adj[c].begin(), adj[c].end());
    adj[c].erase(std::unique(adj[c].begin(), adj[c].end()), adj[c].end());
    deg[c] = (int)adj[c].size();
  }
  for (int c = 0; c < nc; c++)
    std::sort(adj[c].begin(), adj[c].end(), [&](int x, int y) { return deg[x] != deg[y] ? deg[x] < deg[y] : x < y; });
  // breadth-first levels from r, neighbours in increasing degree
  std::vector<int> level(nc, -1), order;
  order.reserve(nc);
  auto bfs = [&](int r, std::vector<int>& out) {
    out.clear();
    level[r] = 0;
    out.push_back(r);
    for (size_t q = 0; q < out.size(); q++)
      for (int n : adj[out[q]])
        if (level[n] < 0) {
          level[n] = level[out[q]] + 1;
          out.push_back(n);
        }
  };
  std::vector<char> done(nc, 0);
  std::vector<int> comp, c2;
  for (int s0 = 0; s0 < nc; s0++) {
    if (done[s0]) continue;
    // pseudo-peripheral start: the lowest-degree vertex of the last level,
    // repeated while the eccentricity grows (George-Liu)
    int r = s0;
    bfs(r, comp);
    for (int it = 0; it < 8; it++) {
      const int ecc = level[comp.back()];
      int best = comp.back();
      for (int v : comp)
        if (level[v] == ecc && deg[v] < deg[best]) best = v;
      for (int v : comp) level[v] = -1;
      bfs(best, c2);
      const bool grew = level[c2.back()] > ecc;
      for (int v : c2) level[v] = -1;
      if (!grew) break;
      r = best;
      bfs(r, comp);
    }
    for (int v : comp) level[v] = -1;
    bfs(r, comp);  // Cuthill-McKee order of this component
    for (int v : comp) {
      done[v] = 1;
      order.push_back(v);
    }
  }
  // reversed: internal position i holds camera order[nc - 1 - i]
  for (int i = 0; i < nc; i++) perm[order[nc - 1 - i]] = i;
  return NL_OK;
}

nl_status nl_permute_rcm_u(nl_problem* h) {
  NL_CHECK_H(h);
  if (h->ready) return NL_ERR_STATE;
  // the edges between variable cameras and variable points
  std::vector<int> cam, pt;
  for (size_t e = 0; e < h->e_cam.size(); e++)
    if (!h->e_camfix[e] && !h->e_ptfix[e]) {
      cam.push_back(h->e_cam[e]);
      pt.push_back(h->e_pt[e]);
    }
  return nl_rcm_order(h->desc.nc_var, h->desc.np_var, (int)cam.size(), cam.data(), pt.data(), h->perm.data());
}

nl_status nl_permute_amd_u(nl_problem* h) {
  NL_CHECK_H(h);
  if (h->ready) return NL_ERR_STATE;
  std::vector<int> cam, pt;
  for (size_t e = 0; e < h->e_cam.size(); e++)
    if (!h->e_camfix[e] && !h->e_ptfix[e]) {
      cam.push_back(h->e_cam[e]);
      pt.push_back(h->e_pt[e]);
    }
  return nl_amd_order_camera_graph(h->desc.nc_var, h->desc.np_var, (int)cam.size(), cam.data(), pt.data(),
                                   h->perm.data());
}

nl_status nl_structure_ready(nl_problem* h) {
  NL_CHECK_H(h);
  if (h->ready) return NL_ERR_STATE;
  NL_CUDA(cudaSetDevice(h->device));
  nl_status s = build_structure(h);
  if (s != NL_OK) return s;
  h->ready = true;
  return NL_OK;
}

nl_status nl_set_observations(nl_problem* h, const double* obs, const double* weight) {
  NL_CHECK_READY(h);
  const int ne = (int)h->e_cam.size(), npo = (int)h->porder.size();
  if (ne == 0) return NL_OK;
  NL_CUDA(cudaSetDevice(h->device));
  if (obs) NL_CUDA(cudaMemcpyAsync(h->stage_obs.p, obs, sizeof(double) * 2 * (size_t)ne, cudaMemcpyHostToDevice, h->st));
  if (weight) NL_CUDA(cudaMemcpyAsync(h->stage_w.p, weight, sizeof(double) * (size_t)ne, cudaMemcpyHostToDevice, h->st));
  if (obs || weight) {
    // unchanged halves keep their previous values: gather both from staging,
    // which holds the last uploaded observations / weights
    gather_obs_kernel<<<cdiv(ne, 256), 256, 0, h->st>>>(h->stage_obs.as<double>(), h->stage_w.as<double>(),
                                                        h->d_eorder.as<int>(), ne, h->d_e_obs.as<double>(),
                                                        h->d_e_w.as<double>());
    if (npo > 0)
      gather_obs_kernel<<<cdiv(npo, 256), 256, 0, h->st>>>(h->stage_obs.as<double>(), h->stage_w.as<double>(),
                                                           h->d_porder.as<int>(), npo, h->d_p_obs.as<double>(),
                                                           h->d_p_w.as<double>());
    h->launches += 2;
  }
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

nl_status nl_get_counts(nl_problem* h, int* counts) {
  NL_CHECK_READY(h);
  counts[0] = h->nU;
  counts[1] = h->nV;
  counts[2] = h->nW;
  counts[3] = (int)h->e_cam.size();
  return NL_OK;
}

nl_status nl_get_patterns(nl_problem* h, int* u_rc, int* v_rc, int* w_rc) {
  NL_CHECK_READY(h);
  if (u_rc) memcpy(u_rc, h->u_rc.data(), sizeof(int) * h->u_rc.size());
  if (v_rc) memcpy(v_rc, h->v_rc.data(), sizeof(int) * h->v_rc.size());
  if (w_rc) memcpy(w_rc, h->w_rc.data(), sizeof(int) * h->w_rc.size());
  return NL_OK;
}

nl_status nl_get_edge_uids(nl_problem* h, int* h11, int* h12, int* h22) {
  NL_CHECK_READY(h);
  if (h11) memcpy(h11, h->h11.data(), sizeof(int) * h->h11.size());
  if (h12) memcpy(h12, h->h12.data(), sizeof(int) * h->h12.size());
  if (h22) memcpy(h22, h->h22.data(), sizeof(int) * h->h22.size());
  return NL_OK;
}

nl_status nl_update(nl_problem* h, int hessian, double* chi2) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  NL_CUDA(cudaEventRecord(h->ev_t0, h->st));
  nl_status s = enqueue_eval(h, hessian != 0, h->scal, h->scal + 1, nullptr);
  if (s != NL_OK) return s;
  NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
  double v;
  if ((s = sync_read(h, h->scal, &v, 1)) != NL_OK) return s;
  if (hessian) NL_CUDA(cudaEventElapsedTime(&h->eval_ms, h->ev_t0, h->ev_t1));
  if (chi2) *chi2 = v;
  return NL_OK;
}

nl_status nl_get_hessian(nl_problem* h, double* U, double* V, double* W, double* bU, double* bV) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  return h->core->get_hessian(U, V, W, bU, bV);
}

nl_status nl_solver_init(nl_problem* h) {
  NL_CHECK_READY(h);
  return NL_OK;
}

nl_status nl_max_abs_hdiag(nl_problem* h, double* out) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  nl_status s = h->core->enqueue_hdiag(h->scal + 2);
  if (s != NL_OK) return s;
  return sync_read(h, h->scal + 2, out, 1);
}

nl_status nl_compute_increment(nl_problem* h, double rel, double abs_, int* ok) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  double lam[2] = {rel, abs_};
  memcpy(h->host_pin + 16, lam, sizeof(lam));
  NL_CUDA(cudaMemcpyAsync(h->d_lam.p, h->host_pin + 16, sizeof(lam), cudaMemcpyHostToDevice, h->st));
  NL_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
  h->core->timing = 1;
  h->core->timing_detail = h->timing_detail;
  nl_status s = h->core->enqueue_increment(h->d_lam.as<double>(), h->status, nullptr);
  h->core->timing = 0;
  if (s != NL_OK) return s;
  int st = 0;
  NL_CUDA(cudaMemcpyAsync(h->host_pin + 20, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  memcpy(&st, h->host_pin + 20, sizeof(int));
  if (ok) *ok = st == 0 ? 1 : 0;
  if (st & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  return NL_OK;
}

nl_status nl_get_increment(nl_problem* h, double* incU, double* incV) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  NL_CUDA(cudaStreamSynchronize(h->st));
  if (incU) NL_CUDA(cudaMemcpy(incU, h->core->incU, sizeof(double) * h->core->n(), cudaMemcpyDeviceToHost));
  if (incV) NL_CUDA(cudaMemcpy(incV, h->core->incV, sizeof(double) * 3 * (size_t)h->desc.np_var, cudaMemcpyDeviceToHost));
  return NL_OK;
}

nl_status nl_inc_sqnorm(nl_problem* h, double* out) {
  NL_CHECK_READY(h);
  std::vector<double> u(h->core->n()), v(3 * (size_t)h->desc.np_var);
  nl_status s = nl_get_increment(h, u.data(), v.data());
  if (s != NL_OK) return s;
  double a = 0;
  for (double x : u) a += x * x;
  for (double x : v) a += x * x;
  *out = a;
  return NL_OK;
}

nl_status nl_get_schur(nl_problem* h, double* S, double* bS, int* n) {
  NL_CHECK_READY(h);
  if (n) *n = h->core->n();
  if (!S && !bS) return NL_OK;
  NL_CUDA(cudaSetDevice(h->device));
  return h->core->get_schur(S, bS);
}

nl_status nl_oplus(nl_problem* h) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  nl_status s = enqueue_oplus(h, nullptr);
  NL_CUDA(cudaStreamSynchronize(h->st));
  return s;
}

nl_status nl_backup(nl_problem* h) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  nl_status s = enqueue_copy_params(h, true, nullptr);
  NL_CUDA(cudaStreamSynchronize(h->st));
  return s;
}

nl_status nl_rollback(nl_problem* h) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  nl_status s = enqueue_copy_params(h, false, nullptr);
  NL_CUDA(cudaStreamSynchronize(h->st));
  return s;
}

nl_status nl_max_abs_b(nl_problem* h, double* out) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  return sync_read(h, h->scal + 1, out, 1);
}

nl_status nl_chi2(nl_problem* h, double* out) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  return sync_read(h, h->scal, out, 1);
}

nl_status nl_rho(nl_problem* h, double mu, double old_chi2, double* out) {
  NL_CHECK_READY(h);
  const int n = h->core->n(), nv = 3 * h->desc.np_var;
  std::vector<double> u(n), v(nv), bu(n), bv(nv);
  nl_status s = nl_get_increment(h, u.data(), v.data());
  if (s != NL_OK) return s;
  if ((s = h->core->get_hessian(nullptr, nullptr, nullptr, bu.data(), bv.data())) != NL_OK) return s;
  double chi2;
  if ((s = nl_chi2(h, &chi2)) != NL_OK) return s;
  double den = 0;
  for (int i = 0; i < n; i++) den += u[i] * (mu * u[i] - bu[i]);
  for (int i = 0; i < nv; i++) den += v[i] * (mu * v[i] - bv[i]);
  *out = (old_chi2 - chi2) / den;
  return NL_OK;
}

nl_status nl_lm_solve(nl_problem* h, const nl_lm_settings* st, nl_solve_report* rep, double* trace, int trace_cap) {
  NL_CHECK_READY(h);
  if (!st) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(h->device));
  LmDev s{};
  s.gn = 0;
  s.maxNumIt = st->maxNumIt;
  s.maxNumSubIt = st->maxNumSubIt;
  s.minNumIt = st->minNumIt;
  s.epsBVector = st->epsBVector;
  s.epsIncSquare = st->epsIncSquare;
  s.epsChi2 = st->epsChi2;
  s.tau = st->tau;
  s.penaltyV = st->penaltyV;
  s.initV = st->initV;
  s.maxScale = st->maxScaleFactor;
  s.minScale = st->minScaleFactor;
  const long long lim = (long long)std::max(st->maxNumIt, 0) * std::max(st->maxNumSubIt, 1) + 2;
  return run_solver(h, s, rep, trace, trace_cap, (int)std::min<long long>(lim, 1 << 30));
}

nl_status nl_lm_solve_batch(nl_problem** hs, int n, const nl_lm_settings* st, nl_solve_report* reps,
                             double* latency_ms) {
  if (!hs || n <= 0 || !st) return NL_ERR_ARG;
  for (int i = 0; i < n; i++) {
    NL_CHECK_READY(hs[i]);
    if (hs[i]->device != hs[0]->device) return NL_ERR_ARG;
    for (int j = 0; j < i; j++)
      if (hs[j] == hs[i]) return NL_ERR_ARG;
  }
  NL_CUDA(cudaSetDevice(hs[0]->device));
  LmDev s{};
  s.gn = 0;
  s.maxNumIt = st->maxNumIt;
  s.maxNumSubIt = st->maxNumSubIt;
  s.minNumIt = st->minNumIt;
  s.epsBVector = st->epsBVector;
  s.epsIncSquare = st->epsIncSquare;
  s.epsChi2 = st->epsChi2;
  s.tau = st->tau;
  s.penaltyV = st->penaltyV;
  s.initV = st->initV;
  s.maxScale = st->maxScaleFactor;
  s.minScale = st->minScaleFactor;
  s.trace_cap = 0;
  s.trace_n = 1;
  const int max_launch =
      (int)std::min<long long>((long long)std::max(st->maxNumIt, 0) * std::max(st->maxNumSubIt, 1) + 2, 1 << 30);
  // timing events: [0] the common start, then two per problem (launch parity)
  struct Events {
    std::vector<cudaEvent_t> e;
    ~Events() {
      for (auto x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  ev.e.assign(1 + 2 * (size_t)n, nullptr);
  for (auto& x : ev.e) NL_CUDA(cudaEventCreate(&x));
  cudaEvent_t ev_start = ev.e[0];
  NL_CUDA(cudaEventRecord(ev_start, hs[0]->st));
  // (1) update(true) everywhere, then one read per problem
  for (int i = 0; i < n; i++) {
    nl_problem* h = hs[i];
    NL_CUDA(cudaStreamWaitEvent(h->st, ev_start, 0));
    nl_status r = enqueue_eval(h, true, h->scal, h->scal + 1, nullptr);
    if (r != NL_OK) return r;
    NL_CUDA(cudaMemcpyAsync(h->host_pin, h->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  }
  std::vector<LmDev> init(n, s);
  std::vector<int> finished(n, 0), launched(n, 0), inflight(n, 0);
  std::vector<double> lat(n, 0.0);
  for (int i = 0; i < n; i++) {
    nl_problem* h = hs[i];
    NL_CUDA(cudaStreamSynchronize(h->st));
    init[i].chi2 = init[i].oldChi2 = h->host_pin[0];
    init[i].maxAbsB = h->host_pin[1];
    if (h->host_pin[1] <= s.epsBVector) {  // SuccessAtStart
      init[i].done = 1;
      init[i].reason = NL_SUCCESS_AT_START;
      init[i].iter = -1;
      finished[i] = 1;
      continue;
    }
    nl_status r = enqueue_copy_params(h, true, nullptr);  // backupSolution
    if (r != NL_OK) return r;
    if ((r = h->core->enqueue_hdiag(h->scal + 2)) != NL_OK) return r;
    NL_CUDA(cudaMemcpyAsync(h->host_pin + 2, h->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  }
  for (int i = 0; i < n; i++) {
    if (finished[i]) continue;
    nl_problem* h = hs[i];
    NL_CUDA(cudaStreamSynchronize(h->st));
    LmDev& q = init[i];
    q.maxAbsHDiag = h->host_pin[2];
    q.mu = q.tau * q.maxAbsHDiag;  // LevenbergMarquardt.hpp:58
    q.curV = q.initV;
    q.iter = q.subiter = q.nsub = 0;
    q.done = q.maxNumIt <= 0 ? 1 : 0;
    q.reason = NL_MAX_ITERATION_REACHED;
    NL_CUDA(cudaMemcpyAsync(h->lm, &q, sizeof(LmDev), cudaMemcpyHostToDevice, h->st));
    if (q.done) finished[i] = 1;
    // one LM sub-iteration as a CUDA graph, captured once per handle
    if (!h->sub_exec) {
      nl_status r = capture_subiteration(h, nullptr, &h->sub_exec);
      if (r != NL_OK) return r;
    }
  }
  for (int i = 0; i < n; i++)
    if (finished[i]) lat[i] = 0.0;
  // (2) interleave the problems: at most two sub-iterations in flight each,
  //     `done` read back behind each launch, completion seen by event query
  int remaining = 0;
  for (int i = 0; i < n; i++) remaining += !finished[i];
  while (remaining > 0) {
    bool progress = false;
    for (int i = 0; i < n; i++) {
      if (finished[i]) continue;
      nl_problem* h = hs[i];
      int* done_pin = reinterpret_cast<int*>(h->host_pin + 8);
      if (inflight[i] > 0) {
        const int old = launched[i] - inflight[i];
        cudaEvent_t e = ev.e[1 + 2 * (size_t)i + (old & 1)];
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) {
          inflight[i]--;
          progress = true;
          if (done_pin[old & 1] || (launched[i] >= max_launch && inflight[i] == 0)) {
            float ms = 0;
            NL_CUDA(cudaEventElapsedTime(&ms, ev_start, e));
            lat[i] = ms;
            finished[i] = 1;
            remaining--;
            continue;
          }
        } else if (q != cudaErrorNotReady) {
          NL_CUDA(q);
        }
      }
      if (inflight[i] < 2 && launched[i] < max_launch) {
        NL_CUDA(cudaGraphLaunch(h->sub_exec, h->st));
        NL_CUDA(cudaMemcpyAsync(done_pin + (launched[i] & 1), &h->lm->done, sizeof(int), cudaMemcpyDeviceToHost,
                                h->st));
        NL_CUDA(cudaEventRecord(ev.e[1 + 2 * (size_t)i + (launched[i] & 1)], h->st));
        launched[i]++;
        inflight[i]++;
        progress = true;
      }
    }
    if (!progress) std::this_thread::yield();
  }
  // (3) reports
  for (int i = 0; i < n; i++) {
    nl_problem* h = hs[i];
    NL_CUDA(cudaStreamSynchronize(h->st));
    LmDev fin;
    NL_CUDA(cudaMemcpy(&fin, h->lm, sizeof(LmDev), cudaMemcpyDeviceToHost));
    if (init[i].reason == NL_SUCCESS_AT_START && init[i].done) fin = init[i];
    if (reps) {
      reps[i].reason = fin.done ? fin.reason : NL_MAX_ITERATION_REACHED;
      reps[i].iterations = fin.iter;
      reps[i].subiterations = fin.nsub;
      reps[i].n_trace = 0;
      reps[i].chi2 = fin.chi2;
      reps[i].mu = fin.mu;
      reps[i].device_ms = lat[i];
    }
    if (latency_ms) latency_ms[i] = lat[i];
  }
  return NL_OK;
}

nl_status nl_gn_solve(nl_problem* h, const nl_gn_settings* st, nl_solve_report* rep, double* trace, int trace_cap) {
  NL_CHECK_READY(h);
  if (!st) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(h->device));
  LmDev s{};
  s.gn = 1;
  s.maxNumIt = st->maxNumIt;
  s.maxNumSubIt = 1 << 30;
  s.minNumIt = st->minNumIt;
  s.epsBVector = st->epsBVector;
  s.epsIncSquare = st->epsIncSquare;
  s.epsChi2 = st->epsChi2;
  s.gnRel = st->relLambda;
  s.gnAbs = st->absLambda;
  s.tau = 0;
  s.initV = 1;
  s.penaltyV = 1;
  return run_solver(h, s, rep, trace, trace_cap, std::max(st->maxNumIt, 0) + 2);
}

}  // extern "C"

namespace {

template <int BC>
void enqueue_hv(nl_problem* h, const double* vU, const double* vV, double* outU, double* outV) {
  if (h->nci > 0) hv_cam_kernel<BC, 128><<<h->nci, 128, 0, h->st>>>(h->ba, vU, vV, outU);
  if (h->desc.np_var > 0)
    hv_pt_kernel<BC><<<cdiv(h->desc.np_var, 128), 128, 0, h->st>>>(h->ba, h->adj_slot2int.as<int>(), vU, vV, outV);
  h->launches += 2;
}

// J'WJ v (MODE kHvGN) or the gradient J'W r (kGrad, v null) in FP64
template <int BC, int MODE>
void enqueue_gn(nl_problem* h, const double* vU, const double* vV, double* outU, double* outV) {
  if (h->nci > 0) hv_cam_kernel<BC, 128, MODE><<<h->nci, 128, 0, h->st>>>(h->ba, vU, vV, outU);
  if (h->desc.np_var > 0)
    hv_pt_kernel<BC, MODE><<<cdiv(h->desc.np_var, 128), 128, 0, h->st>>>(h->ba, h->adj_slot2int.as<int>(), vU, vV,
                                                                        outV);
  h->launches += 2;
}

// Work of nl_adjoint ([g | res | hv | mu], FP64, internal camera order then
// points; per-edge outputs) and the camera slot -> internal camera map used
// by the adjoint kernels, allocated on first use.
nl_status ensure_adjoint_buffers(nl_problem* h) {
  if (h->adj_vec.p) return NL_OK;
  const int ntot = h->nci * h->desc.bc + 3 * h->desc.np_var, ne = (int)h->e_cam.size();
  nl_status s;
  if ((s = h->adj_vec.alloc(sizeof(double) * 4 * (size_t)std::max(ntot, 1))) != NL_OK) return s;
  std::vector<int> s2i(h->nc_all(), -1);
  for (int u = 0; u < h->desc.nc_var; u++) s2i[u] = h->perm[u];
  if ((s = upload(h->adj_slot2int, s2i, h->st)) != NL_OK) return s;
  if ((s = h->adj_out.alloc(sizeof(double) * 3 * (size_t)std::max(ne, 1))) != NL_OK) return s;
  return NL_OK;
}

template <typename T>
void enqueue_neg_to_b(nl_problem* h, const double* res, int nU, int nV3) {
  if (nU > 0) neg_to_b_kernel<T><<<cdiv(nU, 256), 256, 0, h->st>>>(res, nU, (T*)h->core->dbU());
  if (nV3 > 0) neg_to_b_kernel<T><<<cdiv(nV3, 256), 256, 0, h->st>>>(res + nU, nV3, (T*)h->core->dbV());
  h->launches += 2;
}

// The mixed handle's step of the unrolled map, made the FP64 one: after
// enqueue_eval(true) and enqueue_increment at x_k (the increment from the
// FP32 Hessian), refine delta against (J'WJ + mu I) delta = -J'W r with both
// sides in FP64, the FP32 factor preconditioning; delta (ntot, internal camera
// order then points) receives the result.  Uses adj_vec's first three slots.
nl_status enqueue_step_fp64(nl_problem* h, const double* mu_dev, double* delta) {
  const int bc = h->desc.bc, nU = h->nci * bc, nV3 = 3 * h->desc.np_var, ntot = nU + nV3;
  if (ntot == 0) return NL_OK;
  double* g = h->adj_vec.as<double>();
  double* res = g + ntot;
  double* hv = res + ntot;
  nl_status s;
  if (nU) NL_CUDA(cudaMemcpyAsync(delta, h->core->incU, sizeof(double) * nU, cudaMemcpyDeviceToDevice, h->st));
  if (nV3) NL_CUDA(cudaMemcpyAsync(delta + nU, h->core->incV, sizeof(double) * nV3, cudaMemcpyDeviceToDevice, h->st));
  if (bc == 9)
    enqueue_gn<9, kGrad>(h, nullptr, nullptr, g, g + nU);
  else
    enqueue_gn<6, kGrad>(h, nullptr, nullptr, g, g + nU);
  for (int it = 0; it < kUnrollRefineSweeps; it++) {
    if (bc == 9)
      enqueue_gn<9, kHvGN>(h, delta, delta + nU, hv, hv + nU);
    else
      enqueue_gn<6, kHvGN>(h, delta, delta + nU, hv, hv + nU);
    step_resid_kernel<<<cdiv(ntot, 256), 256, 0, h->st>>>(g, hv, delta, mu_dev, ntot, res);
    enqueue_neg_to_b<float>(h, res, nU, nV3);
    if ((s = h->core->enqueue_resolve(h->status)) != NL_OK) return s;
    if (nU) acc_kernel<<<cdiv(nU, 256), 256, 0, h->st>>>(delta, h->core->incU, nU);
    if (nV3) acc_kernel<<<cdiv(nV3, 256), 256, 0, h->st>>>(delta + nU, h->core->incV, nV3);
    h->launches += 3;
  }
  return NL_OK;
}

}  // namespace

extern "C" {

nl_status nl_adjoint(nl_problem* h, const double* dL_dcams, const double* dL_dpts, int sweeps, double* g_obs,
                     double* g_weight, double* mu_cams, double* mu_pts, nl_adjoint_report* rep) {
  NL_CHECK_READY(h);
  if (sweeps < 0 || sweeps > 64) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(h->device));
  const int bc = h->desc.bc, nci = h->nci, npv = h->desc.np_var, ncv = h->desc.nc_var;
  const int nU = nci * bc, nV3 = 3 * npv, ntot = nU + nV3;
  const int ne = (int)h->e_cam.size();
  nl_status s;
  if ((s = ensure_adjoint_buffers(h)) != NL_OK) return s;
  double* g = h->adj_vec.as<double>();
  double* res = g + ntot;
  double* hv = res + ntot;
  double* mu = hv + ntot;
  std::vector<double> gh(ntot, 0.0);
  if (dL_dcams)
    for (int u = 0; u < ncv; u++)
      for (int i = 0; i < bc; i++) gh[(size_t)h->perm[u] * bc + i] = dL_dcams[(size_t)u * bc + i];
  if (dL_dpts) std::copy(dL_dpts, dL_dpts + nV3, gh.begin() + nU);
  double gnorm = 0;
  for (double x : gh) gnorm += x * x;
  gnorm = std::sqrt(gnorm);
  NL_CUDA(cudaEventRecord(h->ev_t0, h->st));
  if (ntot > 0) {
    NL_CUDA(cudaMemcpyAsync(g, gh.data(), sizeof(double) * ntot, cudaMemcpyHostToDevice, h->st));
    NL_CUDA(cudaMemcpyAsync(res, g, sizeof(double) * ntot, cudaMemcpyDeviceToDevice, h->st));
    NL_CUDA(cudaMemsetAsync(mu, 0, sizeof(double) * ntot, h->st));
  }
  // J'WJ at x* (and the cost); its factorisation preconditions the exact Hessian
  if ((s = enqueue_eval(h, true, h->scal, h->scal + 1, nullptr)) != NL_OK) return s;
  h->host_pin[16] = 0.0;
  h->host_pin[17] = 0.0;
  NL_CUDA(cudaMemcpyAsync(h->d_lam.p, h->host_pin + 16, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
  NL_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
  const bool f64 = h->desc.precision == NL_PREC_FP64;
  for (int it = 0; it <= sweeps; it++) {
    if (f64)
      enqueue_neg_to_b<double>(h, res, nU, nV3);
    else
      enqueue_neg_to_b<float>(h, res, nU, nV3);
    s = it == 0 ? h->core->enqueue_increment(h->d_lam.as<double>(), h->status, nullptr)
                : h->core->enqueue_resolve(h->status);
    if (s != NL_OK) return s;
    if (nU > 0) acc_kernel<<<cdiv(nU, 256), 256, 0, h->st>>>(mu, h->core->incU, nU);
    if (nV3 > 0) acc_kernel<<<cdiv(nV3, 256), 256, 0, h->st>>>(mu + nU, h->core->incV, nV3);
    if (bc == 9)
      enqueue_hv<9>(h, mu, mu + nU, hv, hv + nU);
    else
      enqueue_hv<6>(h, mu, mu + nU, hv, hv + nU);
    if (ntot > 0) resid_kernel<<<cdiv(ntot, 256), 256, 0, h->st>>>(g, hv, ntot, res);
    h->launches += 3;
  }
  double* dobs = h->adj_out.as<double>();
  double* dw = dobs + 2 * (size_t)ne;
  if ((g_obs || g_weight) && ne > 0) {
    if (bc == 9)
      vjp_edge_kernel<9><<<cdiv(ne, 128), 128, 0, h->st>>>(h->ba, h->d_eorder.as<int>(), h->adj_slot2int.as<int>(),
                                                            mu, mu + nU, dobs, dw);
    else
      vjp_edge_kernel<6><<<cdiv(ne, 128), 128, 0, h->st>>>(h->ba, h->d_eorder.as<int>(), h->adj_slot2int.as<int>(),
                                                            mu, mu + nU, dobs, dw);
    h->launches++;
  }
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
  std::vector<double> rh(ntot), muh(ntot);
  if (ntot > 0) {
    NL_CUDA(cudaMemcpyAsync(rh.data(), res, sizeof(double) * ntot, cudaMemcpyDeviceToHost, h->st));
    NL_CUDA(cudaMemcpyAsync(muh.data(), mu, sizeof(double) * ntot, cudaMemcpyDeviceToHost, h->st));
  }
  if (g_obs && ne > 0) NL_CUDA(cudaMemcpyAsync(g_obs, dobs, sizeof(double) * 2 * ne, cudaMemcpyDeviceToHost, h->st));
  if (g_weight && ne > 0) NL_CUDA(cudaMemcpyAsync(g_weight, dw, sizeof(double) * ne, cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaMemcpyAsync(h->host_pin + 20, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  int st = 0;
  memcpy(&st, h->host_pin + 20, sizeof(int));
  double rnorm = 0;
  for (double x : rh) rnorm += x * x;
  if (mu_cams)
    for (int u = 0; u < ncv; u++)
      for (int i = 0; i < bc; i++) mu_cams[(size_t)u * bc + i] = muh[(size_t)h->perm[u] * bc + i];
  if (mu_pts) std::copy(muh.begin() + nU, muh.end(), mu_pts);
  if (rep) {
    rep->ok = st == 0 ? 1 : 0;
    rep->sweeps = sweeps;
    rep->grad_norm = gnorm;
    rep->residual_norm = std::sqrt(rnorm);
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
    rep->device_ms = ms;
  }
  if (st & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  if (st) return NL_ERR_NOT_SPD;
  return NL_OK;
}

// ---------------------------------------------------------------------------
// Unrolled differentiation (see unroll.cuh for the algebra).
nl_status nl_unroll_record(nl_problem* h, int nsteps, const double* mu, nl_unroll_report* rep) {
  NL_CHECK_READY(h);
  if (nsteps < 0 || nsteps > 100000 || (nsteps > 0 && !mu)) return NL_ERR_ARG;
  for (int k = 0; k < nsteps; k++)
    if (!(mu[k] >= 0.0) || !std::isfinite(mu[k])) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(h->device));
  const size_t nc = (size_t)h->nc_all() * 16, np = (size_t)h->np_all() * 3, per = nc + np;
  nl_status s;
  if (h->unr_ckpt.bytes < sizeof(double) * per * (size_t)std::max(nsteps, 1))
    if ((s = h->unr_ckpt.alloc(sizeof(double) * per * (size_t)std::max(nsteps, 1))) != NL_OK) return s;
  h->unr_n = -1;
  h->unr_mu.assign(mu, mu + nsteps);
  double* ck = h->unr_ckpt.as<double>();
  const bool f64 = h->desc.precision == NL_PREC_FP64;
  const int nU = h->nci * h->desc.bc, nV3 = 3 * h->desc.np_var, ntot = nU + nV3;
  double* dstep = nullptr;  // the refined step (mixed handle)
  if (!f64) {
    if ((s = ensure_adjoint_buffers(h)) != NL_OK) return s;
    dstep = h->adj_vec.as<double>() + 3 * (size_t)std::max(ntot, 1);
  }
  NL_CUDA(cudaEventRecord(h->ev_t0, h->st));
  int st = 0, done = 0;
  for (int k = 0; k < nsteps; k++) {
    // checkpoint x_k, then the step at x_k with damping mu_k
    NL_CUDA(cudaMemcpyAsync(ck + per * k, h->cam.p, sizeof(double) * nc, cudaMemcpyDeviceToDevice, h->st));
    if (np) NL_CUDA(cudaMemcpyAsync(ck + per * k + nc, h->pt.p, sizeof(double) * np, cudaMemcpyDeviceToDevice, h->st));
    if ((s = enqueue_eval(h, true, h->scal, h->scal + 1, nullptr)) != NL_OK) return s;
    h->host_pin[16] = 0.0;
    h->host_pin[17] = mu[k];
    NL_CUDA(cudaMemcpyAsync(h->d_lam.p, h->host_pin + 16, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    NL_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
    if ((s = h->core->enqueue_increment(h->d_lam.as<double>(), h->status, nullptr)) != NL_OK) return s;
    if (!f64 && ntot) {
      // the mixed handle follows the FP64 map: the step refined in FP64
      if ((s = enqueue_step_fp64(h, h->d_lam.as<double>() + 1, dstep)) != NL_OK) return s;
      if (nU) NL_CUDA(cudaMemcpyAsync(h->core->incU, dstep, sizeof(double) * nU, cudaMemcpyDeviceToDevice, h->st));
      if (nV3)
        NL_CUDA(cudaMemcpyAsync(h->core->incV, dstep + nU, sizeof(double) * nV3, cudaMemcpyDeviceToDevice, h->st));
    }
    NL_CUDA(cudaMemcpyAsync(h->host_pin + 20, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    NL_CUDA(cudaStreamSynchronize(h->st));
    memcpy(&st, h->host_pin + 20, sizeof(int));
    if (st) break;  // the step failed: the schedule is not a valid LM trajectory
    if ((s = enqueue_oplus(h, nullptr)) != NL_OK) return s;
    done = k + 1;
  }
  if ((s = enqueue_eval(h, false, h->scal, nullptr, nullptr)) != NL_OK) return s;
  NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
  double chi2 = 0;
  if ((s = sync_read(h, h->scal, &chi2, 1)) != NL_OK) return s;
  if (rep) {
    rep->steps = done;
    rep->ok = st == 0 ? 1 : 0;
    rep->chi2 = chi2;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
    rep->device_ms = ms;
  }
  if (st & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  if (st) return NL_ERR_NOT_SPD;
  h->unr_n = nsteps;
  return NL_OK;
}

nl_status nl_unroll_adjoint(nl_problem* h, const double* dL_dcams, const double* dL_dpts, double* g_obs,
                            double* g_weight, double* g_cams0, double* g_pts0, nl_unroll_report* rep) {
  NL_CHECK_READY(h);
  if (h->unr_n < 0) return NL_ERR_STATE;
  NL_CUDA(cudaSetDevice(h->device));
  const int K = h->unr_n, bc = h->desc.bc, nci = h->nci, npv = h->desc.np_var, ncv = h->desc.nc_var;
  const int nU = nci * bc, nV3 = 3 * npv, ntot = nU + nV3, ne = (int)h->e_cam.size();
  const size_t nc = (size_t)h->nc_all() * 16, np = (size_t)h->np_all() * 3, per = nc + np;
  nl_status s;
  if ((s = ensure_adjoint_buffers(h)) != NL_OK) return s;
  // [lam | a | delta | grad] (ntot each) | g_obs (2 ne) | g_w (ne) | x_K (per) | g_cams (ncv bc) |
  // the (rel, abs) damping pairs of the steps (2 K)
  const size_t need =
      4 * (size_t)std::max(ntot, 1) + 3 * (size_t)std::max(ne, 1) + per + (size_t)ncv * bc + 2 * (size_t)K + 1;
  if (h->unr_work.bytes < sizeof(double) * need)
    if ((s = h->unr_work.alloc(sizeof(double) * need)) != NL_OK) return s;
  double* lam = h->unr_work.as<double>();
  double* a = lam + std::max(ntot, 1);
  double* delta = a + std::max(ntot, 1);
  double* grad = delta + std::max(ntot, 1);
  double* gobs = grad + std::max(ntot, 1);
  double* gw = gobs + 2 * (size_t)std::max(ne, 1);
  double* xK = gw + std::max(ne, 1);
  double* gcam = xK + per;
  double* lams = gcam + (size_t)ncv * bc;
  const double* ck = h->unr_ckpt.as<double>();
  const bool f64 = h->desc.precision == NL_PREC_FP64;
  const int* s2i = h->adj_slot2int.as<int>();
  // lam_K = dL/dx_K in internal camera order
  std::vector<double> lh(ntot, 0.0);
  if (dL_dcams)
    for (int u = 0; u < ncv; u++)
      for (int i = 0; i < bc; i++) lh[(size_t)h->perm[u] * bc + i] = dL_dcams[(size_t)u * bc + i];
  if (dL_dpts) std::copy(dL_dpts, dL_dpts + nV3, lh.begin() + nU);
  std::vector<double> lamh(2 * (size_t)K);
  for (int k = 0; k < K; k++) {
    lamh[2 * (size_t)k] = 0.0;
    lamh[2 * (size_t)k + 1] = h->unr_mu[k];
  }
  NL_CUDA(cudaEventRecord(h->ev_t0, h->st));
  if (ntot) NL_CUDA(cudaMemcpyAsync(lam, lh.data(), sizeof(double) * ntot, cudaMemcpyHostToDevice, h->st));
  if (K) NL_CUDA(cudaMemcpyAsync(lams, lamh.data(), sizeof(double) * 2 * K, cudaMemcpyHostToDevice, h->st));
  NL_CUDA(cudaMemsetAsync(gobs, 0, sizeof(double) * 3 * (size_t)std::max(ne, 1), h->st));
  NL_CUDA(cudaMemcpyAsync(xK, h->cam.p, sizeof(double) * nc, cudaMemcpyDeviceToDevice, h->st));
  if (np) NL_CUDA(cudaMemcpyAsync(xK + nc, h->pt.p, sizeof(double) * np, cudaMemcpyDeviceToDevice, h->st));
  NL_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
  for (int k = K - 1; k >= 0; k--) {
    // x_k from its checkpoint; J, r, J'WJ and b there; the step delta_k (and
    // its factorisation) with the recorded damping
    NL_CUDA(cudaMemcpyAsync(h->cam.p, ck + per * k, sizeof(double) * nc, cudaMemcpyDeviceToDevice, h->st));
    if (np) NL_CUDA(cudaMemcpyAsync(h->pt.p, ck + per * k + nc, sizeof(double) * np, cudaMemcpyDeviceToDevice, h->st));
    if ((s = enqueue_eval(h, true, h->scal, h->scal + 1, nullptr)) != NL_OK) return s;
    if ((s = h->core->enqueue_increment(lams + 2 * (size_t)k, h->status, nullptr)) != NL_OK) return s;
    if (f64) {
      if (nU) NL_CUDA(cudaMemcpyAsync(delta, h->core->incU, sizeof(double) * nU, cudaMemcpyDeviceToDevice, h->st));
      if (nV3)
        NL_CUDA(cudaMemcpyAsync(delta + nU, h->core->incV, sizeof(double) * nV3, cudaMemcpyDeviceToDevice, h->st));
    } else if ((s = enqueue_step_fp64(h, lams + 2 * (size_t)k + 1, delta)) != NL_OK) {
      return s;
    }
    // through the retraction: a (the step's adjoint) and the direct part of lam_k
    if (ntot) {
      if (bc == 9)
        unroll_split_kernel<9><<<cdiv(nci + nV3, 256), 256, 0, h->st>>>(nci, nV3, delta, lam, a);
      else
        unroll_split_kernel<6><<<cdiv(nci + nV3, 256), 256, 0, h->st>>>(nci, nV3, delta, lam, a);
      h->launches++;
    }
    // u = A^-1 a with the step's factorisation (b := -a, so the increment is
    // u).  The mixed handle's factor is of the FP32 Hessian: u is refined
    // against A v = J'WJ v + mu_k v taken in FP64, the factor preconditioning.
    const double* uU = h->core->incU;
    const double* uV = h->core->incV;
    if (f64) {
      enqueue_neg_to_b<double>(h, a, nU, nV3);
      if ((s = h->core->enqueue_resolve(h->status)) != NL_OK) return s;
    } else {
      double* u = h->adj_vec.as<double>();
      double* res = u + std::max(ntot, 1);
      double* hv = res + std::max(ntot, 1);
      if (ntot) NL_CUDA(cudaMemsetAsync(u, 0, sizeof(double) * ntot, h->st));
      for (int it = 0; it <= kUnrollRefineSweeps; it++) {
        enqueue_neg_to_b<float>(h, it == 0 ? a : res, nU, nV3);
        if ((s = h->core->enqueue_resolve(h->status)) != NL_OK) return s;
        if (nU) acc_kernel<<<cdiv(nU, 256), 256, 0, h->st>>>(u, h->core->incU, nU);
        if (nV3) acc_kernel<<<cdiv(nV3, 256), 256, 0, h->st>>>(u + nU, h->core->incV, nV3);
        h->launches += 2;
        if (it == kUnrollRefineSweeps) break;
        if (bc == 9)
          enqueue_gn<9, kHvGN>(h, u, u + nU, hv, hv + nU);
        else
          enqueue_gn<6, kHvGN>(h, u, u + nU, hv, hv + nU);
        if (ntot) damped_resid_kernel<<<cdiv(ntot, 256), 256, 0, h->st>>>(a, hv, u, lams + 2 * (size_t)k + 1, ntot, res);
        h->launches++;
      }
      uU = u;
      uV = u + nU;
    }
    // lam_k -= grad_x (psi + phi); per-edge contributions to g_obs / g_w
    if (bc == 9) {
      if (nci) unroll_grad_cam_kernel<9, 128><<<nci, 128, 0, h->st>>>(h->ba, uU, uV, delta, delta + nU, grad);
      if (npv) unroll_grad_pt_kernel<9><<<cdiv(npv, 128), 128, 0, h->st>>>(h->ba, s2i, uU, uV, delta, delta + nU, grad + nU);
      if (ne) unroll_vjp_edge_kernel<9><<<cdiv(ne, 128), 128, 0, h->st>>>(h->ba, h->d_eorder.as<int>(), s2i, uU, uV, delta,
                                                                             delta + nU, gobs, gw);
    } else {
      if (nci) unroll_grad_cam_kernel<6, 128><<<nci, 128, 0, h->st>>>(h->ba, uU, uV, delta, delta + nU, grad);
      if (npv) unroll_grad_pt_kernel<6><<<cdiv(npv, 128), 128, 0, h->st>>>(h->ba, s2i, uU, uV, delta, delta + nU, grad + nU);
      if (ne) unroll_vjp_edge_kernel<6><<<cdiv(ne, 128), 128, 0, h->st>>>(h->ba, h->d_eorder.as<int>(), s2i, uU, uV, delta,
                                                                             delta + nU, gobs, gw);
    }
    if (ntot) sub_kernel<<<cdiv(ntot, 256), 256, 0, h->st>>>(lam, grad, ntot);
    h->launches += 4;
    NL_CUDA(cudaGetLastError());
  }
  // lam_0 in the caller's parameters (axis-angle cameras in user order)
  if (ncv) {
    if (bc == 9)
      unroll_to_params_kernel<9><<<cdiv(ncv, 128), 128, 0, h->st>>>(ncv, s2i, K > 0 ? ck : xK, lam, gcam);
    else
      unroll_to_params_kernel<6><<<cdiv(ncv, 128), 128, 0, h->st>>>(ncv, s2i, K > 0 ? ck : xK, lam, gcam);
    h->launches++;
  }
  NL_CUDA(cudaGetLastError());
  // back to x_K
  NL_CUDA(cudaMemcpyAsync(h->cam.p, xK, sizeof(double) * nc, cudaMemcpyDeviceToDevice, h->st));
  if (np) NL_CUDA(cudaMemcpyAsync(h->pt.p, xK + nc, sizeof(double) * np, cudaMemcpyDeviceToDevice, h->st));
  NL_CUDA(cudaEventRecord(h->ev_t1, h->st));
  if (g_cams0 && ncv) NL_CUDA(cudaMemcpyAsync(g_cams0, gcam, sizeof(double) * ncv * bc, cudaMemcpyDeviceToHost, h->st));
  if (g_pts0 && nV3) NL_CUDA(cudaMemcpyAsync(g_pts0, lam + nU, sizeof(double) * nV3, cudaMemcpyDeviceToHost, h->st));
  if (g_obs && ne) NL_CUDA(cudaMemcpyAsync(g_obs, gobs, sizeof(double) * 2 * ne, cudaMemcpyDeviceToHost, h->st));
  if (g_weight && ne) NL_CUDA(cudaMemcpyAsync(g_weight, gw, sizeof(double) * ne, cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaMemcpyAsync(h->host_pin + 20, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  int st = 0;
  memcpy(&st, h->host_pin + 20, sizeof(int));
  if (rep) {
    rep->steps = K;
    rep->ok = st == 0 ? 1 : 0;
    rep->chi2 = 0.0;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
    rep->device_ms = ms;
  }
  if (st & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  if (st) return NL_ERR_NOT_SPD;
  return NL_OK;
}

}  // extern "C"

nl_status nl_problem_get_view(nl_problem* h, nl_problem_view* v) {
  if (!h || !v) return NL_ERR_ARG;
  v->bc = h->desc.bc;
  v->ncv = h->desc.nc_var;
  v->ncf = h->desc.nc_fix;
  v->npv = h->desc.np_var;
  v->npf = h->desc.np_fix;
  v->f = h->desc.f;
  v->cx = h->desc.cx;
  v->cy = h->desc.cy;
  v->e_cam = &h->e_cam;
  v->e_camfix = &h->e_camfix;
  v->e_pt = &h->e_pt;
  v->e_ptfix = &h->e_ptfix;
  v->perm = &h->perm;
  v->eorder = &h->eorder;
  v->porder = &h->porder;
  v->e_obs = &h->e_obs;
  v->e_w = &h->e_w;
  v->d_cam = h->cam.as<double>();
  v->d_pt = h->pt.as<double>();
  v->ready = h->ready;
  return NL_OK;
}

extern "C" {

nl_status nl_phase_timings(nl_problem* h, nl_phase_times* out) {
  NL_CHECK_READY(h);
  *out = h->core->times;
  out->eval_ms = h->eval_ms;
  return NL_OK;
}

nl_status nl_set_solver_kind(nl_problem* h, int kind) {
  NL_CHECK_H(h);
  if (kind != NL_SOLVER_DENSE && kind != NL_SOLVER_ENVELOPE) return NL_ERR_ARG;
  if (!h->core) return NL_ERR_STATE;
  h->core->envelope = kind == NL_SOLVER_ENVELOPE ? 1 : 0;
  return NL_OK;
}

nl_status nl_set_timing_detail(nl_problem* h, int detail) {
  NL_CHECK_H(h);
  h->timing_detail = detail ? 1 : 0;
  return NL_OK;
}

nl_status nl_set_wait_limit(nl_problem* h, long long polls) {
  NL_CHECK_H(h);
  if (!h->core) return NL_ERR_STATE;
  h->core->wait_limit = polls > 0 ? polls : kSpinLimit;
  return NL_OK;
}

nl_status nl_check_wait_timeout(nl_problem* h) {
  NL_CHECK_READY(h);
  NL_CUDA(cudaSetDevice(h->device));
  NL_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), h->st));
  nl_status s = h->core->enqueue_solve_withheld(h->status);
  if (s != NL_OK) return s;
  NL_CUDA(cudaMemcpyAsync(h->host_pin + 20, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  int st = 0;
  memcpy(&st, h->host_pin + 20, sizeof(int));
  return (st & ST_SPIN_TIMEOUT) ? NL_ERR_TIMEOUT : NL_OK;
}

nl_status nl_kernel_launches(nl_problem* h, long long* out) {
  NL_CHECK_H(h);
  *out = h->launches + (h->core ? h->core->launches : 0);
  return NL_OK;
}

}  // extern "C"

// ===========================================================================
// Solver-only drop-in: SolverCholeskySchur on a caller-assembled Hessian.
struct nl_solver {
  nl_solver_desc d{};
  cudaStream_t st = nullptr;
  cublasHandle_t cublas = nullptr;
  DevBuf ws, lam;
  std::unique_ptr<SchurCore> core;
  double* pin = nullptr;
  ~nl_solver() {
    core.reset();
    if (cublas) cublasDestroy(cublas);
    if (pin) cudaFreeHost(pin);
    if (st) cudaStreamDestroy(st);
  }
};

extern "C" {

nl_status nl_solver_create(const nl_solver_desc* d, const int* u_rc, const int* v_rc, const int* w_rc,
                           nl_solver** out) {
  if (!d || !out || d->bu < 1 || d->bu > 9 || d->nu < 0 || d->nv < 0 || d->nU < 0 || d->nV < 0 || d->nW < 0)
    return NL_ERR_ARG;
  if ((d->nU > 0 && !u_rc) || (d->nV > 0 && !v_rc) || (d->nW > 0 && !w_rc)) return NL_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<nl_solver> s(new nl_solver());
  s->d = *d;
  NL_CUDA(cudaSetDevice(d->device));
  {
    int lo = 0, hi = 0;
    NL_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    NL_CUDA(cudaStreamCreateWithPriority(&s->st, cudaStreamNonBlocking, hi));
  }
  if (d->precision == NL_PREC_FP64) {
    if (cublasCreate(&s->cublas) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
    cublasSetStream(s->cublas, s->st);
    nl_status r = s->ws.alloc(64u << 20);
    if (r != NL_OK) return r;
    cublasSetWorkspace(s->cublas, s->ws.p, s->ws.bytes);
  }
  s->core = make_schur_core(d->precision, d->bu, s->cublas);
  if (!s->core) return NL_ERR_UNSUPPORTED;
  s->core->refine_sweeps = d->refine_sweeps >= 0 ? d->refine_sweeps : (d->precision == NL_PREC_MIXED ? 1 : 0);
  s->core->keep_schur = 0;
  s->core->use_tc = d->precision == NL_PREC_MIXED ? 1 : 0;
  SchurStructure ss;
  ss.bc = d->bu;
  ss.nci = d->nu;
  ss.np = d->nv;
  for (int q = 0; q < d->nU; q++) {
    ss.u_r.push_back(u_rc[2 * q]);
    ss.u_c.push_back(u_rc[2 * q + 1]);
    if (q > 0) {  // CSC order of the upper pattern
      const int pc = u_rc[2 * q - 1], pr = u_rc[2 * q - 2];
      if (u_rc[2 * q + 1] < pc || (u_rc[2 * q + 1] == pc && u_rc[2 * q] <= pr)) return NL_ERR_ARG;
    }
  }
  ss.v_uid.assign(d->nv, -1);
  for (int q = 0; q < d->nV; q++) {
    const int r = v_rc[2 * q], c = v_rc[2 * q + 1];
    if (r != c) return NL_ERR_UNSUPPORTED;  // V must be block diagonal (MatrixDiagInv)
    if (c < 0 || c >= d->nv || ss.v_uid[c] >= 0) return NL_ERR_ARG;
    ss.v_uid[c] = q;
  }
  for (int q = 0; q < d->nW; q++) {
    ss.w_r.push_back(w_rc[2 * q]);
    ss.w_c.push_back(w_rc[2 * q + 1]);
  }
  nl_status r = s->core->setup(ss, s->st);
  if (r != NL_OK) return r;
  if ((r = s->lam.alloc(64)) != NL_OK) return r;
  NL_CUDA(cudaMallocHost(&s->pin, 256));
  NL_CUDA(cudaStreamSynchronize(s->st));
  *out = s.release();
  return NL_OK;
}

nl_status nl_solver_destroy(nl_solver* s) {
  if (!s) return NL_ERR_ARG;
  cudaSetDevice(s->d.device);
  cudaStreamSynchronize(s->st);
  delete s;
  return NL_OK;
}

nl_status nl_solver_set_hessian(nl_solver* s, const double* U, const double* V, const double* W, const double* bU,
                                const double* bV) {
  if (!s) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(s->d.device));
  return s->core->set_hessian(U, V, W, bU, bV);
}

nl_status nl_solver_max_abs_hdiag(nl_solver* s, double* out) {
  if (!s || !out) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(s->d.device));
  double* dv = s->lam.as<double>() + 4;
  nl_status r = s->core->enqueue_hdiag(dv);
  if (r != NL_OK) return r;
  NL_CUDA(cudaMemcpyAsync(s->pin, dv, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  NL_CUDA(cudaStreamSynchronize(s->st));
  *out = s->pin[0];
  return NL_OK;
}

nl_status nl_solver_set_kind(nl_solver* s, int kind) {
  if (!s || !s->core) return NL_ERR_ARG;
  if (kind != NL_SOLVER_DENSE && kind != NL_SOLVER_ENVELOPE) return NL_ERR_ARG;
  s->core->envelope = kind == NL_SOLVER_ENVELOPE ? 1 : 0;
  return NL_OK;
}

nl_status nl_solver_compute_increment(nl_solver* s, double rel, double abs_, double* incU, double* incV, int* ok) {
  if (!s) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(s->d.device));
  s->pin[0] = rel;
  s->pin[1] = abs_;
  NL_CUDA(cudaMemcpyAsync(s->lam.p, s->pin, 2 * sizeof(double), cudaMemcpyHostToDevice, s->st));
  int* status = reinterpret_cast<int*>(s->lam.as<double>() + 2);
  NL_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s->st));
  nl_status r = s->core->enqueue_increment(s->lam.as<double>(), status, nullptr);
  if (r != NL_OK) return r;
  NL_CUDA(cudaMemcpyAsync(s->pin + 4, status, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if (incU) NL_CUDA(cudaMemcpyAsync(incU, s->core->incU, sizeof(double) * s->core->n(), cudaMemcpyDeviceToHost, s->st));
  if (incV) NL_CUDA(cudaMemcpyAsync(incV, s->core->incV, sizeof(double) * 3 * (size_t)s->d.nv, cudaMemcpyDeviceToHost, s->st));
  NL_CUDA(cudaStreamSynchronize(s->st));
  int st;
  memcpy(&st, s->pin + 4, sizeof(int));
  if (ok) *ok = st == 0 ? 1 : 0;
  if (st & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  return NL_OK;
}

}  // extern "C"

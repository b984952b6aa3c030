// schur_core.cu -- SolverCholeskySchur on the device (see schur_core.cuh).
#include <cstring>

#include "schur_core.cuh"

namespace nl {

namespace {

constexpr int kNT = 256;
constexpr int kRedCTAs = 296;  // 2 x 148 SMs for grid-stride reductions
constexpr int kSymvChunks = 8;
constexpr int kSchurWarps = 8;

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

template <typename T, int BC>
class SchurCoreT final : public SchurCore {
 public:
  explicit SchurCoreT(cublasHandle_t cb, int precision) : cublas_(cb), precision_(precision) {}

  int n() const override { return n_; }
  int ld() const override { return ld_; }
  void* dU() override { return U_.p; }
  void* dV() override { return V_.p; }
  void* dW() override { return W_.p; }
  void* dbU() override { return bU_.p; }
  void* dbV() override { return bV_.p; }

  nl_status setup(const SchurStructure& st, cudaStream_t stream) override {
    st_ = stream;
    nci_ = st.nci;
    np_ = st.np;
    nU_ = (int)st.u_r.size();
    nW_ = (int)st.w_r.size();
    nV_ = 0;
    for (int q : st.v_uid) nV_ = std::max(nV_, q + 1);
    n_ = nci_ * BC;
    ld_ = std::max(NB, cdiv(n_, NB) * NB);
    ntiles_ = ld_ / NB;
    // ---- derived host structure ----
    std::vector<int> w_row_ptr(nci_ + 1, 0), w_col_ptr(np_ + 1, 0), w_col_uid(nW_);
    for (int q = 0; q < nW_; q++) {
      if (st.w_r[q] < 0 || st.w_r[q] >= nci_ || st.w_c[q] < 0 || st.w_c[q] >= np_) return NL_ERR_ARG;
      if (q > 0 && (st.w_r[q] < st.w_r[q - 1] || (st.w_r[q] == st.w_r[q - 1] && st.w_c[q] <= st.w_c[q - 1])))
        return NL_ERR_ARG;  // W UIDs must follow CSR order
      w_row_ptr[st.w_r[q] + 1]++;
      w_col_ptr[st.w_c[q] + 1]++;
    }
    for (int i = 0; i < nci_; i++) w_row_ptr[i + 1] += w_row_ptr[i];
    for (int j = 0; j < np_; j++) w_col_ptr[j + 1] += w_col_ptr[j];
    {
      std::vector<int> fill(w_col_ptr.begin(), w_col_ptr.end() - 1);
      for (int q = 0; q < nW_; q++) w_col_uid[fill[st.w_c[q]]++] = q;
    }
    std::vector<int> u_diag(nci_, -1);
    for (int q = 0; q < nU_; q++) {
      if (st.u_r[q] > st.u_c[q] || st.u_c[q] >= nci_) return NL_ERR_ARG;
      if (st.u_r[q] == st.u_c[q]) u_diag[st.u_r[q]] = q;
    }
    // ---- output blocks of S: U pattern + W W' pattern + every diagonal ----
    if ((long long)nci_ * nci_ > (1LL << 28)) return NL_ERR_UNSUPPORTED;  // dense S too large anyway
    std::vector<int> bmap((size_t)nci_ * nci_, 0);       // pair counts, then block ids
    std::vector<long long> cnt;
    for (int i = 0; i < nci_; i++) bmap[(size_t)i * nci_ + i] = 1;  // mark
    for (int q = 0; q < nU_; q++) bmap[(size_t)st.u_r[q] * nci_ + st.u_c[q]] = 1;
    long long npairs = 0;
    std::vector<int> pc((size_t)nci_ * nci_, 0);
    for (int p = 0; p < np_; p++) {
      for (int s = w_col_ptr[p]; s < w_col_ptr[p + 1]; s++)
        for (int t = s; t < w_col_ptr[p + 1]; t++) {
          const int i = st.w_r[w_col_uid[s]], j = st.w_r[w_col_uid[t]];
          bmap[(size_t)i * nci_ + j] = 1;
          pc[(size_t)i * nci_ + j]++;
          npairs++;
        }
    }
    std::vector<int> s_i, s_j, s_uuid;
    std::vector<long long> s_ptr(1, 0);
    std::vector<int> bid((size_t)nci_ * nci_, -1);
    for (int i = 0; i < nci_; i++)
      for (int j = i; j < nci_; j++)
        if (bmap[(size_t)i * nci_ + j]) {
          bid[(size_t)i * nci_ + j] = (int)s_i.size();
          s_i.push_back(i);
          s_j.push_back(j);
          s_uuid.push_back(-1);
          s_ptr.push_back(s_ptr.back() + pc[(size_t)i * nci_ + j]);
        }
    for (int q = 0; q < nU_; q++) s_uuid[bid[(size_t)st.u_r[q] * nci_ + st.u_c[q]]] = q;
    nS_ = (int)s_i.size();
    // Cholesky envelope of S by 128-tiles: env_first_[T] = first tile column
    // with a nonzero in tile row T (block (i, j), i <= j, sits at rows j BC..,
    // columns i BC.. of the lower storage).  The factor has no fill before a
    // row's first nonzero, so L_TJ = 0 for J < env_first_[T].
    // env_last_[k] = last tile row T with env_first_[T] <= k (the last
    // nonzero tile of L's column k); env_run_[k] = max over k' <= k of it.
    env_first_.assign(ntiles_, 0);
    for (int t = 0; t < ntiles_; t++) env_first_[t] = t;
    for (int b = 0; b < nS_; b++) {
      const int tc = (s_i[b] * BC) / NB;
      for (int t = (s_j[b] * BC) / NB; t <= (s_j[b] * BC + BC - 1) / NB; t++) env_first_[t] = std::min(env_first_[t], tc);
    }
    env_last_.assign(ntiles_, 0);
    for (int k = 0; k < ntiles_; k++) env_last_[k] = k;
    for (int t = 0; t < ntiles_; t++)
      for (int k = env_first_[t]; k < t; k++) env_last_[k] = std::max(env_last_[k], t);
    env_run_.assign(ntiles_, 0);
    for (int k = 0; k < ntiles_; k++) env_run_[k] = std::max(env_last_[k], k > 0 ? env_run_[k - 1] : 0);
    // Schur work order: output blocks by pair count, heaviest first
    std::vector<int> s_order(std::max(nS_, 1), 0);
    for (int b = 0; b < nS_; b++) s_order[b] = b;
    std::stable_sort(s_order.begin(), s_order.begin() + nS_,
                     [&](int x, int y) { return s_ptr[x + 1] - s_ptr[x] > s_ptr[y + 1] - s_ptr[y]; });
    std::vector<int> pa(std::max<long long>(npairs, 1)), pb(std::max<long long>(npairs, 1));
    {
      std::vector<long long> fill(s_ptr.begin(), s_ptr.end() - 1);
      for (int p = 0; p < np_; p++)  // points ascending: the merge order of MatrixWWtMultiplier
        for (int s = w_col_ptr[p]; s < w_col_ptr[p + 1]; s++)
          for (int t = s; t < w_col_ptr[p + 1]; t++) {
            const int a = w_col_uid[s], b = w_col_uid[t];
            const long long slot = fill[bid[(size_t)st.w_r[a] * nci_ + st.w_r[b]]]++;
            pa[slot] = a;
            pb[slot] = b;
          }
    }
    npairs_ = npairs;
    // ---- device allocations ----
    nl_status s;
#define NL_TRY(x)           \
  do {                      \
    if ((s = (x)) != NL_OK) \
      return s;             \
  } while (0)
    NL_TRY(U_.alloc(sizeof(T) * (size_t)std::max(nU_, 1) * Layout<T, BC>::U));
    NL_TRY(V_.alloc(sizeof(T) * (size_t)std::max(nV_, 1) * Layout<T, BC>::V));
    NL_TRY(W_.alloc(sizeof(T) * (size_t)std::max(nW_, 1) * Layout<T, BC>::W));
    NL_TRY(Y_.alloc(sizeof(T) * (size_t)std::max(nW_, 1) * Layout<T, BC>::W));
    NL_TRY(Vinv_.alloc(sizeof(T) * (size_t)std::max(np_, 1) * Layout<T, BC>::V));
    NL_TRY(bU_.alloc(sizeof(T) * (size_t)ld_));
    NL_TRY(bV_.alloc(sizeof(T) * (size_t)std::max(3 * np_, 1)));
    NL_TRY(bS_.alloc(sizeof(double) * (size_t)ld_));
    NL_TRY(incU_.alloc(sizeof(double) * (size_t)ld_));
    NL_TRY(incV_.alloc(sizeof(double) * (size_t)std::max(3 * np_, 1)));
    NL_TRY(y_.alloc(sizeof(double) * (size_t)ld_));
    NL_TRY(r_.alloc(sizeof(double) * (size_t)ld_));
    NL_TRY(dx_.alloc(sizeof(double) * (size_t)ld_));
    NL_TRY(part_.alloc(sizeof(double) * (size_t)std::max(kSymvChunks * ld_, 4 * kRedCTAs)));
    NL_TRY(Linv_.alloc(sizeof(T) * (size_t)ntiles_ * NB * NB));
    NL_TRY(hop_.alloc(sizeof(T) * 2 * kHopDepth * (size_t)ntiles_ * NB * NB));
    // the diagonal-tile factor writes only the blocks on and below the
    // diagonal: the strictly upper blocks of every inverse stay zero
    NL_CUDA(cudaMemsetAsync(Linv_.p, 0, Linv_.bytes, st_));
    NL_TRY(env_dev_.alloc(sizeof(int) * 2 * (size_t)ntiles_));
    NL_CUDA(cudaMemcpyAsync(env_dev_.p, env_first_.data(), sizeof(int) * ntiles_, cudaMemcpyHostToDevice, st_));
    NL_CUDA(cudaMemcpyAsync(env_dev_.as<int>() + ntiles_, env_last_.data(), sizeof(int) * ntiles_,
                            cudaMemcpyHostToDevice, st_));
    NL_TRY(flags_.alloc(sizeof(int) * (size_t)(ntiles_ + 1)));
    NL_TRY(S_.alloc(sizeof(T) * (size_t)ld_ * ld_));
    s_cleared_ = false;
    need_s0_ = refine_sweeps > 0 || keep_schur;
    if (need_s0_) NL_TRY(S0_.alloc(sizeof(T) * (size_t)ld_ * ld_));
    if (sizeof(T) == 4 && use_tc) {
      NL_CUDA(tc_prepare());
      tcs_half_ = (tc_syrk_scratch_bytes(ld_) + 255) / 256 * 256;
      NL_TRY(tcs_.alloc(kPackSlots * tcs_half_));
    }
    NL_TRY(upload(v_uid_, st.v_uid, st_));
    NL_TRY(upload(w_row_ptr_, w_row_ptr, st_));
    NL_TRY(upload(w_col_, st.w_c, st_));
    NL_TRY(upload(w_row_, st.w_r, st_));
    NL_TRY(upload(w_col_ptr_, w_col_ptr, st_));
    NL_TRY(upload(w_col_uid_, w_col_uid, st_));
    NL_TRY(upload(u_diag_, u_diag, st_));
    NL_TRY(upload(s_i_, s_i, st_));
    NL_TRY(upload(s_j_, s_j, st_));
    NL_TRY(upload(s_uuid_, s_uuid, st_));
    NL_TRY(upload(s_order_, s_order, st_));
    NL_TRY(sched_.alloc(sizeof(int) * 4));
    NL_TRY(upload(s_ptr_, s_ptr, st_));
    NL_TRY(upload(pa_, pa, st_));
    NL_TRY(upload(pb_, pb, st_));
#undef NL_TRY
    NL_CUDA(cudaMemsetAsync(U_.p, 0, U_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(V_.p, 0, V_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(W_.p, 0, W_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(bU_.p, 0, bU_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(bV_.p, 0, bV_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(bS_.p, 0, bS_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(incU_.p, 0, incU_.bytes, st_));
    NL_CUDA(cudaMemsetAsync(incV_.p, 0, incV_.bytes, st_));
    incU = incU_.as<double>();
    incV = incV_.as<double>();
    d_.bc = BC;
    d_.nci = nci_;
    d_.np = np_;
    d_.nU = nU_;
    d_.nW = nW_;
    d_.nS = nS_;
    d_.n = n_;
    d_.ld = ld_;
    d_.v_uid = v_uid_.as<int>();
    d_.w_row_ptr = w_row_ptr_.as<int>();
    d_.w_col = w_col_.as<int>();
    d_.w_row = w_row_.as<int>();
    d_.w_col_ptr = w_col_ptr_.as<int>();
    d_.w_col_uid = w_col_uid_.as<int>();
    d_.u_diag_uid = u_diag_.as<int>();
    d_.s_i = s_i_.as<int>();
    d_.s_j = s_j_.as<int>();
    d_.s_uuid = s_uuid_.as<int>();
    d_.s_pair_ptr = s_ptr_.as<long long>();
    d_.pair_a = pa_.as<int>();
    d_.pair_b = pb_.as<int>();
    NL_CUDA(cudaFuncSetAttribute(trsm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<T>()));
    NL_CUDA(cudaFuncSetAttribute(trsv_fwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsv_smem<T>()));
    NL_CUDA(cudaFuncSetAttribute(trsv_bwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsv_smem<T>()));
    NL_CUDA(cudaFuncSetAttribute(trsm_tile_kernel<kChainRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTrsmTileSmem));
    NL_CUDA(cudaFuncSetAttribute(diag_update_kernel<kChainRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 2 * (int)kDiagUpdSmem));
    if (!ev_[0]) {
      for (auto& e : ev_) NL_CUDA(cudaEventCreate(&e));
      NL_CUDA(cudaEventCreateWithFlags(&ev_panel_, cudaEventDisableTiming));
      NL_CUDA(cudaEventCreateWithFlags(&ev_b_, cudaEventDisableTiming));
      {
        // the side stream (bulk trailing updates) yields SMs to the critical path
        int lo = 0, hi = 0;
        NL_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        NL_CUDA(cudaStreamCreateWithPriority(&st2_, cudaStreamNonBlocking, lo));
        // the auxiliary stream (panel work off the critical path) runs at the top priority
        NL_CUDA(cudaStreamCreateWithPriority(&st3_, cudaStreamNonBlocking, hi));
      }
      for (auto& e : dev_) NL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      if (cublas_) {
        if (cublasCreate(&cublas2_) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
        nl_status ws = ws2_.alloc(64u << 20);
        if (ws != NL_OK) return ws;
        cublasSetWorkspace(cublas2_, ws2_.p, ws2_.bytes);
        cublasSetStream(cublas2_, st2_);
      }
    }
    return NL_OK;
  }

  // ---- solves with the factor: x = S^-1 b (trsv fwd + bwd) ----
  nl_status enqueue_solve(const double* b, double* x, int* status, const int* active) {
    NL_CUDA(cudaMemsetAsync(flags_.p, 0, flags_.bytes, st_));
    const int* env = envelope ? env_dev_.as<int>() : nullptr;
    trsv_fwd_kernel<T><<<ntiles_, SV, trsv_smem<T>(), st_>>>(S_.as<T>(), ld_, ntiles_, Linv_.as<T>(), hop_.as<T>(), b,
                                                 y_.as<double>(),
                                                 flags_.as<int>(), flags_.as<int>() + 1, 1, status, wait_limit, env,
                                                 active);
    NL_CUDA(cudaMemsetAsync(flags_.p, 0, flags_.bytes, st_));
    trsv_bwd_kernel<T><<<ntiles_, SV, trsv_smem<T>(), st_>>>(S_.as<T>(), ld_, ntiles_, Linv_.as<T>(), hop_.as<T>(),
                                                 y_.as<double>(), x,
                                                 flags_.as<int>(), flags_.as<int>() + 1, 1, status, wait_limit, env,
                                                 active);
    launches += 2;
    return NL_OK;
  }

  // The forward solve with tile 0 left out: the ticket counter starts at 1,
  // so the ntiles - 1 CTAs take tiles 1 .. ntiles - 1 and each first waits
  // for tile 0's flag, which nothing publishes.  Every CTA's wait runs out
  // after wait_limit polls, records ST_SPIN_TIMEOUT and returns before it
  // writes anything; no access leaves the buffers (tiles 1 .. ntiles - 1 of
  // L and Linv).
  nl_status enqueue_solve_withheld(int* status) override {
    if (ntiles_ < 2) return NL_ERR_STATE;
    NL_CUDA(cudaMemsetAsync(flags_.p, 0, flags_.bytes, st_));
    set_int_kernel<<<1, 1, 0, st_>>>(flags_.as<int>(), 1);
    trsv_fwd_kernel<T><<<ntiles_ - 1, SV, trsv_smem<T>(), st_>>>(S_.as<T>(), ld_, ntiles_, Linv_.as<T>(), hop_.as<T>(),
                                                     bS_.as<double>(),
                                                     y_.as<double>(), flags_.as<int>(), flags_.as<int>() + 1, 1,
                                                     status, wait_limit, nullptr, nullptr);
    launches += 2;
    NL_CUDA(cudaGetLastError());
    return NL_OK;
  }

  // Right-looking blocked Cholesky with look-ahead.  After panel k is
  // factored (diagonal tile + TRSM below it), its trailing update is split:
  //   update A(k): block column k+1 (tiles (I, k+1), I >= k+1), main stream;
  //   update B(k): the triangle of tiles >= k+2, side stream,
  // so the factorisation of panel k+1 (which needs only A(k)) overlaps B(k).
  // A(k) waits for B(k-1) (both touch block column k+1); B(k) follows B(k-1)
  // on the side stream and waits for panel k.  The BF16 pack of panel k is
  // double-buffered.
  nl_status launch_update(int k, int t0, int nt, bool col_only, cudaStream_t st, int* status, const int* active) {
    nt = std::min(nt, env_end(k) - t0 + 1);  // tile rows past the envelope get zero updates
    if (nt <= 0) return NL_OK;
    if (sizeof(T) == 8 && precision_ == NL_PREC_FP64 && cublas_) {
      // Row-major lower storage = column-major upper.  X = rows >= r0 of
      // panel k; the column-major view of S is M(a, b) = S[b][a].
      double* Sd = reinterpret_cast<double*>(S_.p);
      const double alpha = -1.0, beta = 1.0;
      const size_t r0 = (size_t)t0 * NB, kc = (size_t)k * NB;
      const int n_rem = nt * NB;  // ld_ - r0 without the envelope
      // each stream has its own handle (and workspace)
      cublasHandle_t hb = (st == st_) ? cublas_ : cublas2_;
      if (cublasSetStream(hb, st) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
      if (col_only) {
        // M(c0.., r0..) -= Pc' Pr : C (128 x n_rem) with A = M(kc.., c0..), B = M(kc.., r0..)
        if (cublasDgemm(hb, CUBLAS_OP_T, CUBLAS_OP_N, NB, n_rem, NB, &alpha, Sd + r0 * ld_ + kc, ld_,
                        Sd + r0 * ld_ + kc, ld_, &beta, Sd + r0 * ld_ + r0, ld_) != CUBLAS_STATUS_SUCCESS)
          return NL_ERR_CUDA;
      } else {
        if (cublasDsyrk(hb, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, n_rem, NB, &alpha, Sd + r0 * ld_ + kc, ld_,
                        &beta, Sd + r0 * ld_ + r0, ld_) != CUBLAS_STATUS_SUCCESS)
          return NL_ERR_CUDA;
      }
    } else if (sizeof(T) == 4 && use_tc) {
      TcPacks pk{{pack_slot(k), nullptr, nullptr, nullptr}, 1};
      NL_CUDA(tc_update_f32(reinterpret_cast<float*>(S_.p), ld_, k, t0, nt, col_only ? 1 : 0, 0, pk, active, status,
                            st));
      launches++;
    } else {
      if (col_only) {
        // column block as a triangle of 1 plus rows below: reuse the tile kernel per row tile
        for (int I = 0; I < nt; I++)
          syrk_cc_tile_kernel<T><<<1, 256, 0, st>>>(S_.as<T>(), ld_, k, t0 + I, t0, active);
        launches += nt;
      } else {
        syrk_cc_kernel<T><<<nt * (nt + 1) / 2, 256, 0, st>>>(S_.as<T>(), ld_, k, t0, nt, active);
        launches++;
      }
    }
    return NL_OK;
  }

  nl_status factor_panel(int k, int* status, const int* active) {
    potrf_diag_kernel<T><<<1, PT, kPotrfSmem, st_>>>(S_.as<T>(), ld_, k, Linv_.as<T>(), status, active);
    launches++;
    const int below = std::min(ld_, (env_end(k) + 1) * NB) - (k + 1) * NB;  // rows past the envelope are zero
    if (below > 0) {
      trsm_kernel<T><<<cdiv(below, TRSM_ROWS), 256, trsm_smem<T>(), st_>>>(S_.as<T>(), ld_, k, (k + 1) * NB, below,
                                                                            Linv_.as<T>(), nullptr, active);
      launches++;
      if (sizeof(T) == 4 && use_tc) {
        NL_CUDA(tc_pack_f32(reinterpret_cast<const float*>(S_.p), ld_, k, 0, below, pack_slot(k), active, st_));
        launches++;
      }
    }
    return NL_OK;
  }

  // A kernel on the main stream; with pdl, as a programmatic dependent of the
  // stream's preceding kernel (it may start before that one ends and waits
  // for it with griddepcontrol.wait).
  template <typename... KArgs, typename... Args>
  cudaError_t launch_chain(void (*kern)(KArgs...), int grid, int block, size_t smem, bool pdl, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st_;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
  }

  uint8_t* pack_slot(int k) const { return static_cast<uint8_t*>(tcs_.p) + (size_t)(k % kPackSlots) * tcs_half_; }

  // Tensor-core schedule: panels in groups of G = kFactorGroup, so the bulk
  // of the trailing update has K = 128 G and every trailing tile is read and
  // written once per group instead of once per panel, and the panel work is
  // split so that only the chain
  //   potrf(j) -> TRSM + pack of row tile j+1 -> update of tile (j+1, j+1)
  //   -> potrf(j+1)
  // runs on the main stream; the rest of each step runs on the auxiliary
  // stream (top priority) or, for the bulk update, on the side stream (lowest
  // priority).  For the group of panels k .. k+G-1, after panel j is factored:
  //   j < k+G-1 (inside the group):
  //     main  tile (j+1, j+1) with panel j (K = 128); potrf(j+1); [wait the
  //           aux update] TRSM + pack of row tile j+2 of panel j+1
  //     aux   block columns j+1 (below its diagonal tile) .. k+G-1 with panel
  //           j; TRSM + pack of the rows below tile j+2 of panel j+1
  //   j = k+G-1 (the group's last panel):
  //     main  [wait B of the previous group] tile (k+G, k+G) with all G
  //           panels; potrf(k+G); [wait the aux update] TRSM + pack of row
  //           tile k+G+1
  //     aux   [wait B] block columns k+G (below its diagonal) .. k+2G-1 with
  //           all G panels; TRSM + pack of the rows below tile k+G+1
  //     side  B: tiles of block columns >= k+2G with all G panels.
  // (The tile updates of the chain are diag_update_kernel, the row-tile TRSMs
  // trsm_tile_kernel: NB / kChainRows CTAs each, FP32 on CUDA cores.)  Packs live in
  // kPackSlots = 2 G slots (panel mod 2 G): a group's B is the last reader of
  // its slots, and the group after next repacks them only after waiting for it.
  // With G = 2 this is the pair schedule (one B per two panels); G = 4 halves
  // the bulk update's HBM traffic again (rank-512 updates).
  enum { EV_PACKF = 0, EV_POTRF, EV_A1R, EV_PACKR, EV_A2R, EV_B, EV_AUX };
  nl_status enqueue_factor_groups(int* status, const int* active) {
    constexpr int G = kFactorGroup;
    const bool tm = timing && !active;
    const bool tmc = tm && timing_detail;  // per-panel chain events
    const int nT = ntiles_;
    // timing events: [0, 8 nT) updates, [8 nT, 10 nT) potrf, [10 nT, 14 nT)
    // per row tile: start (after its waits) and end of the TRSM and of the
    // diagonal-tile update
    if (tm && (int)upd_ev_.size() < 14 * nT + 10) {
      for (size_t i = upd_ev_.size(); i < (size_t)14 * nT + 10; i++) {
        cudaEvent_t e;
        NL_CUDA(cudaEventCreate(&e));
        upd_ev_.push_back(e);
      }
    }
    float* S = reinterpret_cast<float*>(S_.p);
    double upd_flop = 0, upd_bytes = 0;
    int nev = 0, nupd = 0;
    auto tiles_of = [](int nt, int ncols, int rb) {
      if (ncols <= 0) return (double)nt * (nt + 1) / 2;
      double t = 0;
      for (int j = 0; j < ncols && j < nt; j++) t += std::max(0, nt - std::max(j, rb));
      return t;
    };
    // update with panels k .. k + npan - 1
    auto upd = [&](int k, int npan, int t0, int nt, int ncols, int rb, cudaStream_t st) -> nl_status {
      nt = std::min(nt, env_end(k + npan - 1) - t0 + 1);  // tile rows past the envelope get zero updates
      if (nt <= 0 || tiles_of(nt, ncols, rb) <= 0) return NL_OK;
      if (tm) NL_CUDA(cudaEventRecord(upd_ev_[nev], st));
      TcPacks pk{{nullptr, nullptr, nullptr, nullptr}, npan};
      for (int i = 0; i < npan; i++) pk.p[i] = pack_slot(k + i);
      NL_CUDA(tc_update_f32(S, ld_, k, t0, nt, ncols, rb, pk, active, status, st));
      if (tm) NL_CUDA(cudaEventRecord(upd_ev_[nev + 1], st));
      nev += 2;
      nupd++;
      launches++;
      upd_bytes += tiles_of(nt, ncols, rb) * (double)NB * NB * sizeof(float) * 2;
      return NL_OK;
    };
    // TRSM + pack of panel j's rows [r0, r0 + nrows) (absolute rows, tile aligned)
    auto trsm_pack = [&](int j, int r0, int nrows, cudaStream_t st) -> nl_status {
      // rows past the envelope are zero in L; the pack covers every row that
      // an update of panel j's group reads (env_end of its last panel, at
      // most j + G - 1)
      nrows = std::min(nrows, (env_end(j + G - 1) + 1) * NB - r0);
      if (nrows <= 0) return NL_OK;
      // the TRSM writes the BF16 pack of its rows in its epilogue
      trsm_kernel<T><<<cdiv(nrows, TRSM_ROWS), 256, trsm_smem<T>(), st>>>(S_.as<T>(), ld_, j, r0, nrows,
                                                                           Linv_.as<T>(), pack_slot(j), active);
      launches++;
      return NL_OK;
    };
    // row tile j+1 of panel j (the critical one) and the diagonal-tile
    // updates: 32-CTA FP32 kernels on the main stream (kChainRows rows each)
    auto trsm_first = [&](int j) {
      if (tmc) cudaEventRecord(upd_ev_[10 * nT + 4 * j], st_);
      trsm_tile_kernel<kChainRows><<<NB / kChainRows, 256, kTrsmTileSmem, st_>>>(
          S, ld_, j, reinterpret_cast<const float*>(Linv_.p), pack_slot(j), active);
      if (tmc) cudaEventRecord(upd_ev_[10 * nT + 4 * j + 1], st_);
      launches++;
    };
    // pdl: launched early against the preceding kernel of the main stream
    // (only where no event wait sits between the two)
    auto diag_upd = [&](int t, int p0, int np, bool pdl) -> nl_status {
      if (tmc) cudaEventRecord(upd_ev_[10 * nT + 4 * (t - 1) + 2], st_);
      NL_CUDA(launch_chain(diag_update_kernel<kChainRows>, NB / kChainRows, 256, std::min(np, 2) * kDiagUpdSmem,
                           pdl && !tmc, S, ld_,
                           t, p0, np, active));
      if (tmc) cudaEventRecord(upd_ev_[10 * nT + 4 * (t - 1) + 3], st_);
      launches++;
      return NL_OK;
    };
    int npev = 0;
    auto potrf = [&](int j) -> nl_status {
      const int e = 8 * nT + 2 * j;  // timing events after the update events
      if (tmc) cudaEventRecord(upd_ev_[e], st_);
      // a programmatic dependent of the diagonal update before it
      NL_CUDA(launch_chain(potrf_diag_kernel<T>, 1, PT, kPotrfSmem, j > 0 && !tmc, S_.as<T>(), ld_, j,
                           Linv_.as<T>(), status, active));
      if (tmc) cudaEventRecord(upd_ev_[e + 1], st_);
      npev = j + 1;
      launches++;
      return NL_OK;
    };
    auto rec = [&](int e, cudaStream_t st) { return cudaEventRecord(dev_[e], st); };
    auto wait = [&](cudaStream_t st, int e) { return cudaStreamWaitEvent(st, dev_[e], 0); };
    for (int k = 0; k + 1 < nT; k++) {
      const double below = (double)ld_ - (double)(k + 1) * NB;
      upd_flop += (double)NB * below * (below + 1);
    }
    nl_status r;
    // panel 0
    if ((r = potrf(0)) != NL_OK) return r;
    if (nT > 1) trsm_first(0);
    NL_CUDA(rec(EV_POTRF, st_));
    NL_CUDA(wait(st3_, EV_POTRF));
    if ((r = trsm_pack(0, 2 * NB, ld_ - 2 * NB, st3_)) != NL_OK) return r;
    bool pending_b = false;
    for (int k = 0; k + 1 < nT; k += G) {
      const int g = std::min(G, nT - k);  // panels k .. k + g - 1 (the last group may be short)
      for (int i = 0; i < g; i++) {
        const int j = k + i;  // panel j is factored, row tile j+1 of it packed (main)
        if (j + 1 >= nT) break;
        NL_CUDA(rec(EV_PACKF, st_));
        if (i + 1 < g) {
          // inside the group: panel j -> block columns j+1 .. k+g-1
          if ((r = diag_upd(j + 1, j, 1, true)) != NL_OK) return r;
          NL_CUDA(wait(st3_, EV_PACKF));
          if ((r = upd(j, 1, j + 1, nT - j - 1, k + g - 1 - j, 1, st3_)) != NL_OK) return r;
          NL_CUDA(rec(EV_A1R, st3_));
          if ((r = potrf(j + 1)) != NL_OK) return r;
          NL_CUDA(rec(EV_POTRF, st_));
          NL_CUDA(wait(st3_, EV_POTRF));
          if ((r = trsm_pack(j + 1, (j + 3) * NB, ld_ - (j + 3) * NB, st3_)) != NL_OK) return r;
          NL_CUDA(rec(EV_PACKR, st3_));
          NL_CUDA(wait(st_, EV_A1R));
          if (j + 2 >= nT) break;
          trsm_first(j + 1);
        } else {
          // the group's last panel: the next group's block columns (main:
          // its first diagonal tile; aux: the rest), then the bulk (side)
          const int kn = k + g;  // first panel of the next group
          if (pending_b) NL_CUDA(wait(st_, EV_B));
          if ((r = diag_upd(kn, k, g, !pending_b)) != NL_OK) return r;
          NL_CUDA(wait(st3_, EV_PACKF));
          if (pending_b) NL_CUDA(wait(st3_, EV_B));
          if ((r = upd(k, g, kn, nT - kn, G, 1, st3_)) != NL_OK) return r;
          NL_CUDA(rec(EV_A2R, st3_));
          if (kn + G < nT) {
            NL_CUDA(wait(st2_, EV_PACKF));
            NL_CUDA(wait(st2_, EV_PACKR));
            if ((r = upd(k, g, kn + G, nT - kn - G, 0, 0, st2_)) != NL_OK) return r;  // B
            NL_CUDA(rec(EV_B, st2_));
            pending_b = true;
          } else {
            pending_b = false;
          }
          if ((r = potrf(kn)) != NL_OK) return r;
          NL_CUDA(rec(EV_POTRF, st_));
          NL_CUDA(wait(st3_, EV_POTRF));
          if ((r = trsm_pack(kn, (kn + 2) * NB, ld_ - (kn + 2) * NB, st3_)) != NL_OK) return r;
          NL_CUDA(rec(EV_PACKR, st3_));
          NL_CUDA(wait(st_, EV_A2R));
          if (kn + 1 < nT) trsm_first(kn);
        }
      }
    }
    // join: the solves that follow read every tile and Linv
    NL_CUDA(rec(EV_AUX, st3_));
    NL_CUDA(wait(st_, EV_AUX));
    if (pending_b) NL_CUDA(wait(st_, EV_B));
    if (tm) {
      NL_CUDA(cudaStreamSynchronize(st_));
      float tot = 0;
      for (int i = 0; i < nev; i += 2) {
        float ms = 0;
        cudaEventElapsedTime(&ms, upd_ev_[i], upd_ev_[i + 1]);
        tot += ms;
      }
      times.update_ms = tot;
      times.update_launches = nupd;
      times.update_flop = upd_flop;
      times.update_bytes = upd_bytes;
      float pt = 0;
      for (int j = 0; j < npev && tmc; j++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, upd_ev_[8 * nT + 2 * j], upd_ev_[8 * nT + 2 * j + 1]);
        pt += ms;
      }
      times.panel_ms = pt;
      times.panels = tmc ? npev : 0;
      // per row tile j+1: the waits for the other streams (potrf(j) end ->
      // TRSM start, TRSM end -> update start) and the two chain kernels
      float wt = 0, ft = 0;
      for (int j = 0; j + 1 < npev && tmc; j++) {
        const cudaEvent_t* e = &upd_ev_[10 * nT + 4 * j];
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, upd_ev_[8 * nT + 2 * j + 1], e[0]);
        cudaEventElapsedTime(&b, e[0], e[1]);
        cudaEventElapsedTime(&c, e[1], e[2]);
        cudaEventElapsedTime(&d, e[2], e[3]);
        wt += a + c;
        ft += b + d;
      }
      times.wait_ms = wt;
      times.first_ms = ft;
    }
    return NL_OK;
  }

  nl_status enqueue_factor(int* status, const int* active) {
    if (sizeof(T) == 4 && use_tc) return enqueue_factor_groups(status, active);
    const bool tm = timing && !active;
    if (tm && (int)upd_ev_.size() < 4 * ntiles_) {
      for (size_t i = upd_ev_.size(); i < (size_t)4 * ntiles_; i++) {
        cudaEvent_t e;
        NL_CUDA(cudaEventCreate(&e));
        upd_ev_.push_back(e);
      }
    }
    double upd_flop = 0;
    nl_status r;
    if ((r = factor_panel(0, status, active)) != NL_OK) return r;
    bool pending_b = false;
    for (int k = 0; k + 1 < ntiles_; k++) {
      const int below = ld_ - (k + 1) * NB;
      upd_flop += (double)NB * below * (below + 1);
      // panel k is factored and packed
      NL_CUDA(cudaEventRecord(ev_panel_, st_));
      // A(k): block column k+1, after B(k-1)
      if (pending_b) NL_CUDA(cudaStreamWaitEvent(st_, ev_b_, 0));
      if (tm) NL_CUDA(cudaEventRecord(upd_ev_[4 * k], st_));
      if ((r = launch_update(k, k + 1, ntiles_ - k - 1, true, st_, status, active)) != NL_OK) return r;
      if (tm) NL_CUDA(cudaEventRecord(upd_ev_[4 * k + 1], st_));
      // B(k): tiles >= k+2 on the side stream
      if (k + 2 < ntiles_) {
        NL_CUDA(cudaStreamWaitEvent(st2_, ev_panel_, 0));
        if (tm) NL_CUDA(cudaEventRecord(upd_ev_[4 * k + 2], st2_));
        if ((r = launch_update(k, k + 2, ntiles_ - k - 2, false, st2_, status, active)) != NL_OK) return r;
        if (tm) NL_CUDA(cudaEventRecord(upd_ev_[4 * k + 3], st2_));
        NL_CUDA(cudaEventRecord(ev_b_, st2_));
        pending_b = true;
      } else {
        pending_b = false;
      }
      if ((r = factor_panel(k + 1, status, active)) != NL_OK) return r;
    }
    if (pending_b) NL_CUDA(cudaStreamWaitEvent(st_, ev_b_, 0));
    if (cublas_) cublasSetStream(cublas_, st_);
    if (tm) {
      NL_CUDA(cudaStreamSynchronize(st_));
      float tot = 0;
      int nupd = 0;
      for (int k = 0; k + 1 < ntiles_; k++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, upd_ev_[4 * k], upd_ev_[4 * k + 1]);
        tot += ms;
        if (k + 2 < ntiles_) {
          cudaEventElapsedTime(&ms, upd_ev_[4 * k + 2], upd_ev_[4 * k + 3]);
          tot += ms;
        }
        nupd++;
      }
      times.update_ms = tot;
      times.update_launches = nupd;
      times.update_flop = upd_flop;
      // tiles read and written per panel: block column k+1 and the triangle
      // below it, both cut at the envelope (launch_update's clipping)
      double tiles = 0;
      for (int k = 0; k + 1 < ntiles_; k++) {
        const int last = env_end(k);
        const double na = std::max(0, last - k), nb = std::max(0, last - k - 1);
        tiles += na + nb * (nb + 1) / 2;
      }
      times.update_bytes = tiles * (double)NB * NB * sizeof(T) * 2;
    }
    return NL_OK;
  }

  nl_status enqueue_increment(const double* lam, int* status, const int* active) override {
    const bool tm = timing && !active;
    NvtxRange rg("nl:computeIncrement");
    if (tm) NL_CUDA(cudaEventRecord(ev_[0], st_));
    nvtxRangePushA("nl:vinv+wvinv_bs");
    vinv_kernel<T, BC><<<cdiv(std::max(np_, 1), 128), 128, 0, st_>>>(d_, V_.as<T>(), Vinv_.as<T>(), lam, status, active);
    if (tm) NL_CUDA(cudaEventRecord(ev_[1], st_));
    if (nci_ > 0)
      wvinv_bs_kernel<T, BC, 128><<<nci_, 128, 0, st_>>>(d_, W_.as<T>(), Vinv_.as<T>(), Y_.as<T>(), bU_.as<T>(),
                                                         bV_.as<T>(), bS_.as<double>(), active);
    if (tm) NL_CUDA(cudaEventRecord(ev_[2], st_));
    nvtxRangePop();
    nvtxRangePushA("nl:schur");
    // The first time the whole of S (and S0); afterwards only the envelope,
    // whose outside stays exactly zero -- but only where every kernel that
    // writes S honours `active`.  The FP64 path's cuBLAS trailing updates
    // cannot: the sub-iterations that a device-side LM loop leaves in flight
    // after it has finished still subtract L L' from the stale factor, and the
    // overflow that builds up there reaches tiles outside the envelope
    // (0 * inf).  That path clears all of S every time.
    const bool unpredicated_writes = sizeof(T) == 8 && cublas_ != nullptr;
    if (!s_cleared_ || unpredicated_writes) {
      NL_CUDA(cudaMemsetAsync(S_.p, 0, S_.bytes, st_));
      if (need_s0_) NL_CUDA(cudaMemsetAsync(S0_.p, 0, S0_.bytes, st_));
      s_cleared_ = true;
    } else {
      clear_envelope_kernel<T><<<ld_, 128, 0, st_>>>(S_.as<T>(), need_s0_ ? S0_.as<T>() : nullptr, ld_, NB,
                                                     env_dev_.as<int>(), active);
      launches++;
    }
    {
      const int grid = std::max(1, std::min(cdiv(nS_, kSchurWarps), 148 * 8));
      NL_CUDA(cudaMemsetAsync(sched_.p, 0, sizeof(int), st_));
      schur_kernel<T, BC, kSchurWarps><<<grid, kSchurWarps * 32, 0, st_>>>(
          d_, U_.as<T>(), Y_.as<T>(), W_.as<T>(), lam, S_.as<T>(), need_s0_ ? S0_.as<T>() : nullptr,
          s_order_.as<int>(), sched_.as<int>(), active);
      if (ld_ > n_)
        pad_identity_kernel<T><<<cdiv(ld_ - n_, 128), 128, 0, st_>>>(S_.as<T>(), need_s0_ ? S0_.as<T>() : nullptr, n_,
                                                                     ld_, active);
    }
    launches += 4;
    nvtxRangePop();
    if (tm) NL_CUDA(cudaEventRecord(ev_[3], st_));
    nl_status s;
    {
      NvtxRange r("nl:factorize");
      s = enqueue_factor(status, active);
      // the hop matrices of the solves (M_d,I, Q_d,I)
      if (s == NL_OK && ntiles_ > 1) {
        hop_mat_kernel<T><<<dim3(ntiles_ - 1, 2 * kHopDepth), 256, 0, st_>>>(S_.as<T>(), ld_, ntiles_, Linv_.as<T>(),
                                                                             hop_.as<T>(), active);
        launches++;
      }
    }
    if (s != NL_OK) return s;
    if (tm) NL_CUDA(cudaEventRecord(ev_[4], st_));
    NvtxRange rs("nl:solve+backsub");
    if ((s = enqueue_solve(bS_.as<double>(), incU, status, active)) != NL_OK) return s;
    for (int it = 0; it < refine_sweeps && need_s0_; it++) {
      symv_partial_kernel<T, kSymvChunks><<<dim3(ntiles_, kSymvChunks), SV, 0, st_>>>(
          S0_.as<T>(), ld_, ntiles_, incU, part_.as<double>(), active);
      resid_finalize_kernel<kSymvChunks><<<cdiv(ld_, 256), 256, 0, st_>>>(part_.as<double>(), bS_.as<double>(), ld_,
                                                                          r_.as<double>(), active);
      if ((s = enqueue_solve(r_.as<double>(), dx_.as<double>(), status, active)) != NL_OK) return s;
      axpy_kernel<<<cdiv(ld_, 256), 256, 0, st_>>>(incU, dx_.as<double>(), ld_, active);
      launches += 3;
    }
    if (tm) NL_CUDA(cudaEventRecord(ev_[5], st_));
    zero_if_failed_kernel<<<cdiv(ld_, 256), 256, 0, st_>>>(incU, ld_, status, active);
    backsub_kernel<T, BC><<<cdiv(std::max(np_, 1), 128), 128, 0, st_>>>(d_, W_.as<T>(), Vinv_.as<T>(), bV_.as<T>(),
                                                                      incU, incV, status, active);
    launches += 2;
    if (tm) NL_CUDA(cudaEventRecord(ev_[6], st_));
    NL_CUDA(cudaGetLastError());
    if (tm) {
      NL_CUDA(cudaEventSynchronize(ev_[6]));
      float ms[6];
      for (int i = 0; i < 6; i++) cudaEventElapsedTime(&ms[i], ev_[i], ev_[i + 1]);
      times.vinv_ms = ms[0];
      times.wvinv_bs_ms = ms[1];
      times.schur_ms = ms[2];
      times.factor_ms = ms[3];
      times.solve_ms = ms[4];
      times.backsub_ms = ms[5];
      cudaEventElapsedTime(&times.total_ms, ev_[0], ev_[6]);
    }
    return NL_OK;
  }

  nl_status enqueue_resolve(int* status) override {
    if (nci_ > 0)
      wvinv_bs_kernel<T, BC, 128><<<nci_, 128, 0, st_>>>(d_, W_.as<T>(), Vinv_.as<T>(), Y_.as<T>(), bU_.as<T>(),
                                                         bV_.as<T>(), bS_.as<double>(), nullptr);
    launches++;
    nl_status s = enqueue_solve(bS_.as<double>(), incU, status, nullptr);
    if (s != NL_OK) return s;
    for (int it = 0; it < refine_sweeps && need_s0_; it++) {
      symv_partial_kernel<T, kSymvChunks><<<dim3(ntiles_, kSymvChunks), SV, 0, st_>>>(
          S0_.as<T>(), ld_, ntiles_, incU, part_.as<double>(), nullptr);
      resid_finalize_kernel<kSymvChunks><<<cdiv(ld_, 256), 256, 0, st_>>>(part_.as<double>(), bS_.as<double>(), ld_,
                                                                          r_.as<double>(), nullptr);
      if ((s = enqueue_solve(r_.as<double>(), dx_.as<double>(), status, nullptr)) != NL_OK) return s;
      axpy_kernel<<<cdiv(ld_, 256), 256, 0, st_>>>(incU, dx_.as<double>(), ld_, nullptr);
      launches += 3;
    }
    zero_if_failed_kernel<<<cdiv(ld_, 256), 256, 0, st_>>>(incU, ld_, status, nullptr);
    backsub_kernel<T, BC><<<cdiv(std::max(np_, 1), 128), 128, 0, st_>>>(d_, W_.as<T>(), Vinv_.as<T>(), bV_.as<T>(),
                                                                      incU, incV, status, nullptr);
    launches += 2;
    NL_CUDA(cudaGetLastError());
    return NL_OK;
  }

  nl_status enqueue_hdiag(double* out) override {
    const int grid = std::max(1, std::min(kRedCTAs, cdiv(nci_ + np_, 256)));
    hdiag_kernel<T, BC><<<grid, 256, 0, st_>>>(U_.as<T>(), d_.u_diag_uid, nci_, V_.as<T>(), d_.v_uid, np_,
                                               part_.as<double>());
    max_finalize_kernel<<<1, 1, 0, st_>>>(part_.as<double>(), grid, out, nullptr);
    launches += 2;
    NL_CUDA(cudaGetLastError());
    return NL_OK;
  }

  nl_status enqueue_maxabs_b(double* out, const int* active) override {
    const int grid = std::max(1, std::min(kRedCTAs, cdiv(n_ + 3 * np_, kNT)));
    maxabs_kernel<T, kNT><<<grid, kNT, 0, st_>>>(bU_.as<T>(), n_, bV_.as<T>(), 3 * np_, part_.as<double>(), active);
    max_finalize_kernel<<<1, 1, 0, st_>>>(part_.as<double>(), grid, out, active);
    launches += 2;
    NL_CUDA(cudaGetLastError());
    return NL_OK;
  }

  nl_status enqueue_inc_dot(const LmDev* s, double* part, int* nparts) override {
    const int grid = std::max(1, std::min(kRedCTAs, cdiv(n_ + 3 * np_, kNT)));
    inc_dot_kernel<T, kNT><<<grid, kNT, 0, st_>>>(incU, bU_.as<T>(), n_, incV, bV_.as<T>(), 3 * np_, s, part);
    *nparts = grid;
    launches++;
    NL_CUDA(cudaGetLastError());
    return NL_OK;
  }

  // ---- host transfers (tests / solver-only API) ----
  template <typename A, typename B>
  static void conv(const A* src, B* dst, size_t nblk, int bs, int sstride, int dstride) {
    for (size_t q = 0; q < nblk; q++)
      for (int i = 0; i < bs; i++) dst[q * dstride + i] = (B)src[q * sstride + i];
  }

  nl_status get_hessian(double* U, double* V, double* W, double* bU, double* bV) override {
    NL_CUDA(cudaStreamSynchronize(st_));
    auto fetch = [&](const DevBuf& b, size_t nblk, int bs, int stride, double* out) -> nl_status {
      if (!out || nblk == 0) return NL_OK;
      std::vector<T> h(nblk * stride);
      NL_CUDA(cudaMemcpy(h.data(), b.p, h.size() * sizeof(T), cudaMemcpyDeviceToHost));
      conv(h.data(), out, nblk, bs, stride, bs);
      return NL_OK;
    };
    nl_status s;
    if ((s = fetch(U_, nU_, BC * BC, Layout<T, BC>::U, U)) != NL_OK) return s;
    if ((s = fetch(V_, nV_, 9, Layout<T, BC>::V, V)) != NL_OK) return s;
    if ((s = fetch(W_, nW_, BC * 3, Layout<T, BC>::W, W)) != NL_OK) return s;
    if ((s = fetch(bU_, 1, n_, n_, bU)) != NL_OK) return s;
    if ((s = fetch(bV_, 1, 3 * np_, 3 * np_, bV)) != NL_OK) return s;
    return NL_OK;
  }

  nl_status set_hessian(const double* U, const double* V, const double* W, const double* bU,
                        const double* bV) override {
    auto put = [&](DevBuf& b, size_t nblk, int bs, int stride, const double* in) -> nl_status {
      if (!in || nblk == 0) return NL_OK;
      std::vector<T> h(nblk * stride, (T)0);
      conv(in, h.data(), nblk, bs, bs, stride);
      NL_CUDA(cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st_));
      NL_CUDA(cudaStreamSynchronize(st_));
      return NL_OK;
    };
    nl_status s;
    if ((s = put(U_, nU_, BC * BC, Layout<T, BC>::U, U)) != NL_OK) return s;
    if ((s = put(V_, nV_, 9, Layout<T, BC>::V, V)) != NL_OK) return s;
    if ((s = put(W_, nW_, BC * 3, Layout<T, BC>::W, W)) != NL_OK) return s;
    if ((s = put(bU_, 1, n_, n_, bU)) != NL_OK) return s;
    if ((s = put(bV_, 1, 3 * np_, 3 * np_, bV)) != NL_OK) return s;
    return NL_OK;
  }

  nl_status get_schur(double* S, double* bS) override {
    if (!need_s0_) return NL_ERR_STATE;
    NL_CUDA(cudaStreamSynchronize(st_));
    std::vector<T> h((size_t)ld_ * ld_);
    NL_CUDA(cudaMemcpy(h.data(), S0_.p, h.size() * sizeof(T), cudaMemcpyDeviceToHost));
    if (S) {
      // reference layout: upper triangle of S (row i, col j >= i) = lower[j][i]
      for (int i = 0; i < n_; i++)
        for (int j = 0; j < n_; j++) S[(size_t)i * n_ + j] = j >= i ? (double)h[(size_t)j * ld_ + i] : 0.0;
    }
    if (bS) NL_CUDA(cudaMemcpy(bS, bS_.p, sizeof(double) * n_, cudaMemcpyDeviceToHost));
    return NL_OK;
  }

 private:
  cublasHandle_t cublas_;
  int precision_;
  cudaStream_t st_ = nullptr;
  int nci_ = 0, np_ = 0, nU_ = 0, nV_ = 0, nW_ = 0, nS_ = 0, n_ = 0, ld_ = 0, ntiles_ = 0;
  long long npairs_ = 0;
  bool need_s0_ = false;
  SchurDev d_{};
  DevBuf U_, V_, W_, Y_, Vinv_, bU_, bV_, bS_, incU_, incV_, y_, r_, dx_, part_, Linv_, hop_, flags_, S_, S0_, tcs_;
  // envelope of S (host) and its first / last arrays on the device (solves)
  std::vector<int> env_first_, env_last_, env_run_;
  DevBuf env_dev_;
  bool s_cleared_ = false;  // S / S0 have had their one full clear (enqueue_increment)
  // last tile row that panel k's TRSM and updates must cover
  int env_end(int k) const { return envelope ? env_run_[std::min(k, ntiles_ - 1)] : ntiles_ - 1; }
  DevBuf v_uid_, w_row_ptr_, w_col_, w_row_, w_col_ptr_, w_col_uid_, u_diag_, s_i_, s_j_, s_uuid_, s_ptr_, pa_, pb_, s_order_,
      sched_;
  cudaEvent_t ev_[7] = {};
  cudaEvent_t ev_panel_ = nullptr, ev_b_ = nullptr;
  cudaStream_t st2_ = nullptr;  // side stream of the look-ahead factorisation
  cudaStream_t st3_ = nullptr;  // auxiliary stream of the tensor-core schedule
  cudaEvent_t dev_[8] = {};     // dependency events of the tensor-core schedule
  cublasHandle_t cublas2_ = nullptr;
  DevBuf ws2_;
  size_t tcs_half_ = 0;
  static constexpr int kFactorGroup = 4;  // panels per bulk trailing update (K = 512)
  static constexpr int kPackSlots = 2 * kFactorGroup;
  std::vector<cudaEvent_t> upd_ev_;

 public:
  ~SchurCoreT() override {
    if (cublas2_) cublasDestroy(cublas2_);
    if (st2_) {
      cudaStreamSynchronize(st2_);
      cudaStreamDestroy(st2_);
    }
    if (st3_) {
      cudaStreamSynchronize(st3_);
      cudaStreamDestroy(st3_);
    }
    for (auto e : dev_)
      if (e) cudaEventDestroy(e);
    for (auto e : ev_)
      if (e) cudaEventDestroy(e);
    if (ev_panel_) cudaEventDestroy(ev_panel_);
    if (ev_b_) cudaEventDestroy(ev_b_);
    for (auto e : upd_ev_) cudaEventDestroy(e);
  }
};

}  // namespace

std::unique_ptr<SchurCore> make_schur_core(int precision, int bc, cublasHandle_t cublas) {
  const bool f64 = precision == NL_PREC_FP64;
#define NL_MK(B)                                                          \
  case B:                                                                 \
    if (f64) return std::unique_ptr<SchurCore>(new SchurCoreT<double, B>(cublas, precision)); \
    return std::unique_ptr<SchurCore>(new SchurCoreT<float, B>(cublas, precision));
  switch (bc) {
    NL_MK(2)
    NL_MK(3)
    NL_MK(6)
    NL_MK(9)
    default:
      return nullptr;
  }
#undef NL_MK
}

}  // namespace nl

// ---------------------------------------------------------------------------
namespace nl {
namespace {
__global__ void selftest_fill_kernel(float* S, size_t n, unsigned long long seed) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  S[i] = (float)((double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5);
}
}  // namespace
}  // namespace nl

extern "C" nl_status nl_selftest_tc_update(int ntiles, unsigned long long seed, int device, double* max_rel_err) {
  using namespace nl;
  if (ntiles < 2 || ntiles > 64 || !max_rel_err) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(device));
  const int ld = ntiles * NB;
  const size_t n = (size_t)ld * ld;
  DevBuf a, b, scratch, st;
  nl_status r;
  if ((r = a.alloc(n * 4)) != NL_OK || (r = b.alloc(n * 4)) != NL_OK ||
      (r = scratch.alloc(tc_syrk_scratch_bytes(ld))) != NL_OK || (r = st.alloc(16)) != NL_OK)
    return r;
  NL_CUDA(cudaMemset(st.p, 0, 16));
  selftest_fill_kernel<<<(unsigned)((n + 255) / 256), 256>>>(a.as<float>(), n, seed);
  NL_CUDA(cudaMemcpy(b.p, a.p, n * 4, cudaMemcpyDeviceToDevice));
  const int nt = ntiles - 1;
  NL_CUDA(tc_syrk_f32(a.as<float>(), ld, 0, 1, nt, scratch.p, nullptr, st.as<int>(), 0));
  syrk_cc_kernel<float><<<nt * (nt + 1) / 2, 256>>>(b.as<float>(), ld, 0, 1, nt, nullptr);
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaDeviceSynchronize());
  int stat = 0;
  NL_CUDA(cudaMemcpy(&stat, st.p, 4, cudaMemcpyDeviceToHost));
  if (stat & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  std::vector<float> ha(n), hb(n);
  NL_CUDA(cudaMemcpy(ha.data(), a.p, n * 4, cudaMemcpyDeviceToHost));
  NL_CUDA(cudaMemcpy(hb.data(), b.p, n * 4, cudaMemcpyDeviceToHost));
  double md = 0, mb = 0;
  for (int i = NB; i < ld; i++)
    for (int j = NB; j <= i; j++) {
      const double x = ha[(size_t)i * ld + j], y = hb[(size_t)i * ld + j];
      md = std::max(md, std::fabs(x - y));
      mb = std::max(mb, std::fabs(y));
    }
  *max_rel_err = md / std::max(mb, 1e-300);
  return NL_OK;
}

// Self-test and in-isolation timing of the rank-K update the factorisation's
// groups use: panels 0 .. np-1 of a random FP32 matrix are packed and applied
// to the trailing tiles np .. ntiles-1 in one launch (K = 128 np), checked
// against the CUDA-core update applied panel by panel, then timed over
// `reps` further launches (best, CUDA events).
extern "C" nl_status nl_selftest_tc_update_k(int ntiles, int np, unsigned long long seed, int device, int reps,
                                             double* max_rel_err, double* best_ms) {
  using namespace nl;
  if (ntiles < 2 || ntiles > 96 || np < 1 || np > kTcMaxPanels || np >= ntiles || reps < 0 || !max_rel_err)
    return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(device));
  NL_CUDA(tc_prepare());
  const int ld = ntiles * NB;
  const size_t n = (size_t)ld * ld;
  const size_t slot = tc_syrk_scratch_bytes(ld);
  DevBuf a, b, packs, st;
  nl_status r;
  if ((r = a.alloc(n * 4)) != NL_OK || (r = b.alloc(n * 4)) != NL_OK ||
      (r = packs.alloc(slot * (size_t)np)) != NL_OK || (r = st.alloc(16)) != NL_OK)
    return r;
  NL_CUDA(cudaMemset(st.p, 0, 16));
  selftest_fill_kernel<<<(unsigned)((n + 255) / 256), 256>>>(a.as<float>(), n, seed);
  NL_CUDA(cudaMemcpy(b.p, a.p, n * 4, cudaMemcpyDeviceToDevice));
  TcPacks pk{{nullptr, nullptr, nullptr, nullptr}, np};
  for (int i = 0; i < np; i++) {
    pk.p[i] = static_cast<uint8_t*>(packs.p) + slot * (size_t)i;
    NL_CUDA(tc_pack_f32(a.as<float>(), ld, i, 0, ld - (i + 1) * NB, const_cast<void*>(pk.p[i]), nullptr, 0));
  }
  const int t0 = np, nt = ntiles - np;
  NL_CUDA(tc_update_f32(a.as<float>(), ld, 0, t0, nt, 0, 0, pk, nullptr, st.as<int>(), 0));
  for (int i = 0; i < np; i++) syrk_cc_kernel<float><<<nt * (nt + 1) / 2, 256>>>(b.as<float>(), ld, i, t0, nt, nullptr);
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaDeviceSynchronize());
  int stat = 0;
  NL_CUDA(cudaMemcpy(&stat, st.p, 4, cudaMemcpyDeviceToHost));
  if (stat & ST_SPIN_TIMEOUT) return NL_ERR_TIMEOUT;
  std::vector<float> ha(n), hb(n);
  NL_CUDA(cudaMemcpy(ha.data(), a.p, n * 4, cudaMemcpyDeviceToHost));
  NL_CUDA(cudaMemcpy(hb.data(), b.p, n * 4, cudaMemcpyDeviceToHost));
  double md = 0, mb = 0;
  for (int i = t0 * NB; i < ld; i++)
    for (int j = t0 * NB; j <= i; j++) {
      const double x = ha[(size_t)i * ld + j], y = hb[(size_t)i * ld + j];
      md = std::max(md, std::fabs(x - y));
      mb = std::max(mb, std::fabs(y));
    }
  *max_rel_err = md / std::max(mb, 1e-300);
  if (best_ms) {
    double best = 0.0;
    cudaEvent_t e0, e1;
    NL_CUDA(cudaEventCreate(&e0));
    NL_CUDA(cudaEventCreate(&e1));
    for (int k = 0; k < reps; k++) {
      NL_CUDA(cudaEventRecord(e0, 0));
      NL_CUDA(tc_update_f32(a.as<float>(), ld, 0, t0, nt, 0, 0, pk, nullptr, st.as<int>(), 0));
      NL_CUDA(cudaEventRecord(e1, 0));
      NL_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      best = (k == 0) ? ms : std::min(best, (double)ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *best_ms = best;
  }
  return NL_OK;
}

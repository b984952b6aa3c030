// ordering.cu -- approximate minimum degree ordering (host code).
//
// Replaces Eigen::AMDOrdering<int> as called by DoubleSection::permuteAMD_SchurU
// (nelson/DoubleSection.hpp:30-63, on the pattern triu(spU + spW spW')) and by
// SingleSection::permuteAMD (nelson/SingleSection.hpp:33-52).  The algorithm is
// the approximate minimum degree ordering of Amestoy, Davis & Duff (SIAM J.
// Matrix Anal. Appl. 17(4), 1996), restated here on a quotient graph:
//   * variables (not yet eliminated) keep a list A_i of variable neighbours
//     and a list E_i of adjacent elements; an element e (an eliminated pivot)
//     keeps the list L_e of the variables it connects;
//   * the pivot is the variable of least approximate external degree (ties:
//     lowest index); its element L_p = (A_p u the L_e of its elements) \ p
//     absorbs those elements;
//   * for each i in L_p the edges now covered by L_p are pruned from A_i, and
//     the approximate degree is
//         d_i = min(n_left - |i|, d_i_old + |L_p \ i|,
//                   |A_i| + |L_p \ i| + sum_{e in E_i, e != p} |L_e \ L_p|),
//     with |L_e \ L_p| found by one scan over the elements of L_p's variables;
//     an element with L_e inside L_p is absorbed (aggressive absorption);
//   * variables of L_p with the same A_i and E_i are merged into one
//     supervariable (found through a hash of the two lists), and a variable
//     left with A_i empty and E_i = {p} is eliminated together with p (mass
//     elimination);
//   * dense rows (degree above max(16, 10 sqrt(n)), at most n - 2) are taken
//     out first and ordered last, as the published algorithm does.
// Sizes |.| count supervariable weights.  The result is deterministic.  It is
// not claimed to reproduce Eigen's permutation entry for entry (tie-breaking
// and absorption details differ between AMD codes); what it shares with them
// is the fill it leads to, which the tests compare with reverse Cuthill-McKee
// and with an exact minimum degree ordering.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <set>
#include <unordered_map>
#include <vector>

#include "nl_common.cuh"
#include "problem_view.h"

namespace {

struct AmdGraph {
  int n = 0;
  std::vector<std::vector<int>> A, E, L;
  std::vector<int> nv, deg, merged_into;
  std::vector<char> elim, elem_alive;
};

// perm[i] = position of node i in the elimination order.
void amd_order(int n, const std::vector<std::vector<int>>& adj_in, int* perm) {
  if (n <= 0) return;
  AmdGraph g;
  g.n = n;
  g.A.resize(n);
  g.E.resize(n);
  g.L.resize(n);
  g.nv.assign(n, 1);
  g.deg.assign(n, 0);
  g.merged_into.assign(n, -1);
  g.elim.assign(n, 0);
  g.elem_alive.assign(n, 0);
  for (int i = 0; i < n; i++) {
    std::vector<int>& a = g.A[i];
    a = adj_in[i];
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    a.erase(std::remove(a.begin(), a.end(), i), a.end());
  }
  // dense rows: out of the graph, last in the order
  int dense = std::max(16, (int)(10.0 * std::sqrt((double)n)));
  dense = std::min(n - 2, dense);
  std::vector<char> is_dense(n, 0);
  std::vector<int> dense_nodes;
  if (n > 2)
    for (int i = 0; i < n; i++)
      if ((int)g.A[i].size() > dense) {
        is_dense[i] = 1;
        dense_nodes.push_back(i);
      }
  if (!dense_nodes.empty())
    for (int i = 0; i < n; i++) {
      std::vector<int>& a = g.A[i];
      a.erase(std::remove_if(a.begin(), a.end(), [&](int j) { return is_dense[j] != 0; }), a.end());
    }
  std::set<std::pair<int, int>> bucket;  // (approximate degree, node)
  int n_left = 0;
  for (int i = 0; i < n; i++)
    if (!is_dense[i]) {
      g.deg[i] = (int)g.A[i].size();
      bucket.insert({g.deg[i], i});
      n_left++;
    }
  // elimination sequence: pivots, each followed by the variables that leave
  // with it (mass elimination); supervariable members are expanded at the end
  std::vector<int> seq;
  seq.reserve(n);
  std::vector<int> stamp(n, -1), wgt(n, 0), wstamp(n, -1);
  std::vector<int> Lp;
  int step = 0;
  auto alive_var = [&](int j) { return !g.elim[j] && g.nv[j] > 0 && !is_dense[j]; };
  while (!bucket.empty()) {
    const int p = bucket.begin()->second;
    bucket.erase(bucket.begin());
    step++;
    // ---- the element L_p ----
    Lp.clear();
    stamp[p] = step;
    for (int e : g.E[p]) {
      if (!g.elem_alive[e]) continue;
      for (int i : g.L[e])
        if (alive_var(i) && stamp[i] != step) {
          stamp[i] = step;
          Lp.push_back(i);
        }
      g.elem_alive[e] = 0;  // absorbed into p
      std::vector<int>().swap(g.L[e]);
    }
    for (int i : g.A[p])
      if (alive_var(i) && stamp[i] != step) {
        stamp[i] = step;
        Lp.push_back(i);
      }
    std::sort(Lp.begin(), Lp.end());
    g.elim[p] = 1;
    g.elem_alive[p] = 1;
    std::vector<int>().swap(g.A[p]);
    std::vector<int>().swap(g.E[p]);
    seq.push_back(p);
    n_left -= g.nv[p];
    int lp_w = 0;
    for (int i : Lp) lp_w += g.nv[i];
    // ---- element and adjacency lists of L_p's variables ----
    for (int i : Lp) {
      bucket.erase({g.deg[i], i});
      std::vector<int>& Ei = g.E[i];
      Ei.erase(std::remove_if(Ei.begin(), Ei.end(), [&](int e) { return !g.elem_alive[e]; }), Ei.end());
      Ei.push_back(p);
      std::vector<int>& Ai = g.A[i];
      Ai.erase(std::remove_if(Ai.begin(), Ai.end(), [&](int j) { return stamp[j] == step || !alive_var(j); }),
               Ai.end());
    }
    // ---- |L_e \ L_p| for the other elements of L_p's variables ----
    for (int i : Lp)
      for (int e : g.E[i]) {
        if (e == p || wstamp[e] == step) continue;
        wstamp[e] = step;
        std::vector<int>& Le = g.L[e];
        Le.erase(std::remove_if(Le.begin(), Le.end(), [&](int j) { return !alive_var(j); }), Le.end());
        int w = 0;
        for (int j : Le)
          if (stamp[j] != step) w += g.nv[j];
        wgt[e] = w;
        if (w == 0) {  // aggressive absorption: L_e lies inside L_p
          g.elem_alive[e] = 0;
          std::vector<int>().swap(Le);
        }
      }
    // ---- approximate degrees ----
    for (int i : Lp) {
      std::vector<int>& Ei = g.E[i];
      Ei.erase(std::remove_if(Ei.begin(), Ei.end(), [&](int e) { return !g.elem_alive[e]; }), Ei.end());
      long long d = lp_w - g.nv[i];
      for (int j : g.A[i]) d += g.nv[j];
      for (int e : Ei)
        if (e != p) d += wgt[e];
      d = std::min<long long>(d, (long long)g.deg[i] + lp_w - g.nv[i]);
      d = std::min<long long>(d, (long long)n_left - g.nv[i]);
      g.deg[i] = (int)std::max<long long>(d, 0);
    }
    // ---- supervariables: same A_i and E_i ----
    std::unordered_map<uint64_t, std::vector<int>> groups;
    std::vector<uint64_t> hash(Lp.size());
    for (size_t q = 0; q < Lp.size(); q++) {
      const int i = Lp[q];
      std::sort(g.A[i].begin(), g.A[i].end());
      std::sort(g.E[i].begin(), g.E[i].end());
      uint64_t h = 1469598103934665603ull;  // FNV-1a over both lists
      for (int j : g.A[i]) h = (h ^ (uint64_t)(j + 1)) * 1099511628211ull;
      h = (h ^ 0x9e3779b97f4a7c15ull) * 1099511628211ull;
      for (int e : g.E[i]) h = (h ^ (uint64_t)(e + 1)) * 1099511628211ull;
      hash[q] = h;
      groups[h].push_back(i);
    }
    for (size_t q = 0; q < Lp.size(); q++) {
      const int i = Lp[q];
      if (g.nv[i] == 0) continue;
      for (int j : groups[hash[q]]) {
        if (j <= i || g.nv[j] == 0) continue;
        if (g.A[j] != g.A[i] || g.E[j] != g.E[i]) continue;
        g.nv[i] += g.nv[j];
        g.deg[i] -= g.nv[j];
        g.nv[j] = 0;
        g.merged_into[j] = i;
        std::vector<int>().swap(g.A[j]);
        std::vector<int>().swap(g.E[j]);
      }
    }
    // ---- mass elimination, then back into the degree order ----
    std::vector<int>& Lnew = g.L[p];
    for (int i : Lp) {
      if (g.nv[i] == 0) continue;
      if (g.A[i].empty() && g.E[i].size() == 1 && g.E[i][0] == p) {
        g.elim[i] = 1;
        n_left -= g.nv[i];
        seq.push_back(i);
        std::vector<int>().swap(g.E[i]);
        continue;
      }
      g.deg[i] = std::max(0, std::min(g.deg[i], n_left - g.nv[i]));
      bucket.insert({g.deg[i], i});
      Lnew.push_back(i);
    }
    if (Lnew.empty()) g.elem_alive[p] = 0;
  }
  // expand supervariables: each principal variable, then what merged into it
  std::vector<std::vector<int>> members(n);
  for (int j = 0; j < n; j++)
    if (g.merged_into[j] >= 0) members[g.merged_into[j]].push_back(j);
  int pos = 0;
  std::vector<int> stack;
  for (int v : seq) {
    stack.assign(1, v);
    while (!stack.empty()) {
      const int x = stack.back();
      stack.pop_back();
      perm[x] = pos++;
      for (auto it = members[x].rbegin(); it != members[x].rend(); ++it) stack.push_back(*it);
    }
  }
  for (int v : dense_nodes) perm[v] = pos++;
}

}  // namespace

extern "C" {

nl_status nl_amd_order(int n, int nnz, const int* row, const int* col, int* perm) {
  if (n < 0 || nnz < 0 || !perm || (nnz > 0 && (!row || !col))) return NL_ERR_ARG;
  for (int k = 0; k < nnz; k++)
    if (row[k] < 0 || row[k] >= n || col[k] < 0 || col[k] >= n) return NL_ERR_ARG;
  std::vector<std::vector<int>> adj(n);
  for (int k = 0; k < nnz; k++)
    if (row[k] != col[k]) {
      adj[row[k]].push_back(col[k]);
      adj[col[k]].push_back(row[k]);
    }
  amd_order(n, adj, perm);
  return NL_OK;
}

nl_status nl_amd_order_camera_graph(int nc, int np, int ne, const int* cam, const int* pt, int* perm) {
  if (nc < 0 || np < 0 || ne < 0 || !perm || (ne > 0 && (!cam || !pt))) return NL_ERR_ARG;
  for (int e = 0; e < ne; e++)
    if (cam[e] < 0 || cam[e] >= nc || pt[e] < 0 || pt[e] >= np) return NL_ERR_ARG;
  // the pattern of U + W W': cameras that observe a common point
  std::vector<std::vector<int>> by_pt(np);
  for (int e = 0; e < ne; e++) by_pt[pt[e]].push_back(cam[e]);
  std::vector<std::vector<int>> adj(nc);
  for (auto& cs : by_pt) {
    std::sort(cs.begin(), cs.end());
    cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
    for (size_t a = 0; a < cs.size(); a++)
      for (size_t b = 0; b < cs.size(); b++)
        if (a != b) adj[cs[a]].push_back(cs[b]);
  }
  amd_order(nc, adj, perm);
  return NL_OK;
}

// Elimination tree of the permuted pattern and the number of entries of its
// Cholesky factor below the diagonal: for each row i (new order) the nodes of
// its row subtree, reached from each neighbour k < i by walking up the tree
// until a node already marked for row i.
nl_status nl_symbolic_fill(int n, int nnz, const int* row, const int* col, const int* perm, int* parent,
                           long long* fill) {
  if (n < 0 || nnz < 0 || !perm || !fill || (nnz > 0 && (!row || !col))) return NL_ERR_ARG;
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; i++) {
    if (perm[i] < 0 || perm[i] >= n || seen[perm[i]]) return NL_ERR_ARG;
    seen[perm[i]] = 1;
  }
  for (int k = 0; k < nnz; k++)
    if (row[k] < 0 || row[k] >= n || col[k] < 0 || col[k] >= n) return NL_ERR_ARG;
  std::vector<std::vector<int>> lower(n);  // new row -> new columns below it
  for (int k = 0; k < nnz; k++) {
    const int a = perm[row[k]], b = perm[col[k]];
    if (a == b) continue;
    lower[std::max(a, b)].push_back(std::min(a, b));
  }
  std::vector<int> par(n, -1), mark(n, -1);
  long long cnt = 0;
  for (int i = 0; i < n; i++) {
    mark[i] = i;
    for (int k : lower[i]) {
      for (int j = k; mark[j] != i; j = par[j]) {
        if (par[j] < 0) par[j] = i;
        mark[j] = i;
        cnt++;
      }
    }
  }
  if (parent) std::copy(par.begin(), par.end(), parent);
  *fill = cnt;
  return NL_OK;
}

}  // extern "C"

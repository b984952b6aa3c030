// problem_view.h -- read access to a BA section's host-side structure, for
// the batched solver (batch_lm.cu), which packs many sections into one arena.
#pragma once

#include <vector>

#include "../../include/nelson_b200.h"

// The fields of an nl_problem that a batch packs: sizes and intrinsics, the
// edges as added (camera / point index, fixed flags, observation, weight),
// the user -> internal camera permutation, the two device edge orders (as
// insertion indices) and the device parameter buffers.
struct nl_problem_view {
  int bc, ncv, ncf, npv, npf;
  double f, cx, cy;
  const std::vector<int>*e_cam, *e_camfix, *e_pt, *e_ptfix, *perm, *eorder, *porder;
  const std::vector<double>*e_obs, *e_w;
  double* d_cam;  // nc_all x 16 camera state
  double* d_pt;   // np_all x 3
  bool ready;
};
nl_status nl_problem_get_view(nl_problem* h, nl_problem_view* v);

"""nl_ba_cost_noalloc: the cost on caller-owned device buffers, no allocation.

Checked through the C ABI against the cost nl_update reports for the same
parameters (FP64 both; the two sum in different orders, so the bound is
1e-12 relative), on two calls in a row, after an LM solve has moved the
parameters, with and without weights, for 6- and 9-parameter cameras.  The
file is named to run last, after every other GPU test, and also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config

NOALLOC_MAX_EDGES = 16777216  # NL_NOALLOC_MAX_EDGES
TOL = 1e-12


def test_noalloc_rejects_oversize():
    L = N.load()
    out = C.c_double()
    rc = L.nl_ba_cost_noalloc(9, NOALLOC_MAX_EDGES + 1, None, None, None, None, None, None, 500.0, 0.0, 0.0,
                              C.c_void_p(C.addressof(out)), None)
    assert rc == 1  # NL_ERR_ARG, before any CUDA call
    rc = L.nl_ba_cost_noalloc(7, 10, None, None, None, None, None, None, 500.0, 0.0, 0.0,
                              C.c_void_p(C.addressof(out)), None)
    assert rc == 1


def _device_inputs(torch, g, p):
    """Camera states, points and edge rows as device tensors (allocated by the
    test, not by the entry point)."""
    cams = torch.from_numpy(np.ascontiguousarray(g.camera_state())).cuda()
    pts = torch.from_numpy(np.ascontiguousarray(g.get_params()[1])).cuda()
    cf = np.zeros(p.ne, np.int32) if p.cam_fixed is None else p.cam_fixed
    pf = np.zeros(p.ne, np.int32) if p.pt_fixed is None else p.pt_fixed
    e_cam = torch.from_numpy((p.cam_idx + cf * p.nc_var).astype(np.int32)).cuda()
    e_pt = torch.from_numpy((p.pt_idx + pf * p.np_var).astype(np.int32)).cuda()
    obs = torch.from_numpy(np.ascontiguousarray(p.obs, np.float64)).cuda()
    w = None if p.weight is None else torch.from_numpy(np.ascontiguousarray(p.weight, np.float64)).cuda()
    return cams, pts, e_cam, e_pt, obs, w


def _call(L, torch, p, cams, pts, e_cam, e_pt, obs, w, out):
    vp = C.c_void_p
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.nl_ba_cost_noalloc(p.bc, p.ne, vp(cams.data_ptr()), vp(pts.data_ptr()), vp(e_cam.data_ptr()),
                              vp(e_pt.data_ptr()), vp(obs.data_ptr()), None if w is None else vp(w.data_ptr()),
                              p.f, p.cx, p.cy, vp(out.data_ptr()), vp(stream))
    assert rc == 0, L.nl_status_string(rc)
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,scale", [(0, 1.0), (1, 0.1), (4, 1.0)])
def test_noalloc_cost_matches_update(cfg, scale):
    import torch
    L = N.load()
    p = make_config(cfg, scale)
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for stage in range(2):
        if stage == 1:  # move the parameters, then compare again
            g.lm_solve(N.LMSettings(maxNumIt=2), trace_cap=0)
        ref = g.update(False)
        args = _device_inputs(torch, g, p)
        first = _call(L, torch, p, *args, out)
        out.fill_(-1.0)
        free0 = torch.cuda.mem_get_info()[0]
        second = _call(L, torch, p, *args, out)
        free1 = torch.cuda.mem_get_info()[0]
        assert abs(first - ref) <= TOL * ref, (stage, first, ref)
        assert second == first  # same inputs, same fixed summation order
        assert free1 == free0   # the call took no device memory
    g.close()


@pytest.mark.gpu
def test_noalloc_empty_edge_set():
    import torch
    L = N.load()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.nl_ba_cost_noalloc(6, 0, None, None, None, None, None, None, 500.0, 320.0, 240.0,
                              C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0

"""The user-edge section (nl_section_*) on the GPU, against the FP64 oracle
(oracle/section.py) on the RangeScene problems (U-V, U-U, U-unary and
V-unary edges).

The user's edge code here is a vectorised torch evaluator.  It writes the
residuals and Jacobian blocks straight into the section's device arrays, on
the section's own stream (torch.cuda.ExternalStream), and applies the
increments to torch-held parameters.  This is the role a DoubleSection
subclass's EdgeBinary / EdgeUnary update() plays in the reference
(nelson/DoubleSection.hpp:338-365, nelson/BaseSection.cpp:5-86).

* update(true): chi2, U / V / W blocks and b equal the oracle's dense
  Hessian (FP64 1e-12, mixed 1e-6), in natural and AMD order;
* computeIncrement equals the oracle's damped dense solve (FP64 1e-9);
* LM and GN traces equal the oracle's (FP64 cost 1e-9, mixed 1e-6);
* the envelope solver gives the dense solver's trace;
* callback errors and out-of-order calls surface as errors.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import range_scene
from oracle.section import SectionOracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


class _DevArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 2}


def dev(ptr, n):
    """A torch view of n doubles of device memory at ptr (no copy)."""
    return torch.as_tensor(_DevArray(ptr, n), device="cuda")


class TorchRangeEdges:
    """The RangeScene edges evaluated with torch on the device."""

    def __init__(self, s, r_off, j_off):
        self.s, self.bu = s, s.bu
        t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
        self.x = t(s.x0)
        self.p = t(s.p0)
        self.R, self.JL = int(r_off[-1]), int(j_off[-1])
        bu = self.bu
        self.groups = {}
        for kind in range(4):
            idx = np.flatnonzero(s.kind == kind)
            self.groups[kind] = dict(
                n=idx.size, a=t(s.a[idx], torch.long), b=t(np.maximum(s.b[idx], 0), torch.long),
                ro=t(r_off[idx], torch.long), jo=t(j_off[idx], torch.long), d=t(s.d[idx]), e=t(s.e[idx]),
                avec=t(s.avec[idx]), cvec=t(s.cvec[idx]), delta=t(s.delta[idx]), prior=t(s.prior[idx]),
                w=t(s.w[idx]))
        self.eye_u = torch.eye(bu, dtype=torch.float64, device="cuda")
        self.eye_v = torch.eye(3, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        self.calls = {"evaluate": 0, "oplus": 0, "backup": 0, "rollback": 0}

    def _put(self, buf, off, vals):
        """buf[off[i] + k] = vals[i, k]."""
        k = torch.arange(vals.shape[1], device="cuda")
        buf[(off[:, None] + k[None, :]).reshape(-1)] = vals.reshape(-1)

    def evaluate(self, jac, r_ptr, j_ptr, stream):
        self.calls["evaluate"] += 1
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            r = dev(r_ptr, self.R)
            J = dev(j_ptr, self.JL) if jac else None
            bu, x, p = self.bu, self.x, self.p
            g = self.groups[0]
            if g["n"]:
                diff = x[g["a"], :3] - p[g["b"]]
                rng = torch.linalg.norm(diff, dim=1)
                r0 = rng - g["d"]
                r1 = (g["avec"] * diff).sum(1) + (g["cvec"] * x[g["a"], 3:]).sum(1) - g["e"]
                self._put(r, g["ro"], torch.stack([r0, r1], 1))
                if jac:
                    ja = torch.zeros((g["n"], 2, bu), dtype=torch.float64, device="cuda")
                    ja[:, 0, :3] = diff / rng[:, None]
                    ja[:, 1, :3] = g["avec"]
                    ja[:, 1, 3:] = g["cvec"]
                    jb = torch.stack([-diff / rng[:, None], -g["avec"]], 1)
                    self._put(J, g["jo"], torch.cat([ja.reshape(g["n"], -1), jb.reshape(g["n"], -1)], 1))
            g = self.groups[1]
            if g["n"]:
                self._put(r, g["ro"], x[g["a"]] - x[g["b"]] - g["delta"])
                if jac:
                    blk = torch.cat([self.eye_u.reshape(-1), -self.eye_u.reshape(-1)]).expand(g["n"], -1)
                    self._put(J, g["jo"], blk)
            g = self.groups[2]
            if g["n"]:
                self._put(r, g["ro"], g["w"][:, None] * (x[g["a"]] - g["prior"]))
                if jac:
                    self._put(J, g["jo"], g["w"][:, None] * self.eye_u.reshape(1, -1))
            g = self.groups[3]
            if g["n"]:
                self._put(r, g["ro"], g["w"][:, None] * (p[g["a"]] - g["prior"][:, :3]))
                if jac:
                    self._put(J, g["jo"], g["w"][:, None] * self.eye_v.reshape(1, -1))

    def oplus(self, du_ptr, dv_ptr, stream):
        self.calls["oplus"] += 1
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            self.x += dev(du_ptr, self.x.numel()).view_as(self.x)
            self.p += dev(dv_ptr, self.p.numel()).view_as(self.p)

    def backup(self, stream):
        self.calls["backup"] += 1
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            self.bck = (self.x.clone(), self.p.clone())

    def rollback(self, stream):
        self.calls["rollback"] += 1
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            self.x.copy_(self.bck[0])
            self.p.copy_(self.bck[1])


def make(s, precision=N.PREC_FP64, order="natural", kind=N.SOLVER_DENSE):
    sec = N.SectionGPU(s.bu, len(s.x0), len(s.p0), precision=precision)
    sec.add_edges(s.kind, s.a, s.b, s.m)
    if order == "amd":
        sec.permute_amd()
    sec.structure_ready()
    sec.set_solver_kind(kind)
    r_off, j_off = sec.layout()
    ev = TorchRangeEdges(s, r_off, j_off)
    sec.set_callbacks(ev.evaluate, ev.oplus, ev.backup, ev.rollback)
    return sec, ev


@pytest.mark.parametrize("bu", [3, 6, 9])
@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
@pytest.mark.parametrize("order", ["natural", "amd"])
def test_hessian_matches_oracle(bu, prec, order):
    s = range_scene(bu, nu=30, nv=300, seed=10 + bu)
    sec, ev = make(s, prec, order)
    o = SectionOracle(s)
    o.update(True)
    chi2 = sec.update(True)
    assert chi2 == pytest.approx(o.chi2, rel=1e-12)
    U, V, W, bU, bV = sec.hessian()
    u_rc, w_rc = sec.patterns()
    perm = sec.user2internal()
    user = np.argsort(perm)
    nub = len(s.x0) * bu
    H, b = o.H, o.b
    tol = (1e-12 if prec == N.PREC_FP64 else 1e-6) * np.abs(H).max()
    blk = lambda i: slice(bu * user[i], bu * user[i] + bu)
    for q, (r, c) in enumerate(u_rc):
        assert np.abs(U[q] - H[blk(r), blk(c)]).max() <= tol
    for v in range(len(s.p0)):
        sl = slice(nub + 3 * v, nub + 3 * v + 3)
        assert np.abs(V[v] - H[sl, sl]).max() <= tol
    for q, (u, v) in enumerate(w_rc):
        assert np.abs(W[q] - H[blk(u), nub + 3 * v:nub + 3 * v + 3]).max() <= tol
    tb = (1e-12 if prec == N.PREC_FP64 else 1e-6) * np.abs(b).max()
    for i in range(len(s.x0)):
        assert np.abs(bU[bu * i:bu * i + bu] - b[blk(i)]).max() <= tb
    assert np.abs(bV - b[nub:]).max() <= tb
    # every U-U edge's pair and every U-V pair is in the patterns
    assert len(w_rc) == len({(int(a), int(c)) for k, a, c in zip(s.kind, s.a, s.b) if k == 0})
    assert sec.update(False) == pytest.approx(o.chi2, rel=1e-12)
    sec.close()


@pytest.mark.parametrize("bu", [3, 6])
def test_increment_matches_dense_solve(bu):
    s = range_scene(bu, nu=30, nv=300, seed=4)
    sec, ev = make(s)
    o = SectionOracle(s)
    o.update(True)
    sec.update(True)
    for rel, ab in ((0.0, 1e-3 * o.max_abs_hdiag()), (0.01, 0.0)):
        ok, du, dv = sec.compute_increment(rel, ab)
        assert ok and o.compute_increment(rel, ab)
        got = np.r_[du, dv]
        assert np.abs(got - o.inc).max() <= 1e-9 * np.abs(o.inc).max()
    sec.close()


def _trace_check(tr, tro, tol):
    assert len(tr) == len(tro)
    assert np.array_equal(tr[:, [0, 1, 6, 7]], tro[:, [0, 1, 6, 7]])
    ok = tro[:, 2] > 0
    assert np.abs(tr[ok, 2] - tro[ok, 2]).max() <= tol * tro[ok, 2].max()
    assert np.abs(tr[:, 3] - tro[:, 3]).max() <= tol * max(np.abs(tro[:, 3]).max(), 1e-300)


@pytest.mark.parametrize("bu", [3, 6, 9])
@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_lm_trace_parity(bu, prec):
    s = range_scene(bu, nu=30, nv=300, seed=20 + bu)
    sec, ev = make(s, prec, "amd")
    # |delta|^2 threshold 1e-12: the step that crosses it goes from ~1e-9 to
    # ~1e-13, far above the round-off floor (~1e-22) where the default 1e-30
    # would let round-off pick the last iteration
    reason, tr, it = sec.lm_solve(N.LMSettings(maxNumIt=15, epsIncSquare=1e-12))
    o = SectionOracle(s)
    r_o, tro, it_o = o.lm_solve(maxNumIt=15, epsIncSquare=1e-12)
    assert reason == r_o and it == it_o
    _trace_check(tr, tro, 1e-9 if prec == N.PREC_FP64 else 1e-6)
    tol = 1e-7 if prec == N.PREC_FP64 else 1e-4
    assert np.abs(ev.x.cpu().numpy() - o.x).max() <= tol
    assert np.abs(ev.p.cpu().numpy() - o.p).max() <= tol
    assert ev.calls["backup"] >= 1 and ev.calls["oplus"] >= 1
    sec.close()


@pytest.mark.parametrize("rel", [0.0, 0.01])
def test_gn_trace_parity(rel):
    s = range_scene(6, nu=30, nv=300, seed=8)
    sec, ev = make(s)
    reason, tr, it = sec.gn_solve(N.GNSettings(maxNumIt=6, relLambda=rel))
    o = SectionOracle(s)
    r_o, tro, it_o = o.gn_solve(maxNumIt=6, relLambda=rel)
    assert reason == r_o and it == it_o
    _trace_check(tr, tro, 1e-9)
    sec.close()


def test_envelope_solver_gives_the_dense_trace():
    s = range_scene(3, nu=60, nv=500, seed=30)
    a, _ = make(s, order="amd", kind=N.SOLVER_DENSE)
    b, _ = make(s, order="amd", kind=N.SOLVER_ENVELOPE)
    ra, tra, _ = a.lm_solve(N.LMSettings(maxNumIt=10, epsIncSquare=1e-12))
    rb, trb, _ = b.lm_solve(N.LMSettings(maxNumIt=10, epsIncSquare=1e-12))
    assert ra == rb
    _trace_check(trb, tra, 1e-12)
    a.close()
    b.close()


def test_errors():
    s = range_scene(3, nu=6, nv=20, obs_per_point=2, uu_edges=2, seed=1)
    sec = N.SectionGPU(3, 6, 20)
    with pytest.raises(N.NelsonError):
        sec.update(True)                                             # before structure_ready
    with pytest.raises(N.NelsonError):
        sec.add_edges([N.EDGE_UU], [2], [2], [3])                     # same block twice
    with pytest.raises(N.NelsonError):
        sec.add_edges([N.EDGE_UV], [0], [20], [2])                    # V block out of range
    with pytest.raises(N.NelsonError):
        sec.add_edges([N.EDGE_U], [0], [-1], [0])                     # empty residual
    with pytest.raises(N.NelsonError):
        sec.add_edges([7], [0], [0], [2])                             # unknown kind
    sec.add_edges(s.kind, s.a, s.b, s.m)
    sec.structure_ready()
    with pytest.raises(N.NelsonError):
        sec.update(True)                                             # no callbacks yet
    r_off, j_off = sec.layout()
    ev = TorchRangeEdges(s, r_off, j_off)
    sec.set_callbacks(ev.evaluate, ev.oplus)                         # no backup / rollback
    with pytest.raises(N.NelsonError):
        sec.lm_solve()                                               # LM needs them
    sec.gn_solve(N.GNSettings(maxNumIt=2))                           # GN does not

    def broken(jac, r, J, st):
        raise ValueError("edge evaluation failed")
    sec.set_callbacks(broken, ev.oplus, ev.backup, ev.rollback)
    with pytest.raises(ValueError):
        sec.update(True)
    sec.close()


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_section_without_v_blocks(prec):
    """Only U-U edges and U priors (no V blocks): the Schur solve degenerates
    to the tiled Cholesky of U, as in a pose graph."""
    s = range_scene(3, nu=12, nv=0, obs_per_point=4, uu_edges=30, seed=3)
    sec, ev = make(s, prec)
    assert sec.counts()[1] == 0
    reason, tr, it = sec.lm_solve(N.LMSettings(maxNumIt=10, epsIncSquare=1e-12))
    o = SectionOracle(s)
    r_o, tro, it_o = o.lm_solve(maxNumIt=10, epsIncSquare=1e-12)
    assert reason == r_o and it == it_o
    _trace_check(tr, tro, 1e-9 if prec == N.PREC_FP64 else 1e-6)
    sec.close()

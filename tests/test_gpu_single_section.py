"""A single-section system through the solver-only handle.

SingleSection problems (nelson/SingleSection.hpp:63-139: one parameter
section, no second section to eliminate) solve H d = -b with the dense
Cholesky (SolverCholeskyDense, nelson/SolverCholeskyDense.hpp:39-67).  The
solver-only handle given no V / W blocks (nv = 0) is exactly that: S is the
damped U and the tiled Cholesky solves it.  The system here has the shape of
a pose graph: 400 nodes of block size 3 on a chain with loop closures, each
edge adding an SPD 3x3 block M_e to its two diagonal blocks and -M_e to the
coupling block, plus a prior on node 0.  Checked against numpy in FP64 (1e-10)
and in mixed precision (1e-4, the increment tolerance of the parity tests),
with the dense and the envelope solver.
"""
import numpy as np
import pytest

from nelson_b200 import native as N

pytestmark = pytest.mark.gpu


def pose_graph_hessian(n=400, bu=3, closures=60, seed=17):
    rng = np.random.default_rng(seed)
    edges = [(i, i + 1) for i in range(n - 1)]
    for _ in range(closures):
        i = int(rng.integers(0, n - 20))
        edges.append((i, i + int(rng.integers(5, 20))))
    H = np.zeros((n * bu, n * bu))
    for i, j in edges:
        A = rng.normal(size=(bu, bu))
        M = A.T @ A + 0.1 * np.eye(bu)
        si, sj = slice(i * bu, (i + 1) * bu), slice(j * bu, (j + 1) * bu)
        H[si, si] += M
        H[sj, sj] += M
        H[si, sj] -= M
        H[sj, si] -= M
    H[:bu, :bu] += np.eye(bu)  # prior on the first pose
    pattern = {(i, i) for i in range(n)} | {(min(i, j), max(i, j)) for i, j in edges}
    # upper blocks in CSC order: by column, then row
    u_rc = sorted(pattern, key=lambda rc: (rc[1], rc[0]))
    U = np.stack([H[r * bu:(r + 1) * bu, c * bu:(c + 1) * bu] for r, c in u_rc])
    b = rng.normal(size=n * bu)
    return H, np.array(u_rc, np.int32), U, b


@pytest.mark.parametrize("kind", [N.SOLVER_DENSE, N.SOLVER_ENVELOPE])
@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_single_section_dense_solve(prec, kind):
    bu, n = 3, 400
    H, u_rc, U, b = pose_graph_hessian(n, bu)
    s = N.SchurSolverGPU(bu, n, 0, u_rc, np.zeros((0, 2), np.int32), np.zeros((0, 2), np.int32), precision=prec)
    s.set_solver_kind(kind)
    s.set_hessian(U, np.zeros((0, 3, 3)), np.zeros((0, bu, 3)), b, np.zeros(0))
    hmax = float(np.abs(np.diag(H)).max())
    # the mixed handle holds U in FP32
    assert s.max_abs_hdiag() == pytest.approx(hmax, rel=1e-12 if prec == N.PREC_FP64 else 1e-7)
    lam = 1e-2 * hmax
    ok, du, dv = s.compute_increment(0.0, lam)
    assert ok and dv.size == 0
    ref = -np.linalg.solve(H + lam * np.eye(n * bu), b)
    tol = 1e-10 if prec == N.PREC_FP64 else 1e-4
    assert np.abs(du - ref).max() <= tol * np.abs(ref).max()
    s.close()

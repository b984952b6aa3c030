"""Seeded synthetic bundle-adjustment problems and the linear test fixture.

The reference publishes no dataset for its Schur LM path; its only BA
workload is a random scene built in nelson/samples/BASchurPerfomances.cpp:30-97
(random SE3 cameras looking at a point cloud, edges from a visibility list).
These generators build scenes of the same kind at the sizes the benchmark
configurations name, with seeded numpy RNG (seed = 1234 + config index), so the
oracle, the CUDA path, the tests and bench.py all see bit-identical inputs.

Camera model (shared by the oracle and the CUDA kernels):
    P = R X + t,  (x, y) = P.xy / P.z,  d = 1 + k1 r^2 + k2 r^4,
    pixel = f d (x, y) + (cx, cy)
A camera is given as axis-angle w (3), t (3) and, for 9-parameter cameras,
f, k1, k2.  Its increment is [dw, dt (, df, dk1, dk2)] with R <- exp(dw) R.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
from scipy.spatial.transform import Rotation

CX, CY, F_FIXED = 320.0, 240.0, 500.0


@dataclass
class BAProblem:
    """A bundle-adjustment instance: U section = cameras, V section = points."""

    bc: int                      # camera block size (6 or 9)
    cams: np.ndarray             # (nc_var + nc_fix, bc) initial values
    pts: np.ndarray              # (np_var + np_fix, 3) initial values
    nc_var: int
    np_var: int
    cam_idx: np.ndarray          # (ne,) int32 camera id per edge
    pt_idx: np.ndarray           # (ne,) int32 point id per edge
    obs: np.ndarray              # (ne, 2) pixel measurements
    weight: np.ndarray | None = None   # (ne,) per-edge weights (cost w |r|^2)
    cam_fixed: np.ndarray | None = None  # (ne,) int32, 1 = camera is a fixed node
    pt_fixed: np.ndarray | None = None   # (ne,) int32, 1 = point is a fixed node
    nc_fix: int = 0
    np_fix: int = 0
    f: float = F_FIXED
    cx: float = CX
    cy: float = CY
    cams_true: np.ndarray | None = None
    pts_true: np.ndarray | None = None
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def ne(self) -> int:
        return int(self.cam_idx.shape[0])


def so3_exp(w: np.ndarray) -> np.ndarray:
    return Rotation.from_rotvec(np.asarray(w, dtype=np.float64).reshape(-1, 3)).as_matrix()


def so3_log(R: np.ndarray) -> np.ndarray:
    return Rotation.from_matrix(np.asarray(R, dtype=np.float64).reshape(-1, 3, 3)).as_rotvec()


def project(cams: np.ndarray, pts: np.ndarray, cam_idx, pt_idx, bc: int,
            f=F_FIXED, cx=CX, cy=CY) -> np.ndarray:
    """Pixel coordinates of pts[pt_idx] seen by cams[cam_idx] (float64)."""
    R = so3_exp(cams[:, :3])[cam_idx]
    t = cams[cam_idx, 3:6]
    P = np.einsum("eij,ej->ei", R, pts[pt_idx]) + t
    x = P[:, 0] / P[:, 2]
    y = P[:, 1] / P[:, 2]
    if bc == 9:
        ff = cams[cam_idx, 6]
        k1 = cams[cam_idx, 7]
        k2 = cams[cam_idx, 8]
    else:
        ff, k1, k2 = f, 0.0, 0.0
    r2 = x * x + y * y
    d = 1.0 + r2 * (k1 + k2 * r2)
    return np.stack([ff * d * x + cx, ff * d * y + cy], axis=1)


def _look_at(centers: np.ndarray, targets: np.ndarray, up: np.ndarray) -> np.ndarray:
    """World-to-camera rotations whose +z axis points from centre to target."""
    z = targets - centers
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    x = np.cross(z, up)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)  # rows


def _choose(rng, ncand_valid: np.ndarray, cand: np.ndarray, kmin: int, kmax: int):
    """Pick k ~ U{kmin..kmax} distinct candidates per row (k clipped to the
    number of valid candidates); invalid candidates are marked -1 in `cand`."""
    npnt, nc = cand.shape
    keys = rng.random((npnt, nc))
    keys[cand < 0] = 2.0
    order = np.argsort(keys, axis=1, kind="stable")
    k = rng.integers(kmin, kmax + 1, size=npnt)
    k = np.minimum(k, ncand_valid)
    kk = min(kmax, nc)
    sel = np.take_along_axis(cand, order[:, :kk], axis=1)
    mask = np.arange(kk)[None, :] < k[:, None]
    # point-major edge list, cameras ascending inside a point
    sel = np.where(mask, sel, np.iinfo(np.int32).max)
    sel.sort(axis=1)  # the k chosen cameras now occupy the first k slots
    pt_idx = np.repeat(np.arange(npnt, dtype=np.int32), k)
    cam_idx = sel[mask].astype(np.int32)
    return cam_idx, pt_idx


def _finish(rng, name, bc, Rt, tt, intr, pts_true, cam_idx, pt_idx, noise=1.0,
            outlier_frac=0.0, rot_sigma=0.01, t_sigma=0.05, pt_sigma=0.05,
            weights=None, meta=None) -> BAProblem:
    nc = Rt.shape[0]
    wt = so3_log(Rt)
    cams_true = np.concatenate([wt, tt] + ([intr] if bc == 9 else []), axis=1)
    z = project(cams_true, pts_true, cam_idx, pt_idx, bc)
    ne = z.shape[0]
    z = z + rng.normal(0.0, noise, size=(ne, 2))
    if outlier_frac > 0:
        nout = int(round(outlier_frac * ne))
        idx = rng.choice(ne, size=nout, replace=False)
        z[idx] = project(cams_true, pts_true, cam_idx[idx], pt_idx[idx], bc) + \
            rng.uniform(-50.0, 50.0, size=(nout, 2))
    # initial values: left-perturbed rotations, shifted translations and points
    dR = so3_exp(rng.normal(0.0, rot_sigma, size=(nc, 3)))
    w0 = so3_log(np.einsum("cij,cjk->cik", dR, Rt))
    t0 = tt + rng.normal(0.0, t_sigma, size=tt.shape)
    parts = [w0, t0]
    if bc == 9:
        f0 = intr[:, 0:1] * (1.0 + 0.01 * rng.normal(size=(nc, 1)))
        parts.append(np.concatenate([f0, np.zeros((nc, 2))], axis=1))
    cams0 = np.concatenate(parts, axis=1)
    pts0 = pts_true + rng.normal(0.0, pt_sigma, size=pts_true.shape)
    return BAProblem(bc=bc, cams=np.ascontiguousarray(cams0), pts=np.ascontiguousarray(pts0),
                     nc_var=nc, np_var=pts_true.shape[0],
                     cam_idx=np.ascontiguousarray(cam_idx, dtype=np.int32),
                     pt_idx=np.ascontiguousarray(pt_idx, dtype=np.int32),
                     obs=np.ascontiguousarray(z), weight=weights,
                     cams_true=cams_true, pts_true=pts_true, name=name, meta=meta or {})


def ring_scene(nc: int, npts: int, kmin: int, kmax: int, bc: int, seed: int,
               name: str = "ring", weights: bool = False, radius: float = 10.0,
               height: float = 1.0, extent: float = 2.0) -> BAProblem:
    """Cameras on a circle looking at the origin, points uniform in a cube;
    each point seen by k ~ U{kmin..kmax} cameras drawn uniformly among those
    that see it in front (every camera does, at these sizes)."""
    rng = np.random.default_rng(seed)
    th = 2.0 * np.pi * np.arange(nc) / nc
    C = np.stack([radius * np.cos(th), radius * np.sin(th), np.full(nc, height)], axis=1)
    Rt = _look_at(C, np.zeros_like(C), np.array([0.0, 0.0, 1.0]))
    tt = -np.einsum("cij,cj->ci", Rt, C)
    intr = None
    if bc == 9:
        intr = np.stack([rng.uniform(400.0, 600.0, nc), rng.normal(0, 0.01, nc),
                         rng.normal(0, 0.01, nc)], axis=1)
    pts = rng.uniform(-extent, extent, size=(npts, 3))
    depth = np.einsum("cj,pj->pc", Rt[:, 2, :], pts) + tt[None, :, 2]
    cand = np.where(depth > 0.1, np.arange(nc)[None, :], -1).astype(np.int64)
    cam_idx, pt_idx = _choose(rng, (cand >= 0).sum(1), cand, kmin, kmax)
    w = rng.uniform(0.5, 2.0, size=cam_idx.shape[0]) if weights else None
    return _finish(rng, name, bc, Rt, tt, intr, pts, cam_idx, pt_idx, weights=w,
                   meta=dict(nc=nc, np=npts, kmin=kmin, kmax=kmax))


def grid_scene(gx: int, gy: int, npts: int, kmin: int, kmax: int, seed: int,
               outlier_frac: float = 0.01, radius: int = 2, height: float = 10.0,
               name: str = "grid") -> BAProblem:
    """Aerial grid: gx*gy 9-parameter cameras at `height` looking down; each
    point is seen by k ~ U{kmin..kmax} cameras drawn from the grid neighbours
    (within `radius` cells) of the cell below it (camera-locality bias)."""
    rng = np.random.default_rng(seed)
    nc = gx * gy
    ix, iy = np.meshgrid(np.arange(gx), np.arange(gy), indexing="ij")
    C = np.stack([ix.ravel().astype(np.float64), iy.ravel().astype(np.float64),
                  np.full(nc, height)], axis=1)
    down = C.copy()
    down[:, 2] = 0.0
    R0 = _look_at(C, down, np.array([0.0, 1.0, 0.0]))
    tilt = so3_exp(rng.normal(0.0, 0.05, size=(nc, 3)))
    Rt = np.einsum("cij,cjk->cik", tilt, R0)
    tt = -np.einsum("cij,cj->ci", Rt, C)
    intr = np.stack([rng.uniform(400.0, 600.0, nc), rng.normal(0, 0.01, nc),
                     rng.normal(0, 0.01, nc)], axis=1)
    pts = np.stack([rng.uniform(-0.5, gx - 0.5, npts), rng.uniform(-0.5, gy - 0.5, npts),
                    rng.uniform(-1.0, 1.0, npts)], axis=1)
    cx0 = np.clip(np.rint(pts[:, 0]).astype(np.int64), 0, gx - 1)
    cy0 = np.clip(np.rint(pts[:, 1]).astype(np.int64), 0, gy - 1)
    offs = np.arange(-radius, radius + 1)
    dx, dy = np.meshgrid(offs, offs, indexing="ij")
    nx = cx0[:, None] + dx.ravel()[None, :]
    ny = cy0[:, None] + dy.ravel()[None, :]
    valid = (nx >= 0) & (nx < gx) & (ny >= 0) & (ny < gy)
    cand = np.where(valid, nx * gy + ny, -1)
    cam_idx, pt_idx = _choose(rng, valid.sum(1), cand, kmin, kmax)
    return _finish(rng, name, 9, Rt, tt, intr, pts, cam_idx, pt_idx,
                   outlier_frac=outlier_frac,
                   meta=dict(nc=nc, np=npts, kmin=kmin, kmax=kmax, grid=(gx, gy)))


# Benchmark configurations (seed = 1234 + index).
CONFIG_NAMES = {
    0: "c0: 20 cams (6-param ring) / 500 pts / k~U{3..8}",
    1: "c1: 200 cams (9-param ring) / 50k pts / k~U{3..12}",
    2: "c2: 1500 cams (9-param 30x50 grid) / 500k pts / k~U{2..12} / 1% outliers",
    4: "c4: 64 cams (6-param ring) / 5k pts / k~U{3..8} / w~U[0.5,2]",
}


def make_config(idx: int, scale: float = 1.0) -> BAProblem:
    """Problem for benchmark configuration `idx`; `scale` < 1 shrinks the
    point count (and the grid) for quick tests while keeping the shape."""
    seed = 1234 + idx
    if idx == 0:
        return ring_scene(20, max(50, int(500 * scale)), 3, 8, 6, seed, name="c0")
    if idx == 1:
        return ring_scene(max(10, int(200 * scale)), max(200, int(50000 * scale)), 3, 12, 9,
                          seed, name="c1")
    if idx == 2:
        gx = max(4, int(round(30 * np.sqrt(scale))))
        gy = max(6, int(round(50 * np.sqrt(scale))))
        return grid_scene(gx, gy, max(500, int(500000 * scale)), 2, 12, seed, name="c2")
    if idx == 4:
        return ring_scene(64, max(200, int(5000 * scale)), 3, 8, 6, seed, name="c4",
                          weights=True)
    raise ValueError(f"no single-problem generator for config {idx}")


def make_batch(n: int = 256, seed: int = 1234 + 3):
    """Config 3: independent ring problems with uneven sizes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nc = int(rng.integers(8, 65))
        npts = int(rng.integers(200, 4001))
        out.append(ring_scene(nc, npts, 3, 8, 6, int(rng.integers(1 << 30)), name=f"c3.{i}"))
    return out


# ---------------------------------------------------------------------------
# The linear fixture of nelson/tests/testDoubleSectionSchurCommon.h:24-413.
@dataclass
class LinearEdge:
    type: int        # 0 unary U, 1 unary V, 2 binary UU, 3 binary UV
    id1: int
    id2: int
    A1: np.ndarray   # dr x B1
    A2: np.ndarray | None
    z: np.ndarray


@dataclass
class LinearProblem:
    bu: int
    bv: int
    u: np.ndarray      # (nu_var + nu_fix, bu)
    v: np.ndarray      # (nv_var + nv_fix, bv)
    nu_var: int
    nv_var: int
    edges: list
    nu_fix: int = 0
    nv_fix: int = 0
    u_true: np.ndarray | None = None
    v_true: np.ndarray | None = None


EDGE_UNARY_U, EDGE_UNARY_V, EDGE_BINARY_UU, EDGE_BINARY_UV = 0, 1, 2, 3


def points2d3d_fixture(seed: int = 7, u_block_diagonal: bool = False,
                       w_block_diagonal: bool = False) -> LinearProblem:
    """5 2D points (U, block 2) and 3 3D points (V, block 3) with identity
    Jacobian edges: unary on every point, binary UU on every pair (unless U is
    block diagonal), binary UV on every (2D, 3D) pair (only (i, i) when W is
    block diagonal).  Measurements are taken at the ground truth, so chi2 = 0
    there (testDoubleSectionCommon.hpp:15-58)."""
    rng = np.random.default_rng(seed)
    gt = rng.uniform(-1.0, 1.0, size=(3, 5))
    p2 = gt[:2, :5].T.copy()
    p3 = gt[:, :3].T.copy()
    fixed2 = rng.uniform(-1, 1, size=(1, 2))
    fixed3 = rng.uniform(-1, 1, size=(1, 3))
    I2 = np.eye(2)
    I3 = np.eye(3)
    sel = np.array([[-1.0, 0, 0], [0, -1.0, 0]])
    edges = []
    for i in range(5):
        edges.append(LinearEdge(EDGE_UNARY_U, i, -1, I2, None, p2[i].copy()))
    for i in range(3):
        edges.append(LinearEdge(EDGE_UNARY_V, i, -1, I3, None, p3[i].copy()))
    if not u_block_diagonal:
        for i in range(5):
            for j in range(i + 1, 5):
                edges.append(LinearEdge(EDGE_BINARY_UU, i, j, I2, -I2, p2[i] - p2[j]))
    if not w_block_diagonal:
        for i in range(5):
            for j in range(3):
                edges.append(LinearEdge(EDGE_BINARY_UV, i, j, I2, sel, p2[i] - p3[j][:2]))
    else:
        for i in range(3):
            edges.append(LinearEdge(EDGE_BINARY_UV, i, i, I2, sel, p2[i] - p3[i][:2]))
    return LinearProblem(bu=2, bv=3, u=np.concatenate([p2, fixed2]), v=np.concatenate([p3, fixed3]),
                         nu_var=5, nv_var=3, edges=edges, nu_fix=1, nv_fix=1,
                         u_true=p2.copy(), v_true=p3.copy())


def add_uniform_noise(lp: LinearProblem, sigma: float, rng) -> None:
    """Points2d3dBase::addNoise: uniform in [-sigma, sigma] on the variable
    parameters (testDoubleSectionSchurCommon.h:347-354)."""
    lp.u[:lp.nu_var] += rng.uniform(-sigma, sigma, size=(lp.nu_var, lp.bu))
    lp.v[:lp.nv_var] += rng.uniform(-sigma, sigma, size=(lp.nv_var, lp.bv))


def with_fixed_nodes(p: BAProblem, ncf: int, npf: int = 0) -> BAProblem:
    """The last `ncf` cameras and `npf` points become fixed nodes
    (NodeType::Fixed): parameters keep their order (variable blocks first,
    then fixed), edges refer to fixed blocks by their index among the fixed
    ones.  Holding two cameras fixed removes the similarity gauge of BA."""
    ncv, npv = p.nc_var - ncf, p.np_var - npf
    cf = (p.cam_idx >= ncv).astype(np.int32)
    pf = (p.pt_idx >= npv).astype(np.int32)
    return BAProblem(bc=p.bc, cams=p.cams, pts=p.pts, nc_var=ncv, np_var=npv,
                     cam_idx=np.where(cf == 1, p.cam_idx - ncv, p.cam_idx).astype(np.int32),
                     pt_idx=np.where(pf == 1, p.pt_idx - npv, p.pt_idx).astype(np.int32),
                     obs=p.obs, weight=p.weight, cam_fixed=cf, pt_fixed=pf, nc_fix=ncf, np_fix=npf,
                     f=p.f, cx=p.cx, cy=p.cy, cams_true=p.cams_true, pts_true=p.pts_true,
                     name=p.name + "+fixed", meta=dict(p.meta))


# ---------------------------------------------------------------------------
# Problem files.
#
# * Visibility lists in the format of the reference's Problem::load
#   (nelson/samples/Problems.cpp:8-30): "nCameras nPoints nEdges" followed by
#   nEdges whitespace-separated (camera, point) pairs.  `problem_from_pairs`
#   builds a seeded synthetic BA problem on such a structure (the reference's
#   sample does the same: random parameters on a given visibility list,
#   nelson/samples/BASchurPerfomances.cpp:30-97).
# * BAL-style files (header "num_cameras num_points num_observations", one
#   "camera point x y" line per observation, then 9 parameters per camera:
#   axis-angle, translation, f, k1, k2, then 3 per point).  Such files predict
#   pixel = -f d (P.x, P.y) / P.z about the image centre; this library's model
#   is f d (P.x, P.y) / P.z + (cx, cy), so a BAL problem loads with cx = cy = 0
#   and negated observations (the same residual norms).

def load_pairs(path: str):
    """(n_cameras, n_points, cam_idx, pt_idx) of a visibility-list file."""
    with open(path) as f:
        tok = f.read().split()
    if len(tok) < 3:
        raise ValueError(f"{path}: missing header")
    nc, npts, ne = int(tok[0]), int(tok[1]), int(tok[2])
    if len(tok) < 3 + 2 * ne:
        raise ValueError(f"{path}: {ne} edges announced, {(len(tok) - 3) // 2} present")
    e = np.array(tok[3:3 + 2 * ne], dtype=np.int64).reshape(ne, 2)
    if ne and (e[:, 0].min() < 0 or e[:, 0].max() >= nc or e[:, 1].min() < 0 or e[:, 1].max() >= npts):
        raise ValueError(f"{path}: edge index out of range")
    return nc, npts, e[:, 0].astype(np.int32), e[:, 1].astype(np.int32)


def save_pairs(path: str, n_cameras: int, n_points: int, cam_idx, pt_idx) -> None:
    with open(path, "w") as f:
        f.write(f"{n_cameras} {n_points} {len(cam_idx)}\n")
        for c, p in zip(cam_idx, pt_idx):
            f.write(f"{int(c)} {int(p)}\n")


def problem_from_pairs(n_cameras: int, n_points: int, cam_idx, pt_idx, bc: int = 9, seed: int = 1234,
                       noise: float = 1.0) -> BAProblem:
    """Seeded synthetic BA problem on a given visibility list: cameras on a
    circle looking at the origin, points in a cube around it (every point is in
    front of every camera), N(0, noise) pixel noise, perturbed initial values."""
    rng = np.random.default_rng(seed)
    th = 2.0 * np.pi * np.arange(n_cameras) / max(n_cameras, 1)
    C = np.stack([10.0 * np.cos(th), 10.0 * np.sin(th), np.ones(n_cameras)], axis=1)
    Rt = _look_at(C, np.zeros_like(C), np.array([0.0, 0.0, 1.0]))
    tt = -np.einsum("cij,cj->ci", Rt, C)
    intr = np.stack([rng.uniform(400.0, 600.0, n_cameras), rng.normal(0, 0.01, n_cameras),
                     rng.normal(0, 0.01, n_cameras)], axis=1) if bc == 9 else None
    pts = rng.uniform(-2.0, 2.0, size=(n_points, 3))
    return _finish(rng, "pairs", bc, Rt, tt, intr, pts, np.asarray(cam_idx, np.int32),
                   np.asarray(pt_idx, np.int32), noise=noise,
                   meta=dict(nc=n_cameras, np=n_points, source="visibility list"))


def load_bal(path: str) -> BAProblem:
    """A BAL-style file as a 9-parameter BA problem (cx = cy = 0, observations
    negated, see above); the file's parameters are the initial values."""
    with open(path) as f:
        tok = f.read().split()
    nc, npts, ne = int(tok[0]), int(tok[1]), int(tok[2])
    need = 3 + 4 * ne + 9 * nc + 3 * npts
    if len(tok) < need:
        raise ValueError(f"{path}: {len(tok)} numbers, {need} expected")
    o = np.array(tok[3:3 + 4 * ne], dtype=np.float64).reshape(ne, 4)
    q = 3 + 4 * ne
    cams = np.array(tok[q:q + 9 * nc], dtype=np.float64).reshape(nc, 9)
    q += 9 * nc
    pts = np.array(tok[q:q + 3 * npts], dtype=np.float64).reshape(npts, 3)
    cam_idx = o[:, 0].astype(np.int32)
    pt_idx = o[:, 1].astype(np.int32)
    if ne and (cam_idx.min() < 0 or cam_idx.max() >= nc or pt_idx.min() < 0 or pt_idx.max() >= npts):
        raise ValueError(f"{path}: observation index out of range")
    return BAProblem(bc=9, cams=cams, pts=pts, nc_var=nc, np_var=npts, cam_idx=cam_idx, pt_idx=pt_idx,
                     obs=np.ascontiguousarray(-o[:, 2:4]), cx=0.0, cy=0.0, name=os.path.basename(path),
                     meta=dict(source="BAL"))


def save_bal(path: str, p: BAProblem) -> None:
    """Writes a 9-parameter problem with cx = cy = 0 in the BAL layout (the
    inverse of load_bal)."""
    if p.bc != 9 or p.cx != 0.0 or p.cy != 0.0 or p.nc_fix or p.np_fix or p.weight is not None:
        raise ValueError("BAL files hold unweighted 9-parameter problems about the image centre")
    with open(path, "w") as f:
        f.write(f"{p.nc_var} {p.np_var} {p.ne}\n")
        for c, q, z in zip(p.cam_idx, p.pt_idx, p.obs):
            f.write(f"{int(c)} {int(q)} {-z[0]:.17g} {-z[1]:.17g}\n")
        for v in p.cams.reshape(-1):
            f.write(f"{v:.17g}\n")
        for v in p.pts.reshape(-1):
            f.write(f"{v:.17g}\n")


# ---------------------------------------------------------------------------
# 2D scan alignment: SE(2) pose graphs with point-to-line edges, shaped like
# the single-section tests of the reference (nelson/tests/
# testGaussNewton2DScansAlign.cpp:485-737): world points in [-100, 100]^2
# with random unit normals, num_poses + 1 scan poses exp((10, 10, pi) * U[-1, 1]^3)
# (scan 0 is the fixed pose), each scan the world points in its own frame;
# edges (i, j), i < j, with scan i as model (points and normals) and scan j as
# target, all pairs ("full") or a star from scan 0 plus random pairs
# ("sparse"); the variable poses start at exp(noise * U[-1, 1]^3) T_true.


def se2_exp(v):
    """exp of se(2) (vx, vy, w): (R(w), V(w) (vx, vy))."""
    vx, vy, w = v
    c, s = np.cos(w), np.sin(w)
    if abs(w) > 1e-9:
        a, b = s / w, (1.0 - c) / w
    else:
        a, b = 1.0 - w * w / 6.0, 0.5 * w
    return np.array([a * vx - b * vy, b * vx + a * vy, w])


def se2_compose(d, p):
    """exp(d) * T_p for pose p = (x, y, theta): theta + w, R(w) t + V(w) v."""
    t = se2_exp(d)
    c, s = np.cos(d[2]), np.sin(d[2])
    return np.array([c * p[0] - s * p[1] + t[0], s * p[0] + c * p[1] + t[1], p[2] + d[2]])


@dataclass
class ScanAlignProblem:
    poses_true: np.ndarray   # (num_poses + 1, 3); row 0 is the fixed pose
    poses0: np.ndarray       # (num_poses, 3) start of the variable poses
    scans: list              # (npts, 2) points of each scan in its own frame
    normals: list            # (npts, 2)
    edges: list              # (i, j): model scan i, target scan j
    name: str = "scan_align"


def scan_align_scene(num_poses: int = 15, points_per_scan: int = 3000, noise=(0.01, 0.01, np.pi / 1000.0),
                     full_edges: bool = True, seed: int = 5) -> ScanAlignProblem:
    rng = np.random.default_rng(seed)
    world = 100.0 * rng.uniform(-1, 1, size=(points_per_scan, 2))
    nrm = np.empty((points_per_scan, 2))
    for k in range(points_per_scan):
        while True:
            v = rng.uniform(-1, 1, size=2)
            if v @ v >= 1e-3:
                break
        nrm[k] = v / np.linalg.norm(v)
    poses = np.array([se2_compose(np.array([10.0, 10.0, np.pi]) * rng.uniform(-1, 1, size=3), np.zeros(3))
                      for _ in range(num_poses + 1)])
    scans, normals = [], []
    for x, y, th in poses:
        c, s = np.cos(th), np.sin(th)
        R = np.array([[c, -s], [s, c]])
        scans.append((world - np.array([x, y])) @ R)       # R' (X - t)
        normals.append(nrm @ R)
    n_all = num_poses + 1
    if full_edges:
        edges = [(i, j) for i in range(n_all) for j in range(i + 1, n_all)]
    else:
        edges = [(0, i) for i in range(1, n_all)]
        for i in range(1, n_all - 1):
            for _ in range(int(rng.integers(0, n_all - i - 1))):
                edges.append((i, int(rng.integers(i + 1, n_all))))
    sig = np.asarray(noise, dtype=float)
    poses0 = np.array([se2_compose(sig * rng.uniform(-1, 1, size=3), poses[i]) for i in range(1, n_all)])
    return ScanAlignProblem(poses, poses0, scans, normals, edges,
                            name=f"scan_align {num_poses} poses {'full' if full_edges else 'sparse'}")


def pose_graph_scene(num_poses: int = 2000, points_per_scan: int = 500, closures: int = 3000, max_span: int = 30,
                     noise=(0.01, 0.01, np.pi / 1000.0), seed: int = 7) -> ScanAlignProblem:
    """A long 2D scan-alignment pose graph: the scans of scan_align_scene
    joined in a chain (i, i + 1) plus `closures` loop-closure edges (i, j),
    0 < j - i <= max_span; pose 0 is fixed."""
    rng = np.random.default_rng(seed)
    world = 100.0 * rng.uniform(-1, 1, size=(points_per_scan, 2))
    ang = rng.uniform(0, 2 * np.pi, size=points_per_scan)
    nrm = np.stack([np.cos(ang), np.sin(ang)], 1)
    n_all = num_poses + 1
    poses = np.stack([np.array([10.0, 10.0, np.pi]) * rng.uniform(-1, 1, size=3) for _ in range(n_all)])
    scans, normals = [], []
    for x, y, th in poses:
        c, s_ = np.cos(th), np.sin(th)
        R = np.array([[c, -s_], [s_, c]])
        scans.append((world - np.array([x, y])) @ R)
        normals.append(nrm @ R)
    edges = [(i, i + 1) for i in range(num_poses)]
    for _ in range(closures):
        i = int(rng.integers(0, max(num_poses - 1, 1)))
        j = min(num_poses, i + int(rng.integers(2, max_span + 1)))
        if j > i:
            edges.append((i, j))
    sig = np.asarray(noise, dtype=float)
    poses0 = np.array([se2_compose(sig * rng.uniform(-1, 1, size=3), poses[i]) for i in range(1, n_all)])
    return ScanAlignProblem(poses, poses0, scans, normals, edges,
                            name=f"pose graph {num_poses} poses, {len(edges)} edges, {points_per_scan} points/scan")


@dataclass
class RangeScene:
    """A DoubleSection with all four user edge kinds, for the user-edge
    section: U blocks x_u (bu = 3, 6 or 9: a 3D position, then bu - 3 extra
    parameters), V blocks p_v (3D points).
      U-V edge (m = 2): r = (|pos_u - p_v| - d,  a . (pos_u - p_v) + c . extra_u - e)
      U-U edge (m = bu): r = x_a - x_b - delta_ab
      U unary (m = bu):  r = w (x_u - prior_u)
      V unary (m = 3):   r = w (p_v - prior_v)
    Measurements are those of the true parameters plus noise; x0 / p0 start
    from the truth plus a perturbation."""
    bu: int
    x_true: np.ndarray
    p_true: np.ndarray
    x0: np.ndarray
    p0: np.ndarray
    kind: np.ndarray          # per edge
    a: np.ndarray
    b: np.ndarray
    m: np.ndarray
    d: np.ndarray             # U-V: range, linear measurement e, unit a (3), c (bu - 3)
    e: np.ndarray
    avec: np.ndarray
    cvec: np.ndarray
    delta: np.ndarray         # U-U: (n, bu)
    prior: np.ndarray         # U / V unary: (n, bu) (V priors use the first 3 entries)
    w: np.ndarray


def range_scene(bu: int = 3, nu: int = 40, nv: int = 400, obs_per_point: int = 4, uu_edges: int = 60,
                noise: float = 0.01, start: float = 0.05, seed: int = 3) -> RangeScene:
    rng = np.random.default_rng(seed)
    x_true = np.concatenate([rng.uniform(-10, 10, size=(nu, 3)), rng.normal(size=(nu, bu - 3))], 1)
    p_true = rng.uniform(-10, 10, size=(nv, 3)) + np.array([0.0, 0.0, 25.0])
    kind, a, b = [], [], []
    for v in range(nv):
        for u in rng.choice(nu, size=obs_per_point, replace=False):
            kind.append(0)
            a.append(int(u))
            b.append(v)
    for _ in range(uu_edges):
        i, j = rng.choice(nu, size=2, replace=False)
        kind.append(1)
        a.append(int(i))
        b.append(int(j))
    for u in range(nu):   # priors on every U block hold the gauge and the extra parameters
        kind.append(2)
        a.append(u)
        b.append(-1)
    for v in range(0, nv, 7):
        kind.append(3)
        a.append(v)
        b.append(-1)
    kind, a, b = np.array(kind, np.int32), np.array(a, np.int32), np.array(b, np.int32)
    ne = kind.size
    m = np.where(kind == 0, 2, np.where(kind == 3, 3, bu)).astype(np.int32)
    avec = rng.normal(size=(ne, 3))
    avec /= np.linalg.norm(avec, axis=1, keepdims=True)
    cvec = rng.normal(size=(ne, bu - 3))
    d = np.zeros(ne)
    e = np.zeros(ne)
    delta = np.zeros((ne, bu))
    prior = np.zeros((ne, bu))
    w = np.ones(ne)
    for k in range(ne):
        if kind[k] == 0:
            diff = x_true[a[k], :3] - p_true[b[k]]
            d[k] = np.linalg.norm(diff) + noise * rng.normal()
            e[k] = avec[k] @ diff + cvec[k] @ x_true[a[k], 3:] + noise * rng.normal()
        elif kind[k] == 1:
            delta[k] = x_true[a[k]] - x_true[b[k]] + noise * rng.normal(size=bu)
        elif kind[k] == 2:
            prior[k] = x_true[a[k]] + rng.normal(size=bu)
            w[k] = 0.1
        else:
            prior[k, :3] = p_true[a[k]] + noise * rng.normal(size=3)
            w[k] = 0.5
    x0 = x_true + start * rng.normal(size=x_true.shape)
    p0 = p_true + start * rng.normal(size=p_true.shape)
    return RangeScene(bu, x_true, p_true, x0, p0, kind, a, b, m, d, e, avec, cvec, delta, prior, w)

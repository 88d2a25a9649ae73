"""Inputs shared by the adjoint tests (CPU oracle and GPU)."""
import numpy as np


def adjoint_case(P=600, K=300, seed=5):
    """Noisy ellipsoid with non-unit normals (exercises the normalisation) and queries on it."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(P, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    ax = np.array([1.0, 0.8, 0.6])
    pos = v * ax + 0.01 * rng.normal(size=(P, 3))
    nrm = v / ax * rng.uniform(0.5, 2.0, size=(P, 1))
    q = rng.normal(size=(K, 3))
    q = q / np.linalg.norm(q, axis=1, keepdims=True) * ax
    return np.hstack([pos, nrm]), q, rng


def fd_coordinates(pts, depth, rng, count, scale=1.1, eps=1e-4):
    """(point, column) pairs for central differences: positions more than 4 eps inside the bbox
    (a step of 2 eps must not make the point a new extreme, which would move the unit-cube
    transform) and with +-2 eps inside one cell of the grid; normals anywhere."""
    pos = pts[:, :3]
    lo, hi = pos.min(0), pos.max(0)
    s = scale / (hi - lo).max()
    h = 1.0 / 2 ** depth
    out = []
    while len(out) < count:
        i, a, kind = int(rng.integers(len(pts))), int(rng.integers(3)), int(rng.integers(2))
        if kind == 0:
            if pos[i, a] - lo[a] <= 4 * eps or hi[a] - pos[i, a] <= 4 * eps:
                continue
            u = (pos[i, a] - (lo[a] + hi[a]) / 2) * s + 0.5
            if np.floor((u - 2 * s * eps) / h) != np.floor((u + 2 * s * eps) / h):
                continue
        out.append((i, a + 3 * kind))
    return out


def fd_gradient(loss_fn, pts, i, col, eps=1e-4):
    """Fourth-order central difference of loss_fn(points) in entry (i, col)."""
    f = {}
    for m in (-2, -1, 1, 2):
        pm = pts.copy()
        pm[i, col] += m * eps
        f[m] = loss_fn(pm)
    return (f[-2] - 8 * f[-1] + 8 * f[1] - f[2]) / (12 * eps)

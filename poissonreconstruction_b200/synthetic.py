"""Seeded synthetic oriented point clouds for tests and benchmarks.

No public dataset is named for this workload, so every input is generated here from a
fixed seed (numpy PCG64, seed = 20260000 + workload number).  Points are AoS rows
``x y z nx ny nz`` in model space (float64 arrays; the "FP32 storage" workloads are
rounded through float32 first).
"""
import numpy as np

SEED_BASE = 20260000


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def sphere(n=100_000, seed=SEED_BASE + 1, radius=1.0):
    """Uniform on a sphere centred at the origin, exact outward unit normals, FP64."""
    rng = _rng(seed)
    g = rng.standard_normal((n, 3))
    u = g / np.linalg.norm(g, axis=1, keepdims=True)
    return np.ascontiguousarray(np.hstack([radius * u, u]))


def _tangent_rotate(rng, normals, angles):
    """Rotate each unit normal by ``angles`` about a uniformly random tangent axis."""
    a = rng.standard_normal(normals.shape)
    a -= np.sum(a * normals, axis=1, keepdims=True) * normals
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = np.cross(normals, a)  # tangent direction the normal tips towards
    c, s = np.cos(angles)[:, None], np.sin(angles)[:, None]
    out = c * normals + s * b
    return out / np.linalg.norm(out, axis=1, keepdims=True)


def torus(n=2_000_000, seed=SEED_BASE + 2, R=1.0, r=0.35, noise=0.002, normal_sigma=0.05, fp32=True):
    """Area-uniform torus samples (rejection on (R + r cos v)/(R + r)), isotropic Gaussian
    position noise, analytic normals tipped by a Gaussian angle about a random tangent axis."""
    rng = _rng(seed)
    us, vs = [], []
    need = n
    while need > 0:
        m = int(need * 1.6) + 1024
        u = rng.uniform(0, 2 * np.pi, m)
        v = rng.uniform(0, 2 * np.pi, m)
        keep = rng.uniform(0, 1, m) < (R + r * np.cos(v)) / (R + r)
        us.append(u[keep])
        vs.append(v[keep])
        need -= int(keep.sum())
    u = np.concatenate(us)[:n]
    v = np.concatenate(vs)[:n]
    cu, su, cv, sv = np.cos(u), np.sin(u), np.cos(v), np.sin(v)
    pos = np.stack([(R + r * cv) * cu, (R + r * cv) * su, r * sv], axis=1)
    nrm = np.stack([cv * cu, cv * su, sv], axis=1)
    pos = pos + noise * rng.standard_normal(pos.shape)
    nrm = _tangent_rotate(rng, nrm, normal_sigma * rng.standard_normal(n))
    out = np.hstack([pos, nrm])
    if fp32:
        out = out.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(out)


def ellipsoid(n, seed, radii=(1.0, 0.7, 0.5), noise=0.0, fp32=False):
    """Approximately area-uniform ellipsoid samples (rejection on the area element)."""
    rng = _rng(seed)
    a, b, c = radii
    pts = []
    need = n
    while need > 0:
        m = int(need * 2) + 1024
        g = rng.standard_normal((m, 3))
        u = g / np.linalg.norm(g, axis=1, keepdims=True)
        p = u * np.array(radii)
        nrm = p / np.array(radii) ** 2
        dens = np.linalg.norm(nrm, axis=1) * a * b * c / np.array(radii).max()
        keep = rng.uniform(0, 1, m) * dens.max() < dens
        pts.append(np.hstack([p[keep], nrm[keep] / np.linalg.norm(nrm[keep], axis=1, keepdims=True)]))
        need -= int(keep.sum())
    out = np.concatenate(pts)[:n]
    out[:, :3] += noise * rng.standard_normal((n, 3))
    if fp32:
        out = out.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(out)


WORKLOADS = {
    "sphere_100k": dict(fn=sphere, depth=8, point_weight=4.0),
    "torus_2m": dict(fn=torus, depth=10, point_weight=4.0),
}


def _spow(x, e):
    return np.sign(x) * np.abs(x) ** e


def _superquadric_surface(u, v, e1, e2, axes):
    a, b, c = axes
    cv, sv, cu, su = np.cos(v), np.sin(v), np.cos(u), np.sin(u)
    pos = np.stack([a * _spow(cv, e1) * _spow(cu, e2), b * _spow(cv, e1) * _spow(su, e2), c * _spow(sv, e1)], axis=1)
    nrm = np.stack([_spow(cv, 2 - e1) * _spow(cu, 2 - e2) / a, _spow(cv, 2 - e1) * _spow(su, 2 - e2) / b,
                    _spow(sv, 2 - e1) / c], axis=1)
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    return pos, nrm / np.where(ln > 0, ln, 1.0)


def _superquadric_params(rng, n, e1, e2, axes, nu=2048, nv=1024):
    """(u, v) with density proportional to surface area: a parameter cell of an nu x nv grid
    is drawn with probability equal to its share of the area (two triangles of the mapped
    cell), then (u, v) uniform inside the cell.  The area element itself is unbounded on the
    singular parameter lines of a superquadric with exponents below 1, so plain rejection
    against its maximum does not work."""
    ue = np.linspace(-np.pi, np.pi, nu + 1)
    ve = np.linspace(-np.pi / 2, np.pi / 2, nv + 1)
    gu, gv = np.meshgrid(ue, ve, indexing="ij")
    pg = _superquadric_surface(gu.ravel(), gv.ravel(), e1, e2, axes)[0].reshape(nu + 1, nv + 1, 3)
    p00, p10, p01, p11 = pg[:-1, :-1], pg[1:, :-1], pg[:-1, 1:], pg[1:, 1:]
    area = 0.5 * (np.linalg.norm(np.cross(p10 - p00, p01 - p00), axis=2) +
                  np.linalg.norm(np.cross(p10 - p11, p01 - p11), axis=2))
    cdf = np.cumsum(area.ravel())
    cell = np.minimum(np.searchsorted(cdf, rng.uniform(0, cdf[-1], n), side="right"), cdf.size - 1)
    iu, iv = cell // nv, cell % nv
    u = ue[iu] + (ue[1] - ue[0]) * rng.uniform(0, 1, n)
    v = ve[iv] + (ve[1] - ve[0]) * rng.uniform(0, 1, n)
    return u, v


def superquadric(n=1_000_000, seed=SEED_BASE + 3, e1=0.5, e2=0.8, axes=(1.0, 0.7, 0.5), max_tilt_deg=20.0,
                 fp32=True):
    """Superquadric samples (area-weighted parameter cells), analytic normals tilted by an angle uniform in
    [0, max_tilt_deg] about a random tangent axis; FP32-rounded."""
    rng = _rng(seed)
    u, v = _superquadric_params(rng, n, e1, e2, axes)
    pos, nrm = _superquadric_surface(u, v, e1, e2, axes)
    nrm = _tangent_rotate(rng, nrm, np.deg2rad(max_tilt_deg) * rng.uniform(0, 1, n))
    out = np.hstack([pos, nrm])
    if fp32:
        out = out.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(out)


def superquadric_queries(k=200_000, seed=SEED_BASE + 103, e1=0.5, e2=0.8, axes=(1.0, 0.7, 0.5)):
    """Query points on the true superquadric surface (a seed of their own)."""
    rng = _rng(seed)
    u, v = _superquadric_params(rng, k, e1, e2, axes)
    return np.ascontiguousarray(_superquadric_surface(u, v, e1, e2, axes)[0])


def batch_clouds(count=256, seed=SEED_BASE + 4, lo=10_000, hi=500_000):
    """Batched workload: `count` clouds with sizes log-uniform in [lo, hi], each an ellipsoid
    (radii U[0.3, 1.0]) or a torus (R, r from U[0.3, 1.0] with r < R), analytic normals,
    position noise 0.001, FP32-rounded.  Returns [(points, depth)], depth 7 below 40k points,
    8 below 160k, else 9."""
    rng = _rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        sub = int(rng.integers(1 << 31))
        if rng.uniform() < 0.5:
            radii = tuple(rng.uniform(0.3, 1.0, 3))
            pts = ellipsoid(n, sub, radii=radii, noise=0.001, fp32=True)
        else:
            a, b = sorted(rng.uniform(0.3, 1.0, 2))
            while b - a < 1e-3:
                a, b = sorted(rng.uniform(0.3, 1.0, 2))
            pts = torus(n, sub, R=b, r=a, noise=0.001, normal_sigma=0.0, fp32=True)
        depth = 7 if n < 40_000 else (8 if n < 160_000 else 9)
        out.append((pts, depth))
    return out


def union_of_spheres(n=20_000_000, seed=SEED_BASE + 5, count=32, rmin=0.05, rmax=0.3, outlier_frac=0.01,
                     fp32=True, sample_seed=None):
    """Large workload: the outer surface of the union of `count` overlapping spheres (centres
    uniform in the unit cube, radii uniform in [rmin, rmax]) with exact outward normals, plus
    `outlier_frac` of the points uniform in the cube with random unit normals; n points in all,
    FP32-rounded.  Surface samples are drawn per sphere in proportion to its area and kept when
    they lie inside no other sphere.  sample_seed: other samples of the same spheres (the spheres
    come from `seed`)."""
    rng = _rng(seed)
    c = rng.uniform(0.0, 1.0, (count, 3))
    r = rng.uniform(rmin, rmax, count)
    if sample_seed is not None:
        rng = _rng(sample_seed)
    n_out = int(round(outlier_frac * n))
    n_surf = n - n_out
    area = r * r
    chunks, have = [], 0
    while have < n_surf:
        m = int((n_surf - have) * 1.5) + 4096
        k = rng.choice(count, m, p=area / area.sum())
        g = rng.standard_normal((m, 3))
        u = g / np.linalg.norm(g, axis=1, keepdims=True)
        pos = c[k] + r[k, None] * u
        inside = np.zeros(m, dtype=bool)
        for j in range(count):
            d2 = np.sum((pos - c[j]) ** 2, axis=1)
            inside |= (d2 < r[j] * r[j]) & (k != j)
        keep = ~inside
        chunks.append(np.hstack([pos[keep], u[keep]]))
        have += int(keep.sum())
    surf = np.concatenate(chunks)[:n_surf]
    g = rng.standard_normal((n_out, 3))
    out_pts = np.hstack([rng.uniform(0.0, 1.0, (n_out, 3)), g / np.linalg.norm(g, axis=1, keepdims=True)])
    pts = np.vstack([surf, out_pts])
    pts = pts[rng.permutation(n)]
    if fp32:
        pts = pts.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(pts)

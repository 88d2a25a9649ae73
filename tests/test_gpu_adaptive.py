"""Adaptive (narrow-band) reconstruction on the GPU: no counterpart in the reference crate, which
refines every leaf to max_depth (src/fem_tree.rs:83-93).  The band system is the dense degree-2
system restricted to the active bricks with the prolonged coarse solution fixed outside them, so
it is checked against the dense path and against the oracle's dense degree-2 restatement:

* every brick active: right-hand side and operator equal the dense path's (1e-13), and so do the
  solution (1e-8) and the mesh;
* a partial band: the right-hand side equals the oracle's dense b on the band nodes, A_BB v the
  oracle's A applied to v extended by zero (1e-12), the fixed coarse function equals the B2
  subdivision of the coarse solution (restated here with numpy), the solution satisfies the
  oracle's equations on the band (relative residual 1e-9 under the oracle's operator with the
  coarse function outside), the iso value is the oracle's evaluation of that function, and the
  band's mesh vertices lie on the oracle's marching cubes of it;
* depth 12 on a union of spheres with outliers: converged, and the mixed-precision solution within
  1e-5 of the FP64 one.
"""
import numpy as np
import pytest

import oracle
import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

pytestmark = pytest.mark.gpu


def _spread(v):
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0x3FF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x09249249)
    return v


def _natural_to_morton(idx, depth):
    res = 1 << depth
    x, y, z = idx % res, (idx // res) % res, idx // (res * res)
    return (_spread(x) | (_spread(y) << np.uint64(1)) | (_spread(z) << np.uint64(2))).astype(np.int64)


def _morton_to_natural_vec(v_morton, depth):
    n = 8 ** depth
    m = _natural_to_morton(np.arange(n), depth)
    return v_morton[m]


def _composite_weights(L):
    """The B2 subdivision (fine 2i + k <- coarse i, k = -1..2, weights 1/4 3/4 3/4 1/4) applied L
    times to a unit coarse coefficient: (first fine offset, weights)."""
    cur, lo = np.array([1.0]), 0
    for _ in range(L):
        nxt = np.zeros(2 * len(cur) + 2)
        for i, c in enumerate(cur):
            for k, w in zip((-1, 0, 1, 2), (0.25, 0.75, 0.75, 0.25)):
                nxt[2 * (lo + i) + k - (2 * lo - 1)] += c * w
        cur, lo = nxt, 2 * lo - 1
    return lo, cur


def _prolong(xc_nat, dc, d):
    """g = sum_I W(f - 2^L I) x_c[I] per axis (natural order in and out)."""
    L, rc, rf = d - dc, 1 << dc, 1 << d
    lo, w = _composite_weights(L)
    P = np.zeros((rf, rc))
    for f in range(rf):
        for i in range(rc):
            k = f - (1 << L) * i - lo
            if 0 <= k < len(w):
                P[f, i] = w[k]
    x = xc_nat.reshape(rc, rc, rc)  # [z][y][x]
    x = np.einsum("ai,zyi->zya", P, x)
    x = np.einsum("bj,zjx->zbx", P, x)
    x = np.einsum("ck,kyx->cyx", P, x)
    return x.ravel()


def _adaptive(depth, coarse, **kw):
    return prb.ReconstructParams(depth=depth, coarse_depth=coarse, degree=2, point_weight=4.0, **kw)


def test_full_refinement_is_the_dense_system(ctx):
    pts = synthetic.torus(20000, seed=22)
    D, Dc = 6, 3
    mesh_d, st_d = ctx.reconstruct(pts, prb.ReconstructParams(depth=D, degree=2, point_weight=4.0,
                                                              target_rel_residual=1e-10))
    b_d, x_d = ctx.rhs(), ctx.coefficients()  # Morton order
    v = np.random.default_rng(6).standard_normal(8 ** D)
    y_d = ctx.apply_operator(v, prb.PR_PRECISION_FP64)
    mesh_a, st_a = ctx.reconstruct(pts, _adaptive(D, Dc, band_flags=prb.PR_BAND_FULL, target_rel_residual=1e-10))
    assert st_a.converged == 1 and st_a.rel_residual <= 1e-10
    d, dc, codes = ctx.band_info()
    assert (d, dc, len(codes)) == (D, Dc, 8 ** (D - 3))
    mo = _natural_to_morton(prb.band_natural_index(codes, D), D)
    b_a = ctx.band_vector(0)
    assert np.max(np.abs(b_a - b_d[mo])) <= 1e-13 * np.max(np.abs(b_d))
    vb = np.empty_like(v)
    vb[:] = v[mo]
    y_a = ctx.band_apply(vb)
    assert np.max(np.abs(y_a - y_d[mo])) <= 1e-13 * np.max(np.abs(y_d))
    f = ctx.band_vector(1)
    assert np.linalg.norm(f - x_d[mo]) <= 1e-8 * np.linalg.norm(x_d)
    assert abs(st_a.iso_value - st_d.iso_value) <= 1e-8 * abs(st_d.iso_value)
    assert len(mesh_a.triangles) > 0 and abs(len(mesh_a.triangles) - len(mesh_d.triangles)) <= 0.001 * len(
        mesh_d.triangles)
    from scipy.spatial import cKDTree
    diag = np.linalg.norm(pts[:, :3].max(0) - pts[:, :3].min(0))
    dist, _ = cKDTree(mesh_d.vertices).query(mesh_a.vertices)
    assert np.quantile(dist, 0.999) <= 1e-6 * diag


@pytest.mark.parametrize("precision", [prb.PR_PRECISION_FP64, prb.PR_PRECISION_MIXED])
def test_partial_band_against_the_oracle(ctx, precision, capsys):
    pts = synthetic.torus(20000, seed=23)
    D, Dc, pw = 7, 4, 4.0
    unit, m = oracle.to_unit(pts)
    # the coarse level: the dense degree-2 reconstruction at Dc with the same parameters
    ctx.solve(pts, prb.ReconstructParams(depth=Dc, degree=2, point_weight=pw, precision=precision,
                                         target_rel_residual=1e-10))
    xc = _morton_to_natural_vec(ctx.coefficients(), Dc)
    mesh, st = ctx.reconstruct(pts, _adaptive(D, Dc, precision=precision, target_rel_residual=1e-10))
    assert st.converged == 1
    _, _, codes = ctx.band_info()
    assert 0 < len(codes) < 8 ** (D - 3)
    nat = prb.band_natural_index(codes, D)
    mo = _natural_to_morton(nat, D)
    tree = oracle.Tree2(D, unit, pw)
    b_ref = tree.rhs()
    b = ctx.band_vector(0)
    assert np.max(np.abs(b - b_ref[mo])) <= 1e-12 * np.max(np.abs(b_ref))
    # A_BB v = (A v_ext)_B, v_ext = v on the band, 0 elsewhere
    v = np.random.default_rng(7).standard_normal(len(nat))
    v_ext = np.zeros(8 ** D)
    v_ext[mo] = v
    y_ref = tree.apply(v_ext)[mo]
    assert np.max(np.abs(ctx.band_apply(v) - y_ref)) <= 1e-12 * np.max(np.abs(y_ref))
    # the fixed coarse function
    g_all = _prolong(xc, Dc, D)
    g = ctx.band_vector(2)
    assert np.max(np.abs(g - g_all[nat])) <= 1e-12 * np.max(np.abs(g_all))
    # the solution solves the oracle's equations on the band with g outside
    f = ctx.band_vector(1)
    u_nat = g_all.copy()
    u_nat[nat] = f
    u = np.empty_like(u_nat)
    u[_natural_to_morton(np.arange(8 ** D), D)] = u_nat
    r = (b_ref - tree.apply(u))[mo]
    relres = np.linalg.norm(r) / np.linalg.norm(b_ref[mo])
    with capsys.disabled():
        print("\nadaptive depth %d over coarse %d: %d of %d bricks, oracle residual on the band %.2e (GPU %.2e)"
              % (D, Dc, len(codes), 8 ** (D - 3), relres, st.rel_residual))
    assert relres <= (1e-9 if precision == prb.PR_PRECISION_FP64 else 1e-8)
    # iso = mean of that function at the points; band mesh vertices on the oracle's mesh of it
    iso_ref = float(np.mean(oracle.evaluate2(D, u, unit[:, :3])))
    assert abs(st.iso_value - iso_ref) <= 1e-9 * abs(iso_ref)
    v_ref, t_ref = oracle.extract_surface2(D, u, st.iso_value)
    assert 0 < len(mesh.triangles) <= len(t_ref)
    mm = np.asarray(m).reshape(4, 4).T
    v_unit = mesh.vertices @ mm[:3, :3].T + mm[:3, 3]
    from scipy.spatial import cKDTree
    dist, _ = cKDTree(v_ref).query(v_unit)
    assert dist.max() <= 1e-9


def test_depth12_union_of_spheres(ctx, capsys):
    """Depth 12 over 9 on 1 M points of the union of spheres with outliers: the mixed-precision
    solve within 1e-5 of the FP64 one, and the adjoint (mean chi^2 at 50 k other samples of the
    surface) converged in both precisions with gradients within 1e-3 of each other."""
    pts = synthetic.union_of_spheres(1_000_000)
    q = synthetic.union_of_spheres(50_000, outlier_frac=0.0, sample_seed=synthetic.SEED_BASE + 56)[:, :3]
    D, Dc = 12, 9
    _, st64 = ctx.reconstruct(pts, _adaptive(D, Dc, precision=prb.PR_PRECISION_FP64, target_rel_residual=1e-6))
    f64 = ctx.band_vector(1)
    _, dp64, dn64, a64 = ctx.loss_backward(q)
    mesh, st = ctx.reconstruct(pts, _adaptive(D, Dc, target_rel_residual=1e-6))
    f32 = ctx.band_vector(1)
    _, dp, dn, a32 = ctx.loss_backward(q)
    _, _, codes = ctx.band_info()
    err = np.linalg.norm(f32 - f64) / np.linalg.norm(f64)
    gp = np.linalg.norm(dp - dp64) / np.linalg.norm(dp64)
    gn = np.linalg.norm(dn - dn64) / np.linalg.norm(dn64)
    with capsys.disabled():
        print("\nadaptive depth 12 over 9, 1M points: %d bricks (%.3g nodes), mixed %.0f ms (%d PCG, %d refinements, "
              "relres %.1e), FP64 %.0f ms, coefficient error %.2e, %d triangles, peak %.1f GB; adjoint %.0f ms "
              "(%d PCG), %d of %d queries off the band, gradients mixed vs FP64 %.2e / %.2e"
              % (len(codes), 512.0 * len(codes), 1000 * st.time_total, st.pcg_iterations, st.refinement_steps,
                 st.rel_residual, 1000 * st64.time_total, err, len(mesh.triangles), st.peak_device_bytes / 1e9,
                 1000 * a32.time_total, a32.pcg_iterations, a32.queries_off_band, len(q), gp, gn))
    assert st.converged == 1 and st64.converged == 1
    assert err <= 1e-5
    assert len(mesh.triangles) > 0 and np.all(np.isfinite(mesh.vertices))
    assert a32.converged == 1 and a64.converged == 1
    assert gp <= 1e-3 and gn <= 1e-3


def _band_params(D, Dc, fp64=True, target=1e-12, **kw):
    return prb.ReconstructParams(depth=D, coarse_depth=Dc, degree=2, point_weight=4.0, max_iters=400,
                                 precision=prb.PR_PRECISION_FP64 if fp64 else prb.PR_PRECISION_MIXED,
                                 target_rel_residual=target, **kw)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_band_adjoint_full_band_is_the_dense_adjoint(ctx):
    """With every brick active the band system is the dense degree-2 system and the fine function
    does not depend on the coarse solution (its adjoint right-hand side P^T (E^T g - A lambda)
    vanishes with the band adjoint's residual): chi and the gradients equal the dense adjoint's."""
    from tests.adjoint_cases import adjoint_case
    pts, q, _ = adjoint_case(P=3000, K=800, seed=41)
    D, Dc = 6, 3
    ctx.solve(pts, _band_params(D, Dc, band_flags=prb.PR_BAND_FULL))
    chi_a, dp_a, dn_a, st_a = ctx.loss_backward(q)
    assert st_a.converged == 1 and st_a.queries_off_band == 0
    ctx.solve(pts, prb.ReconstructParams(depth=D, degree=2, point_weight=4.0, max_iters=400,
                                         precision=prb.PR_PRECISION_FP64, target_rel_residual=1e-12))
    chi_d, dp_d, dn_d, st_d = ctx.loss_backward(q)
    assert _rel(chi_a, chi_d) <= 1e-9 and abs(st_a.loss - st_d.loss) <= 1e-9 * abs(st_d.loss)
    assert _rel(dp_a, dp_d) <= 1e-7 and _rel(dn_a, dn_d) <= 1e-7


def test_band_adjoint_finite_differences(ctx, capsys):
    """A partial band (depth 7 over 4): the gradient of mean chi^2 at queries on the surface against
    fourth-order central differences of the band forward (FP64 solves to 1e-12) on coordinates
    whose gradient is at least 10% of the largest of its kind, at <= 1e-4 relative; linear in the
    upstream gradient; the forward state left as it was."""
    from tests.adjoint_cases import adjoint_case, fd_coordinates, fd_gradient
    pts, q, rng = adjoint_case(P=4000, K=1000, seed=43)
    D, Dc = 7, 4
    p = _band_params(D, Dc)
    ctx.solve(pts, p)
    _, _, codes = ctx.band_info()
    assert 0 < len(codes) < 8 ** (D - 3)
    f_before = ctx.band_vector(1)
    chi, dp, dn, st = ctx.loss_backward(q)
    assert st.converged == 1
    assert np.array_equal(ctx.band_vector(1), f_before)
    g1, g2 = rng.standard_normal(len(q)), rng.standard_normal(len(q))
    _, a1, b1, _ = ctx.loss_backward(q, dl_dchi=g1)
    _, a2, b2, _ = ctx.loss_backward(q, dl_dchi=g2)
    _, a12, b12, _ = ctx.loss_backward(q, dl_dchi=2.0 * g1 - g2)
    assert _rel(a12, 2.0 * a1 - a2) <= 1e-9 and _rel(b12, 2.0 * b1 - b2) <= 1e-9

    def loss(points):
        ctx.solve(points, p)
        return ctx.loss_backward(q)[3].loss

    grads = np.hstack([dp, dn])
    big = [np.abs(grads[:, :3]).max(), np.abs(grads[:, 3:]).max()]
    coords = [(i, c) for i, c in fd_coordinates(pts, D, rng, 4000) if abs(grads[i, c]) >= 0.1 * big[c // 3]]
    coords = [coords[k] for k in rng.choice(len(coords), min(12, len(coords)), replace=False)]
    errs = []
    for i, col in coords:
        fd = fd_gradient(loss, pts, i, col)
        errs.append(abs(fd - grads[i, col]) / abs(grads[i, col]))
    with capsys.disabled():
        print("\nband adjoint, depth 7 over 4: %d bricks, %d of %d queries off the band, %d central differences, "
              "max relative error %.2e" % (len(codes), st.queries_off_band, len(q), len(errs), max(errs)))
    assert len(errs) >= 8 and max(errs) <= 1e-4, errs

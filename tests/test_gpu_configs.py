"""GPU parity at the benchmark workloads' own sizes, against the CPU oracle.

* Plain method (100,000 points on the unit sphere, depth 8, screening weight 4): the
  converged FP64 and mixed-precision solves against the oracle's FP64 solve of the crate's fine
  system; the marching cubes of the GPU coefficients bit-exact against the oracle's
  extract_surface; the crate's own cascade (cg_iters = 8) against the oracle's, with the
  coarse right-hand side of build_system_at_depth bit-exact and the deviation of the
  (8-colour Gauss-Seidel) schedule reported.
* Depth 10 on the 2,000,000-point torus of the headline benchmark: the right-hand side
  bit-exact, A v element-wise within 1e-13 of the oracle's FP64 matrix-free operator, and the
  first 20 iterations of the crate's FP64 CG loop (||r||^2 after every iteration and the 20th
  iterate) against the oracle's.
* Degree 2 at depth 9 on the same torus: right-hand side and FP64 A v against the oracle's
  degree-2 restatement (depth 10 would need two 2-minute single-socket passes of the 125-point
  oracle stencil; depth 9 keeps the test within a minute).

The oracle's converged solve at depth 8 starts from the GPU's FP64 solution (a cold CG needs
thousands of iterations at 16.8 M unknowns): the oracle's own CG then drives the residual under
the ORACLE's operator to 1e-13, so a GPU solution of a different system would start far from
convergence and fail the comparison.
"""
import numpy as np
import pytest

import oracle
import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

pytestmark = pytest.mark.gpu

COEF_TOL = 1e-6    # relative L2 of coefficients vs the FP64 oracle
VERT_TOL = 1e-5    # x bbox diagonal
OP64_TOL = 1e-13   # FP64 operator, max-abs error / max-abs value
CG_TOL = 1e-9      # CG iterates: ||r||^2 history (relative) and x_20 (relative L2)


def _host_gb():
    try:
        import psutil
        return psutil.virtual_memory().available / 1e9
    except ImportError:
        return float("inf")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _permute_lex_to_morton(v_lex, depth):
    """Coarse vectors of the oracle are lexicographic (x fastest); the GPU's are Morton."""
    res = 1 << depth
    z, y, x = np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij")
    m = np.array([oracle.morton(int(a), int(b), int(c)) for a, b, c in
                  zip(x.ravel(), y.ravel(), z.ravel())], dtype=np.int64)
    out = np.empty_like(v_lex)
    out[m] = v_lex
    return out


@pytest.fixture(scope="module")
def sphere100k():
    pts = synthetic.sphere(100_000)
    unit, m = oracle.to_unit(pts)
    return pts, unit, m


def test_plain_method_sphere_depth8_converged_vs_oracle(ctx, sphere100k, capsys):
    pts, unit, m = sphere100k
    depth, pw = 8, 4.0
    tree = oracle.Tree(depth, unit)
    b_ref = tree.rhs(pw)

    sols = {}
    runs = [("fp64_tight", prb.PR_PRECISION_FP64, 1e-12), ("mixed_tight", prb.PR_PRECISION_MIXED, 1e-12),
            ("fp64", prb.PR_PRECISION_FP64, 1e-6), ("mixed", prb.PR_PRECISION_MIXED, 1e-6)]
    runs += [("mixed_%.0e" % tol, prb.PR_PRECISION_MIXED, tol) for tol in (1e-7, 1e-8, 1e-9, 1e-10)]
    for name, prec, tol in runs:
        mesh, st = ctx.reconstruct(pts, prb.ReconstructParams(depth=depth, point_weight=pw, precision=prec,
                                                              target_rel_residual=tol, max_iters=400))
        assert st.converged == 1 and st.rel_residual <= tol, (name, st.rel_residual)
        if name == "fp64_tight":
            assert np.array_equal(ctx.rhs(), b_ref), "right-hand side differs from the oracle"
        sols[name] = (ctx.coefficients(), mesh, st)

    # the oracle's own CG on its own (matrix-free) operator, from the GPU's FP64 solution
    tree.release_field()
    x0 = sols["fp64_tight"][0]
    r0 = np.linalg.norm(b_ref - tree.apply_mf(x0, pw)) / np.linalg.norm(b_ref)
    assert r0 <= 1e-11, "GPU solution's residual under the oracle's operator: %.3e" % r0
    x_ref, it, rr = tree.solve_converged_mf(b_ref, pw, tol=1e-13, maxit=20000, x0=x0)
    assert rr <= 1e-13

    errs = {k: _rel(v[0], x_ref) for k, v in sols.items()}
    with capsys.disabled():
        print("\nplain method, depth 8: oracle residual of the GPU FP64 solution %.2e; oracle CG %d more "
              "iterations; coefficient error vs the oracle: %s"
              % (r0, it, ", ".join("%s %.2e" % kv for kv in errs.items())))
    assert errs["fp64_tight"] <= COEF_TOL and errs["mixed_tight"] <= COEF_TOL
    # at the default 1e-6 residual the coefficients are within 1e-4 (reported above); the
    # residual that meets the 1e-6 coefficient bound is checked below
    assert errs["fp64"] <= 1e-4 and errs["mixed"] <= 1e-4
    meets = [tol for name, _, tol in runs if name.startswith("mixed") and errs[name] <= COEF_TOL]
    with capsys.disabled():
        print("plain method, depth 8: largest mixed target residual whose coefficients meet %.0e: %s"
              % (COEF_TOL, max(meets) if meets else None))
    assert meets

    # marching cubes of the GPU coefficients: bit-exact against the oracle's extract_surface
    x_mixed, mesh, st = sols["mixed"]
    v_ref, t_ref = oracle.extract_surface(depth, x_mixed, st.iso_value)
    assert np.array_equal(mesh.triangles, t_ref)
    # the default mixed mesh against the oracle's mesh of its converged solution
    iso_ref = oracle.iso(depth, x_ref, unit)
    v_conv, _ = oracle.extract_surface(depth, x_ref, iso_ref)
    minv = np.asarray(oracle.mat4_inverse(m)).reshape(4, 4).T  # column-major -> rows
    v_conv = v_conv @ minv[:3, :3].T + minv[:3, 3]
    lo, hi = pts[:, :3].min(0), pts[:, :3].max(0)
    diag = np.linalg.norm(hi - lo)
    from scipy.spatial import cKDTree
    d, _ = cKDTree(v_conv).query(mesh.vertices)
    with capsys.disabled():
        print("plain method, depth 8: mixed (1e-6) vertices vs the oracle's converged mesh: max %.2e, "
              "99.9%% %.2e of the bbox diagonal" % (d.max() / diag, np.quantile(d, 0.999) / diag))
    assert np.quantile(d, 0.999) <= VERT_TOL * diag


def test_plain_method_sphere_depth8_reference_schedule(ctx, sphere100k, capsys):
    """The crate's cascade with cg_iters = 8 (the plain method's 8 iterations per depth)."""
    pts, unit, _ = sphere100k
    depth, pw = 8, 4.0
    params = prb.ReconstructParams(depth=depth, point_weight=pw, solve_mode=prb.PR_SOLVE_REFERENCE_SCHEDULE,
                                   cg_iters=8)
    mesh, st = ctx.reconstruct(pts, params)
    x_gpu = ctx.coefficients()
    dc, brhs_gpu = ctx.coarse_rhs()
    assert dc == depth - 2
    tree = oracle.Tree(depth, unit)
    brhs_ref = _permute_lex_to_morton(tree.coarse_rhs(pw), dc)
    assert np.array_equal(brhs_gpu, brhs_ref), "coarse right-hand side differs from build_system_at_depth"
    x_ref, info = tree.solve_reference(pw, 8, params.cg_accuracy)
    # the solution both schedules approach: the GPU's FP64 solve to 1e-12, checked under the
    # oracle's operator
    b = tree.rhs(pw)
    tree.release_field()
    ctx.reconstruct(pts, prb.ReconstructParams(depth=depth, point_weight=pw, precision=prb.PR_PRECISION_FP64,
                                               target_rel_residual=1e-12, max_iters=400))
    x_conv = ctx.coefficients()
    assert np.linalg.norm(b - tree.apply_mf(x_conv, pw)) <= 1e-11 * np.linalg.norm(b)
    dev = _rel(x_gpu, x_ref)
    with capsys.disabled():
        print("\nreference schedule, depth 8, cg_iters 8: GPU (8-colour GS) vs oracle (Morton GS) %.3e; "
              "oracle schedule vs converged %.3e; GPU schedule vs converged %.3e; oracle CG iterations %s"
              % (dev, _rel(x_ref, x_conv), _rel(x_gpu, x_conv), list(info)))
    assert np.all(np.isfinite(x_gpu)) and len(mesh.triangles) > 0
    assert dev <= max(0.5, 2 * _rel(x_ref, x_conv))
    # both schedules are the same distance from the solution they approach
    assert _rel(x_gpu, x_conv) <= 2 * _rel(x_ref, x_conv) + 1e-3


@pytest.fixture(scope="module")
def torus2m():
    return synthetic.torus(2_000_000)


def test_depth10_rhs_operator_and_cg_iterates_vs_oracle(torus2m, capsys):
    if _host_gb() < 70:
        pytest.skip("needs about 70 GB of free host memory for the depth-10 oracle (%.0f GB free)" % _host_gb())
    pts = torus2m
    depth, pw = 10, 4.0
    with prb.Context(0) as ctx:
        ctx.solve(pts, prb.ReconstructParams(depth=depth, point_weight=pw))
        unit, _ = oracle.to_unit(pts)
        tree = oracle.Tree(depth, unit)
        b = tree.rhs(pw)
        tree.release_field()
        assert np.array_equal(ctx.rhs(), b), "depth-10 right-hand side differs from the oracle"
        v = np.random.default_rng(10).standard_normal(tree.n)
        y_ref = tree.apply_mf(v, pw)
        y = ctx.apply_operator(v, prb.PR_PRECISION_FP64)
        op_err = float(np.max(np.abs(y - y_ref)) / np.max(np.abs(y_ref)))
        del y, y_ref, v
        assert op_err <= OP64_TOL, op_err
        x_gpu, it_gpu, delta_gpu = ctx.cg_reference(20, 1e-30)
    x_ref, it_ref, delta_ref = tree.cg_mf(b, pw, 20, 1e-30)
    hist = float(np.max(np.abs(delta_gpu - delta_ref) / delta_ref))
    xerr = _rel(x_gpu, x_ref)
    with capsys.disabled():
        print("\ndepth 10, 2M-point torus: b bit-exact; A v max error %.2e; CG ||r||^2 history max rel %.2e, "
              "x_20 rel L2 %.2e (||r_20||/||r_0|| = %.3e)"
              % (op_err, hist, xerr, np.sqrt(delta_ref[-1] / delta_ref[0])))
    assert it_gpu == it_ref == 20
    assert hist <= CG_TOL and xerr <= CG_TOL


def test_degree2_depth9_rhs_and_operator_vs_oracle(torus2m, capsys):
    pts = torus2m
    depth, pw = 9, 4.0
    with prb.Context(0) as ctx:
        ctx.solve(pts, prb.ReconstructParams(depth=depth, point_weight=pw, degree=2))
        unit, _ = oracle.to_unit(pts)
        tree = oracle.Tree2(depth, unit, pw)
        b_ref = tree.rhs()
        b = ctx.rhs()
        b_err = float(np.max(np.abs(b - b_ref)) / np.max(np.abs(b_ref)))
        v = np.random.default_rng(9).standard_normal(len(b))
        y_ref = tree.apply(v)
        y = ctx.apply_operator(v, prb.PR_PRECISION_FP64)
        op_err = float(np.max(np.abs(y - y_ref)) / np.max(np.abs(y_ref)))
    with capsys.disabled():
        print("\ndegree 2, depth 9, 2M-point torus: b max error %.2e, A v max error %.2e" % (b_err, op_err))
    assert b_err <= 1e-12 and op_err <= 1e-12

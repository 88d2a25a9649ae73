"""Adjoint (gradients of a loss on the implicit function) on the GPU, through the C ABI:
against the FP64 CPU oracle's adjoint, against finite differences of the GPU forward, and
through the torch.autograd bridge.  No counterpart in the reference crate; the forward it
differentiates is src/fem_tree.rs:130-299 and :490-513."""
import numpy as np
import pytest

import oracle
import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic
from tests.adjoint_cases import adjoint_case, fd_coordinates, fd_gradient

pytestmark = pytest.mark.gpu


def _params(depth, fp64=True, target=1e-12):
    return prb.ReconstructParams(depth=depth, point_weight=4.0,
                                 precision=prb.PR_PRECISION_FP64 if fp64 else prb.PR_PRECISION_MIXED,
                                 target_rel_residual=target, max_iters=400)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("depth", [4, 5, 6])
@pytest.mark.parametrize("upstream", [False, True])
def test_adjoint_matches_oracle_fp64(ctx, depth, upstream):
    """FP64 GPU solve and adjoint vs the oracle's FP64 adjoint: relative L2 <= 1e-7."""
    pts, q, rng = adjoint_case(P=2000, K=700, seed=11 + depth)
    g = rng.normal(size=len(q)) if upstream else None
    ctx.solve(pts, _params(depth))
    chi, dp, dn, st = ctx.loss_backward(q, dl_dchi=g)
    chi_o, dp_o, dn_o, L_o = oracle.loss_backward(pts, q, depth, dl_dchi=g)
    assert st.converged == 1 and st.rel_residual <= 1e-12
    assert _rel(chi, chi_o) <= 1e-9
    assert st.loss == pytest.approx(L_o, rel=1e-9)
    assert _rel(dp, dp_o) <= 1e-7
    assert _rel(dn, dn_o) <= 1e-7


def test_adjoint_mixed_precision(ctx):
    """FP32 multigrid PCG + FP64 refinement at the default 1e-6 target: gradients within
    relative L2 1e-5 of the oracle's."""
    D = 6
    pts, q, _ = adjoint_case(P=4000, K=1000, seed=3)
    ctx.solve(pts, _params(D, fp64=False, target=1e-6))
    _, dp, dn, st = ctx.loss_backward(q)
    _, dp_o, dn_o, _ = oracle.loss_backward(pts, q, D)
    assert st.converged == 1 and st.rel_residual <= 1e-6
    assert _rel(dp, dp_o) <= 1e-5
    assert _rel(dn, dn_o) <= 1e-5


def test_adjoint_finite_differences_gpu(ctx):
    """Central differences (fourth order, step 1e-4, model space) of the GPU forward (FP64
    solve to 1e-13) vs the GPU adjoint, on 16 coordinates: <= 1e-4 relative."""
    D = 6
    pts, q, rng = adjoint_case(P=3000, K=800, seed=21)
    p = _params(D, target=1e-13)

    def loss(points):
        ctx.solve(points, p)
        _, _, m = ctx.info()
        m = m.reshape(4, 4).T
        chi = ctx.evaluate(q @ m[:3, :3].T + m[:3, 3])
        return float(np.mean(chi ** 2))

    ctx.solve(pts, p)
    _, dp, dn, st = ctx.loss_backward(q)
    grads = np.hstack([dp, dn])
    gmax = np.abs(grads).max(axis=0)
    for i, col in fd_coordinates(pts, D, rng, 16):
        fd = fd_gradient(loss, pts, i, col)
        an = grads[i, col]
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-2 * gmax[col]), (i, col, fd, an)


def test_adjoint_is_deterministic_and_linear(ctx):
    """Same call twice -> identical bits; gradients are linear in the upstream gradient."""
    D = 6
    pts, q, rng = adjoint_case(P=3000, K=900, seed=4)
    ctx.solve(pts, _params(D, fp64=False, target=1e-6))
    g1, g2 = rng.normal(size=len(q)), rng.normal(size=len(q))
    _, a1, b1, _ = ctx.loss_backward(q, dl_dchi=g1)
    _, a1b, b1b, _ = ctx.loss_backward(q, dl_dchi=g1)
    assert np.array_equal(a1, a1b) and np.array_equal(b1, b1b)
    _, a2, b2, _ = ctx.loss_backward(q, dl_dchi=g2)
    _, a3, b3, _ = ctx.loss_backward(q, dl_dchi=g1 + g2)
    assert _rel(a1 + a2, a3) <= 1e-5 and _rel(b1 + b2, b3) <= 1e-5


def test_adjoint_one_shot_and_errors(ctx):
    pts, q, _ = adjoint_case(P=1500, K=400, seed=8)
    p = _params(5)
    chi, dp, dn, st = prb.loss_backward(pts, q, p)
    ctx.solve(pts, p)
    chi2, dp2, dn2, _ = ctx.loss_backward(q)
    assert np.array_equal(chi, chi2) and np.array_equal(dp, dp2) and np.array_equal(dn, dn2)
    # the reference schedule does not solve A x = b: refused
    ctx.solve(pts, prb.ReconstructParams(depth=5, point_weight=4.0, solve_mode=prb.PR_SOLVE_REFERENCE_SCHEDULE,
                                         cg_iters=8))
    with pytest.raises(prb.ReconstructError) as e:
        ctx.loss_backward(q)
    assert e.value.code == prb.PR_ERR_STATE
    ctx.solve(pts, p)
    with pytest.raises(prb.ReconstructError) as e:
        ctx.loss_backward(np.zeros((0, 3)))
    assert e.value.code == prb.PR_ERR_INVALID_ARGUMENT
    with pytest.raises(prb.ReconstructError) as e:
        ctx.loss_backward(np.array([[0.0, np.nan, 0.0]]))
    assert e.value.code == prb.PR_ERR_INVALID_ARGUMENT


def test_autograd_bridge():
    torch = pytest.importorskip("torch")
    from poissonreconstruction_b200.autograd import implicit_function
    pts, q, _ = adjoint_case(P=2000, K=500, seed=9)
    params = _params(5)
    pos = torch.tensor(pts[:, :3], requires_grad=True)
    nrm = torch.tensor(pts[:, 3:], requires_grad=True)
    chi = implicit_function(pos, nrm, torch.tensor(q), params)
    loss = (chi ** 2).mean()
    loss.backward()
    _, dp, dn, st = prb.loss_backward(pts, q, params)
    assert float(loss) == pytest.approx(st.loss, rel=1e-12)
    assert _rel(pos.grad.numpy(), dp) <= 1e-12
    assert _rel(nrm.grad.numpy(), dn) <= 1e-12


def test_adjoint_superquadric_depth8(ctx):
    """Superquadric workload (eps1 0.5, eps2 0.8, axes 1/0.7/0.5, normals tilted up to 20 deg,
    queries on the true surface) at depth 8 with 200k points: mixed-precision gradients vs the
    FP64 GPU adjoint (1e-4 relative L2), and 8 finite differences of the FP64 GPU forward."""
    D = 8
    pts = synthetic.superquadric(200_000, seed=synthetic.SEED_BASE + 3)
    q = synthetic.superquadric_queries(40_000)
    ctx.solve(pts, _params(D, target=1e-12))
    _, dp64, dn64, st64 = ctx.loss_backward(q)
    assert st64.converged == 1
    ctx.solve(pts, _params(D, fp64=False, target=1e-6))
    _, dp, dn, st = ctx.loss_backward(q)
    assert st.converged == 1
    assert _rel(dp, dp64) <= 1e-4 and _rel(dn, dn64) <= 1e-4
    p = _params(D, target=1e-12)

    def loss(points):
        ctx.solve(points, p)
        _, _, m = ctx.info()
        m = m.reshape(4, 4).T
        chi = ctx.evaluate(q @ m[:3, :3].T + m[:3, 3])
        return float(np.mean(chi ** 2))

    rng = np.random.default_rng(1)
    grads = np.hstack([dp64, dn64])
    gmax = np.abs(grads).max(axis=0)
    for i, col in fd_coordinates(pts, D, rng, 8):
        fd = fd_gradient(loss, pts, i, col)
        an = grads[i, col]
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-2 * gmax[col]), (i, col, fd, an)


def test_adjoint_superquadric_depth9_full_size(ctx, capsys):
    """The adjoint workload at its own size: 1,000,000 superquadric points (eps1 0.5, eps2 0.8,
    axes 1/0.7/0.5, normals tilted up to 20 deg), depth 9, loss = mean chi^2 at 200,000 seeded
    points on the true surface.  The FP64 GPU gradient against 64 central differences (step 1e-4,
    fourth order: four forward solves to a 1e-12 residual each) at <= 1e-4 relative, with no
    floor: the coordinates are drawn among those whose gradient is at least 10% of the largest
    gradient of the same kind (position or normal), off the bbox extremes (the unit-cube transform
    is held fixed) and 2 steps away from any cell face.  The mixed-precision gradient is checked
    against the FP64 one (1e-4 relative L2).  The oracle's FP64 adjoint is not run at this size:
    its CSR system at depth 9 (134 M unknowns) does not fit the host's time; it is compared with
    the GPU at depths 4-6 above."""
    D = 9
    pts = synthetic.superquadric(1_000_000)
    q = synthetic.superquadric_queries(200_000)
    p = _params(D, target=1e-12)
    ctx.solve(pts, p)
    _, dp64, dn64, st64 = ctx.loss_backward(q)
    assert st64.converged == 1
    ctx.solve(pts, _params(D, fp64=False, target=1e-6))
    _, dp, dn, st = ctx.loss_backward(q)
    assert st.converged == 1
    assert _rel(dp, dp64) <= 1e-4 and _rel(dn, dn64) <= 1e-4

    def loss(points):
        ctx.solve(points, p)
        _, _, m = ctx.info()
        m = m.reshape(4, 4).T
        chi = ctx.evaluate(q @ m[:3, :3].T + m[:3, 3])
        return float(np.mean(chi ** 2))

    grads = np.hstack([dp64, dn64])
    big = [np.abs(grads[:, :3]).max(), np.abs(grads[:, 3:]).max()]
    rng = np.random.default_rng(64)
    coords = [(i, c) for i, c in fd_coordinates(pts, D, rng, 20000)
              if abs(grads[i, c]) >= 0.1 * big[c // 3]]
    assert len(coords) >= 64
    coords = [coords[k] for k in rng.choice(len(coords), 64, replace=False)]
    errs = []
    for i, col in coords:
        fd = fd_gradient(loss, pts, i, col)
        an = grads[i, col]
        errs.append(abs(fd - an) / abs(an))
    with capsys.disabled():
        print("\nadjoint, depth 9, 1M points, 200k queries: 64 central differences, relative error max %.2e, "
              "median %.2e; mixed vs FP64 gradient %.2e / %.2e; adjoint solve %.1f ms (mixed), total %.1f ms"
              % (max(errs), float(np.median(errs)), _rel(dp, dp64), _rel(dn, dn64), 1000 * st.time_solve,
                 1000 * st.time_total))
    assert max(errs) <= 1e-4, errs


# ---------------------------------------------------------------- degree 2 (quadratic B-splines)
def _params2(depth, fp64=True, target=1e-12):
    return prb.ReconstructParams(depth=depth, point_weight=4.0, degree=2,
                                 precision=prb.PR_PRECISION_FP64 if fp64 else prb.PR_PRECISION_MIXED,
                                 target_rel_residual=target, max_iters=400)


def test_adjoint_degree2_against_oracle_differences(ctx):
    """Degree-2 gradients of the FP64 GPU adjoint against fourth-order central differences of the
    oracle's own degree-2 forward (CG to 1e-13), at <= 1e-4 relative on coordinates whose gradient
    is at least 5% of the largest of its kind; the loss value against the oracle's."""
    D = 4
    pts, q, rng = adjoint_case(P=1500, K=500, seed=21)
    ctx.solve(pts, _params2(D, target=1e-12))
    chi, dp, dn, st = ctx.loss_backward(q)
    assert st.converged == 1
    assert st.loss == pytest.approx(oracle.loss2(pts, q, D), rel=1e-9)
    grads = np.hstack([dp, dn])
    big = [np.abs(grads[:, :3]).max(), np.abs(grads[:, 3:]).max()]
    coords = [(i, c) for i, c in fd_coordinates(pts, D, rng, 400) if abs(grads[i, c]) >= 0.05 * big[c // 3]][:12]
    assert len(coords) >= 8
    for i, col in coords:
        fd = fd_gradient(lambda p: oracle.loss2(p, q, D), pts, i, col)
        assert abs(fd - grads[i, col]) <= 1e-4 * abs(grads[i, col]), (i, col, fd, grads[i, col])


def test_adjoint_degree2_gpu_differences_and_precision(ctx, capsys):
    """Depth 7, 50k superquadric points, 10k queries: 16 central differences of the GPU's own
    degree-2 forward (FP64 solves to 1e-12) at <= 1e-4 relative with no floor, the mixed-precision
    gradient against the FP64 one (1e-4 relative L2), linearity in the upstream gradient, and the
    context's forward solution left intact by the adjoint solve."""
    D = 7
    pts = synthetic.superquadric(50_000, seed=synthetic.SEED_BASE + 33)
    q = synthetic.superquadric_queries(10_000, seed=synthetic.SEED_BASE + 133)
    p = _params2(D, target=1e-12)
    ctx.solve(pts, p)
    x_before = ctx.coefficients()
    _, dp64, dn64, st64 = ctx.loss_backward(q)
    assert st64.converged == 1
    assert np.array_equal(ctx.coefficients(), x_before)
    rng = np.random.default_rng(77)
    g1, g2 = rng.standard_normal(len(q)), rng.standard_normal(len(q))
    _, a1, b1, _ = ctx.loss_backward(q, dl_dchi=g1)
    _, a2, b2, _ = ctx.loss_backward(q, dl_dchi=g2)
    _, a12, b12, _ = ctx.loss_backward(q, dl_dchi=2.0 * g1 - g2)
    assert _rel(a12, 2.0 * a1 - a2) <= 1e-9 and _rel(b12, 2.0 * b1 - b2) <= 1e-9

    def loss(points):
        ctx.solve(points, p)
        _, _, m = ctx.info()
        m = m.reshape(4, 4).T
        chi = ctx.evaluate(q @ m[:3, :3].T + m[:3, 3])
        return float(np.mean(chi ** 2))

    grads = np.hstack([dp64, dn64])
    big = [np.abs(grads[:, :3]).max(), np.abs(grads[:, 3:]).max()]
    coords = [(i, c) for i, c in fd_coordinates(pts, D, rng, 4000) if abs(grads[i, c]) >= 0.1 * big[c // 3]]
    coords = [coords[k] for k in rng.choice(len(coords), min(16, len(coords)), replace=False)]
    errs = []
    for i, col in coords:
        fd = fd_gradient(loss, pts, i, col)
        errs.append(abs(fd - grads[i, col]) / abs(grads[i, col]))
    ctx.solve(pts, _params2(D, fp64=False, target=1e-6))
    _, dp, dn, st = ctx.loss_backward(q)
    with capsys.disabled():
        print("\ndegree-2 adjoint, depth 7: %d central differences, max relative error %.2e; mixed vs FP64 %.2e / %.2e"
              % (len(errs), max(errs), _rel(dp, dp64), _rel(dn, dn64)))
    assert len(errs) >= 8 and max(errs) <= 1e-4, errs
    assert st.converged == 1 and _rel(dp, dp64) <= 1e-4 and _rel(dn, dn64) <= 1e-4

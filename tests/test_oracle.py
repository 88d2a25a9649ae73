"""CPU oracle: pinned by the reference crate's own unit tests (ported here) and by
hand-derived known answers.  No GPU needed."""
import os
import re

import numpy as np
import pytest

import oracle
from poissonreconstruction_b200 import synthetic
from tests.adjoint_cases import adjoint_case, fd_coordinates, fd_gradient


# ---------------------------------------------------------------- ported crate unit tests
def test_cg_simple():
    """src/solvers.rs:235-268: CG on tridiag(-1,2,-1), b = 1, x_i = (i+1)(n-i)/2."""
    n = 10
    ptr, col, val = [0], [], []
    for i in range(n):
        if i > 0:
            col.append(i - 1); val.append(-1.0)
        col.append(i); val.append(2.0)
        if i < n - 1:
            col.append(i + 1); val.append(-1.0)
        ptr.append(len(col))
    x, it = oracle.csr_cg(ptr, col, val, np.ones(n), np.zeros(n), 100, 1e-10)
    expected = np.array([(i + 1) * (n - i) / 2.0 for i in range(n)])
    assert np.all(np.abs(x - expected) < 1e-6)


def test_sparse_matrix_multiply():
    """src/sparse.rs:175-196."""
    y = oracle.csr_spmv([0, 2, 3, 4], [0, 1, 1, 2], [2.0, 1.0, 3.0, 4.0], [1.0, 2.0, 3.0])
    assert np.allclose(y, [4.0, 6.0, 12.0], atol=1e-10)


def test_bbox():
    """src/geometry.rs:437-446."""
    pts = np.array([[-1.0, -2.0, -3.0, 0, 0, 1], [1.0, 2.0, 3.0, 0, 0, 1]])
    lo, hi = oracle.bbox(pts)
    assert np.array_equal((lo + hi) * 0.5, [0.0, 0.0, 0.0])
    assert np.array_equal(hi - lo, [2.0, 4.0, 6.0])
    assert abs((hi - lo).max() - 6.0) < 1e-10


def test_mat4_inverse_identity():
    """src/geometry.rs:424-434."""
    m = np.zeros(16)
    m[[0, 5, 10, 15]] = 1.0
    inv = oracle.mat4_inverse(m)
    p = np.array([1.0, 2.0, 3.0])
    r = oracle.transform_point(inv, oracle.transform_point(m, p))
    assert np.all(np.abs(r - p) < 1e-10)


def test_bspline_degree1():
    """src/bspline.rs:408-411 values of N_1, for the evaluation kernel bspline1
    (src/fem_tree.rs:640-642), which is N_1 shifted to peak at t = 1."""
    assert oracle.bspline1(0.5) == 0.5
    assert oracle.bspline1(1.0) == 1.0
    assert oracle.bspline1(1.5) == 0.5
    assert oracle.bspline1(0.0) == 0.0 and oracle.bspline1(2.0) == 0.0
    assert oracle.bspline1(-0.1) == 0.0 and oracle.bspline1(2.1) == 0.0


def test_sorted_tree_leaf_order_is_morton():
    """src/octree.rs:145-153,235-248: the depth-first leaf order of the full tree is the
    Morton order with x in bit 0 (the FEM index of src/fem_tree.rs:104-121)."""
    D = 3
    order = []

    def dfs(d, off):
        if d == D:
            order.append(off)
            return
        for i in range(8):
            dfs(d + 1, (off[0] * 2 + (i & 1), off[1] * 2 + ((i >> 1) & 1), off[2] * 2 + ((i >> 2) & 1)))

    dfs(0, (0, 0, 0))
    assert len(order) == 8 ** D
    assert [oracle.morton(*o) for o in order] == list(range(8 ** D))


# ---------------------------------------------------------------- hand-derived known answers
def test_stiffness_constants():
    """src/fem_tree.rs:39-48: centre 8/3 h, faces exactly 0 (dropped), edges -h/6, corners -h/12."""
    h = 1.0 / 256
    assert oracle.stiffness_entry(h, 0, 0, 0) == (2.0 / 3 * 2.0 / 3 * 2 * 3) * h or \
        abs(oracle.stiffness_entry(h, 0, 0, 0) - 8.0 / 3 * h) < 1e-18
    for d in [(1, 0, 0), (0, -1, 0), (0, 0, 1)]:
        assert oracle.stiffness_entry(h, *d) == 0.0
    for d in [(1, 1, 0), (-1, 0, 1), (0, 1, -1)]:
        assert abs(oracle.stiffness_entry(h, *d) + h / 6) < 1e-18
    for d in [(1, 1, 1), (-1, 1, -1)]:
        assert abs(oracle.stiffness_entry(h, *d) + h / 12) < 1e-18


def test_csr_is_the_21_point_stencil():
    """Assembled rows (no screening): interior rows have 21 entries, symmetric."""
    unit = np.array([[0.5, 0.5, 0.5, 0.0, 0.0, 1.0]])
    t = oracle.Tree(3, unit)
    ptr, col, val = t.assemble(0.0)
    nnz_row = np.diff(ptr.astype(np.int64))
    i = oracle.morton(3, 4, 2)
    assert nnz_row[i] == 21
    assert nnz_row[oracle.morton(0, 0, 0)] == 1 + 3 + 1  # centre, 3 edges, 1 corner
    A = np.zeros((t.n, t.n))
    for r in range(t.n):
        A[r, col[ptr[r]:ptr[r + 1]]] = val[ptr[r]:ptr[r + 1]]
    assert np.array_equal(A, A.T)
    assert np.all(np.linalg.eigvalsh(A) > 0)


def test_single_point_splat():
    """src/fem_tree.rs:130-178: one point splats trilinear weights, normalised and negated."""
    D = 3
    h = 1.0 / 8
    p = np.array([[2.25 * h, 3.5 * h, 4.75 * h, 0.0, 0.6, 0.8]])
    t = oracle.Tree(D, p)
    nf, w = t.normal_field()
    tx, ty, tz = 0.25, 0.5, 0.75
    for k in range(8):
        dx, dy, dz = k & 1, (k >> 1) & 1, k >> 2
        wk = (tx if dx else 1 - tx) * (ty if dy else 1 - ty) * (tz if dz else 1 - tz)
        idx = oracle.morton(2 + dx, 3 + dy, 4 + dz)
        assert w[idx] == pytest.approx(wk, rel=1e-15)
        assert np.allclose(nf[idx], [-0.0, -0.6, -0.8])
    assert np.count_nonzero(w) == 8


def test_evaluate_shifted_one_cell():
    """src/fem_tree.rs:490-513,645-649: at integer grid positions evaluate(k) = x[k-1]
    per axis, 0 at k = 0 and 2 x[res-1] per axis at k = res."""
    D = 2
    res = 4
    rng = np.random.default_rng(0)
    x = rng.standard_normal(64)
    h = 1.0 / res
    for (kx, ky, kz) in [(1, 1, 1), (3, 2, 1), (0, 2, 2), (4, 1, 1), (4, 4, 2), (4, 4, 4)]:
        v = oracle.evaluate(D, x, np.array([[kx * h, ky * h, kz * h]]))[0]
        mult = np.prod([0 if k == 0 else (2 if k == res else 1) for k in (kx, ky, kz)])
        node = oracle.morton(*[res - 1 if k == res else max(k - 1, 0) for k in (kx, ky, kz)])
        assert v == pytest.approx(mult * x[node], rel=1e-15, abs=0)


def _corner_values_numpy(D, x):
    """Corner values of every cell by the shifted-gather rule, independently of the oracle."""
    res = 1 << D
    idx = np.arange(res ** 3)
    def comp(m):
        r = np.zeros_like(m)
        for b in range(10):
            r |= ((m >> (3 * b)) & 1) << b
        return r
    gx, gy, gz = comp(idx), comp(idx >> 1), comp(idx >> 2)
    grid = np.zeros((res, res, res))
    grid[gz, gy, gx] = x
    co = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    cv = np.zeros((res ** 3, 8))
    for k, (a, b, c) in enumerate(co):
        kx, ky, kz = gx + a, gy + b, gz + c
        mult = np.ones(res ** 3)
        for kk in (kx, ky, kz):
            mult = mult * np.where(kk == 0, 0, np.where(kk == res, 2, 1))
        nx, ny, nz = [np.clip(np.where(kk == res, res - 1, kk - 1), 0, res - 1) for kk in (kx, ky, kz)]
        cv[:, k] = mult * grid[nz, ny, nx]
    return cv


def test_mc_triangle_count_matches_table():
    """Triangle count of the oracle's MC = sum over cells of the table's triangle count for
    the case computed independently in numpy."""
    D = 3
    rng = np.random.default_rng(5)
    x = rng.standard_normal(8 ** D)
    iso = 0.1
    v, t = oracle.extract_surface(D, x, iso)
    cv = _corner_values_numpy(D, x)
    cases = ((cv < iso) * (1 << np.arange(8))).sum(axis=1)
    ntri = [int((oracle.mc_tri_row(c) >= 0).sum()) // 3 for c in range(256)]
    assert len(t) == sum(ntri[c] for c in cases)
    assert t.max() < len(v) and len(np.unique(t)) == len(v)


def test_edge_table_derivation_matches_reference(reference_src):
    """The crate's EDGE_TABLE (src/fem_tree.rs:13-30) equals the corner-sign derivation."""
    path = os.path.join(reference_src, "fem_tree.rs")
    if not os.path.exists(path):
        pytest.skip("reference sources not present")
    m = re.search(r"const EDGE_TABLE: \[u16; 256\] = \[(.*?)\];", open(path).read(), re.S)
    et = [int(v, 16) for v in re.findall(r"0x[0-9a-f]+", m.group(1))]
    assert [oracle.mc_edge_mask(c) for c in range(256)] == et


def test_tri_table_matches_reference(reference_src):
    """The packed table equals the crate's TRI_TABLE (src/tri_table.inl)."""
    path = os.path.join(reference_src, "tri_table.inl")
    if not os.path.exists(path):
        pytest.skip("reference sources not present")
    rows = re.findall(r"\[([-0-9, ]+)\]", open(path).read())
    rows = [[int(v) for v in r.split(",")] for r in rows if len(r.split(",")) == 16]
    for c in range(256):
        assert list(oracle.mc_tri_row(c)) == rows[c]


# ---------------------------------------------------------------- oracle self-consistency
def test_converged_solve_residual():
    pts = synthetic.sphere(3000, seed=7)
    unit, _ = oracle.to_unit(pts)
    t = oracle.Tree(4, unit)
    x, it, rr = t.solve_converged(4.0, tol=1e-12)
    assert rr < 1e-11
    ptr, col, val = t.assemble(4.0)
    b = t.rhs(4.0)
    r = b - oracle.csr_spmv(ptr, col, val, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-11


def test_reference_pipeline_runs():
    pts = synthetic.sphere(5000, seed=3)
    v, t, st, c = oracle.reconstruct(pts, depth=4, point_weight=4.0, solve_mode=0, want_coeffs=True)
    assert st["fem_nodes"] == 8 ** 4 and len(t) > 100 and len(v) > 50
    assert t.max() < len(v)


def test_empty_input():
    """src/reconstructor.rs:28: empty input -> empty mesh, default stats."""
    v, t, st, c = oracle.reconstruct(np.zeros((0, 6)), depth=4)
    assert len(v) == 0 and len(t) == 0 and st["iso_value"] == 0.0


# ---------------------------------------------------------------- adjoint (no reference counterpart)
@pytest.mark.parametrize("upstream", [False, True])
def test_adjoint_matches_finite_differences(upstream):
    """Oracle's analytic gradient (adjoint solve) vs central differences of the oracle's own
    forward (fourth-order 5-point stencil, step 1e-4 in model space: the second-order stencil's
    own error reaches 2e-4 where the splat normalisation 1/w is large): relative error <= 1e-4
    against the coordinate's gradient, or against 1% of the largest entry of that column."""
    D, eps = 5, 1e-4
    pts, q, rng = adjoint_case()
    g = rng.normal(size=len(q)) if upstream else None
    chi, dp, dn, L = oracle.loss_backward(pts, q, D, dl_dchi=g)
    assert L == pytest.approx(oracle.loss(pts, q, D, dl_dchi=g), rel=1e-12)
    grads = np.hstack([dp, dn])
    gmax = np.abs(grads).max(axis=0)
    for i, col in fd_coordinates(pts, D, rng, 10):
        fd = fd_gradient(lambda p: oracle.loss(p, q, D, dl_dchi=g), pts, i, col, eps)
        an = grads[i, col]
        ref = max(abs(an), 1e-2 * gmax[col])
        assert abs(fd - an) <= 1e-4 * ref, (i, col, fd, an)


# ---------------------------------------------------------------- degree 2 (extension)
def test_deg2_constants_exact():
    """1-D integrals of the quadratic B-spline (src/bspline.rs:334-345) at offsets -2..2."""
    m, s, g = oracle.deg2_constants()
    assert np.allclose(m, [1 / 120, 13 / 60, 11 / 20, 13 / 60, 1 / 120], rtol=0, atol=1e-15)
    assert np.allclose(s, [-1 / 6, -1 / 3, 1.0, -1 / 3, -1 / 6], rtol=0, atol=1e-15)
    assert np.allclose(g, [1 / 24, 5 / 12, 0.0, -5 / 12, -1 / 24], rtol=0, atol=1e-15)


def test_deg2_basis_matches_crate_values():
    """src/bspline.rs:412-417: N_2(0.5) = 0.125, N_2(1.5) = 0.75.  Node i carries
    N_2(x/h - i + 1), so at s = x/h = 1.5 nodes 0, 1, 2 weigh N_2(2.5), N_2(1.5), N_2(0.5)."""
    D = 2
    h = 1.0 / (1 << D)
    p = np.array([[1.5 * h, 1.5 * h, 1.5 * h]])
    for node, weight in (((1, 1, 1), 0.75 ** 3), ((2, 1, 1), 0.125 * 0.75 ** 2), ((0, 2, 1), 0.125 ** 2 * 0.75),
                         ((3, 1, 1), 0.0)):
        x = np.zeros(8 ** D)
        x[oracle.morton(*node)] = 1.0
        assert oracle.evaluate2(D, x, p)[0] == weight


def _kron_operator(D, pw_unit=None):
    """Dense h (S M M + M S M + M M S) with truncated rows, in Morton order (x fastest axis)."""
    m, s, _ = oracle.deg2_constants()
    res = 1 << D

    def band(c):
        a = np.zeros((res, res))
        for i in range(res):
            for d in range(-2, 3):
                if 0 <= i + d < res:
                    a[i, i + d] = c[d + 2]
        return a

    M, S = band(m), band(s)
    K = (np.kron(np.kron(M, M), S) + np.kron(np.kron(M, S), M) + np.kron(np.kron(S, M), M)) / res
    perm = np.array([oracle.morton(i % res, (i // res) % res, i // (res * res)) for i in range(res ** 3)])
    P = np.zeros_like(K)
    P[perm[:, None], perm[None, :]] = K
    return P


def test_deg2_operator_matches_kronecker_definition():
    pts = synthetic.sphere(500, seed=31)
    unit, _ = oracle.to_unit(pts)
    D = 3
    t = oracle.Tree2(D, unit, 0.0)  # no screening: A = K exactly (wg = 0)
    K = _kron_operator(D)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(t.n)
    assert np.allclose(t.apply(x), K @ x, rtol=0, atol=1e-13 * np.abs(K @ x).max())
    assert np.allclose(K, K.T)
    assert np.linalg.eigvalsh(K).min() > 0


def test_deg2_rhs_matches_kronecker_definition():
    m, s, g = oracle.deg2_constants()
    pts = synthetic.sphere(800, seed=32)
    unit, _ = oracle.to_unit(pts)
    D = 3
    res = 1 << D
    t = oracle.Tree2(D, unit, 0.0)
    nf, w = t.normal_field()

    def band(c):
        a = np.zeros((res, res))
        for i in range(res):
            for d in range(-2, 3):
                if 0 <= i + d < res:
                    a[i, i + d] = c[d + 2]
        return a

    M, G = band(m), band(g)
    perm = np.array([oracle.morton(i % res, (i // res) % res, i // (res * res)) for i in range(res ** 3)])
    nat = nf[perm]  # natural order (x fastest)
    b = (np.kron(np.kron(M, M), G) @ nat[:, 0] + np.kron(np.kron(M, G), M) @ nat[:, 1] +
         np.kron(np.kron(G, M), M) @ nat[:, 2]) / res ** 2
    b_ref = t.rhs()[perm]
    assert np.allclose(b_ref, b, rtol=0, atol=1e-14 * np.abs(b).max())


def test_deg2_normal_field_is_normalised_splat():
    pts = synthetic.sphere(300, seed=33)
    unit, _ = oracle.to_unit(pts, 0.5)  # unit coordinates in [0.25, 0.75]: all 27 nodes inside
    t = oracle.Tree2(3, unit, 0.0)
    nf, w = t.normal_field()
    assert np.isclose(w.sum(), len(pts))  # partition of unity: 27 weights of a point sum to 1
    hit = w > 0
    assert np.all(np.linalg.norm(nf[hit], axis=1) <= 1.0 + 1e-12)


def test_deg2_solve_and_pipeline():
    pts = synthetic.sphere(3000, seed=34)
    unit, _ = oracle.to_unit(pts)
    t = oracle.Tree2(4, unit, 4.0)
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal(t.n), rng.standard_normal(t.n)
    assert abs(y @ t.apply(x) - x @ t.apply(y)) <= 1e-12 * abs(y @ t.apply(x))
    sol, it, rr = t.solve(tol=1e-12)
    assert rr <= 1e-12
    v, tri, iso, rr2, c = oracle.reconstruct2(pts, 4)
    assert rr2 <= 1e-12 and len(tri) > 100 and tri.max() < len(v)
    # closed surface: every edge is shared by exactly two triangles
    e = np.sort(np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    assert np.all(counts == 2)


# ---------------------------------------------------------------- matrix-free oracle operator
@pytest.mark.parametrize("depth,pw", [(3, 4.0), (4, 4.0), (5, 4.0), (4, 0.0)])
def test_matrix_free_operator_and_cg_match_the_csr(depth, pw):
    """The matrix-free operator (used where the crate's CSR does not fit in host memory) gives
    the CSR product of assemble_system to rounding, and its CG (the crate's loop) the same
    iterates as the CSR CG."""
    pts = synthetic.sphere(3000, seed=7)
    unit, _ = oracle.to_unit(pts)
    t = oracle.Tree(depth, unit)
    ptr, col, val = t.assemble(pw)
    x = np.random.default_rng(depth).standard_normal(t.n)
    y_csr, y_mf = t.spmv(x), t.apply_mf(x, pw)
    assert np.max(np.abs(y_csr - y_mf)) <= 1e-14 * np.max(np.abs(y_csr))
    b = t.rhs(pw)
    x_mf, it_mf, delta = t.cg_mf(b, pw, 20, 1e-30)
    x_csr, it_csr = oracle.csr_cg(ptr, col, val, b, np.zeros(t.n), 20, 1e-30)
    assert it_mf == it_csr == 20 and np.all(np.isfinite(delta))
    assert np.linalg.norm(x_mf - x_csr) <= 1e-13 * np.linalg.norm(x_csr)
    xc, _, rr = t.solve_converged(pw, tol=1e-12)
    t.release_field()
    xm, _, rm = t.solve_converged_mf(b, pw, tol=1e-12)
    assert rm <= 1e-12 and np.linalg.norm(xm - xc) <= 1e-12 * np.linalg.norm(xc)

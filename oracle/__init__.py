"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (``liboracle.so``).

The oracle is a C++ FP64 restatement of the reference crate's reconstruction path
(``oracle.cpp`` cites the Rust file:line of every step).  It is imported by the tests,
by ``bench.py``'s CPU-baseline leg and by the smoke check — never by the library.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = C.c_double
_u64 = C.c_uint64
_u32 = C.c_uint32
_i32 = C.c_int32
_p = C.c_void_p


class OrcMesh(C.Structure):
    _fields_ = [("verts", C.POINTER(C.c_double)), ("nv", C.c_uint64),
                ("tris", C.POINTER(C.c_uint64)), ("nt", C.c_uint64)]


class OrcParams(C.Structure):
    _fields_ = [("depth", _u32), ("scale", _d), ("cg_accuracy", _d), ("cg_iters", _u64),
                ("point_weight", _d), ("solve_mode", _i32), ("target_rel_residual", _d),
                ("max_iters", _u64)]


class OrcStats(C.Structure):
    _fields_ = [("iso_value", _d), ("fem_nodes", _u64), ("mesh_vertices", _u64),
                ("mesh_triangles", _u64), ("rel_residual", _d), ("iterations", _u64),
                ("time_tree", _d), ("time_solve", _d), ("time_extract", _d), ("time_total", _d)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    sig = {
        "orc_num_threads": (C.c_int, []),
        "orc_bspline1": (_d, [_d]),
        "orc_stiffness_entry": (_d, [_d, C.c_int, C.c_int, C.c_int]),
        "orc_morton": (_u64, [_u64, _u64, _u64]),
        "orc_mc_edge_mask": (_u32, [_u32]),
        "orc_mc_tri_row": (None, [_u32, _p]),
        "orc_bbox": (None, [_p, _u64, _p, _p]),
        "orc_unit_cube_transform": (None, [_p, _p, _d, _p]),
        "orc_mat4_inverse": (None, [_p, _p]),
        "orc_transform_point": (None, [_p, _p, _p]),
        "orc_transform_points": (None, [_p, _p, _u64, _p]),
        "orc_tree_new": (_p, [_u32, _p, _u64]),
        "orc_tree_free": (None, [_p]),
        "orc_tree_nodes": (_u64, [_p]),
        "orc_tree_normal_field": (None, [_p, _p, _p]),
        "orc_tree_rhs": (None, [_p, _d, _p]),
        "orc_tree_assemble": (C.c_int64, [_p, _d]),
        "orc_tree_csr": (None, [_p, _p, _p, _p]),
        "orc_tree_spmv": (C.c_int, [_p, _p, _p]),
        "orc_tree_solve_reference": (C.c_int, [_p, _d, _u64, _d, _p, _p]),
        "orc_tree_coarse_rhs": (C.c_int, [_p, _d, _p]),
        "orc_tree_prolongate": (C.c_int, [_p, _p, _u32, _p]),
        "orc_tree_solve_converged": (_u64, [_p, _d, _d, _u64, _p, _p]),
        "orc_tree_apply_mf": (None, [_p, _d, _p, _p]),
        "orc_tree_release_field": (None, [_p]),
        "orc_tree_cg_mf": (_u64, [_p, _d, _p, _p, _u64, _d, _p]),
        "orc_tree_solve_converged_mf": (_u64, [_p, _d, _p, _d, _u64, _p, _p]),
        "orc_evaluate": (_d, [_u32, _p, _d, _d, _d]),
        "orc_evaluate_many": (None, [_u32, _p, _p, _u64, _u64, _p]),
        "orc_iso": (_d, [_u32, _p, _p, _u64]),
        "orc_extract_surface": (C.c_int, [_u32, _p, _d, C.POINTER(OrcMesh)]),
        "orc_mesh_free": (None, [C.POINTER(OrcMesh)]),
        "orc_csr_cg": (_u64, [_u64, _p, _p, _p, _p, _p, _u64, _d]),
        "orc_csr_spmv": (None, [_u64, _p, _p, _p, _p, _p]),
        "orc_csr_gs_sweep": (None, [_u64, _p, _p, _p, _p, _p]),
        "orc_reconstruct": (C.c_int, [_p, _u64, C.POINTER(OrcParams), C.POINTER(OrcMesh),
                                      C.POINTER(OrcStats), _p]),
        "orc_deg2_constants": (None, [_p, _p, _p]),
        "orc_evaluate2": (_d, [_u32, _p, _d, _d, _d]),
        "orc_tree2_new": (_p, [_u32, _p, _u64, _d]),
        "orc_tree2_free": (None, [_p]),
        "orc_tree2_normal_field": (None, [_p, _p, _p]),
        "orc_tree2_rhs": (None, [_p, _p]),
        "orc_tree2_apply": (None, [_p, _p, _p]),
        "orc_tree2_solve": (_u64, [_p, _d, _u64, _p, _p]),
        "orc_tree2_release_field": (None, [_p]),
        "orc_cg2_new": (_p, [_p, _p]),
        "orc_cg1_new": (_p, [_p, _d, _p]),
        "orc_cg_step": (_d, [_p]),
        "orc_cg_free": (None, [_p]),
        "orc_extract_surface2": (C.c_int, [_u32, _p, _d, C.POINTER(OrcMesh)]),
        "orc_reconstruct2": (C.c_int, [_p, _u64, _u32, _d, _d, _d, _u64, C.POINTER(OrcMesh), _p, _p, _p]),
        "orc_loss": (_d, [_p, _u64, _u32, _d, _d, _p, _u64, _p, _d]),
        "orc_loss_backward": (C.c_int, [_p, _u64, _u32, _d, _d, _p, _u64, _p, _d, _p, _p, _p, _p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


# ------------------------------------------------------------------ scalar helpers
def num_threads():
    return lib().orc_num_threads()


def bspline1(t):
    return lib().orc_bspline1(float(t))


def stiffness_entry(h, dx, dy, dz):
    return lib().orc_stiffness_entry(float(h), int(dx), int(dy), int(dz))


def morton(x, y, z):
    return lib().orc_morton(int(x), int(y), int(z))


def mc_edge_mask(case):
    return lib().orc_mc_edge_mask(int(case))


def mc_tri_row(case):
    out = np.zeros(16, dtype=np.int32)
    lib().orc_mc_tri_row(int(case), _ptr(out))
    return out


# ------------------------------------------------------------------ geometry
def bbox(pts6):
    pts6 = _f64(pts6, (-1, 6))
    lo, hi = np.zeros(3), np.zeros(3)
    lib().orc_bbox(_ptr(pts6), pts6.shape[0], _ptr(lo), _ptr(hi))
    return lo, hi


def unit_cube_transform(bmin, bmax, scale):
    m = np.zeros(16)
    lib().orc_unit_cube_transform(_ptr(_f64(bmin)), _ptr(_f64(bmax)), float(scale), _ptr(m))
    return m


def mat4_inverse(m):
    out = np.zeros(16)
    lib().orc_mat4_inverse(_ptr(_f64(m)), _ptr(out))
    return out


def transform_point(m, p):
    out = np.zeros(3)
    lib().orc_transform_point(_ptr(_f64(m)), _ptr(_f64(p)), _ptr(out))
    return out


def transform_points(m, pts6):
    pts6 = _f64(pts6, (-1, 6))
    out = np.zeros_like(pts6)
    lib().orc_transform_points(_ptr(_f64(m)), _ptr(pts6), pts6.shape[0], _ptr(out))
    return out


def to_unit(pts6, scale=1.1):
    """bbox -> unit-cube transform -> transformed points (src/reconstructor.rs:31-40)."""
    lo, hi = bbox(pts6)
    m = unit_cube_transform(lo, hi, scale)
    return transform_points(m, pts6), m


# ------------------------------------------------------------------ tree
class Tree:
    """FEMTree of the crate at a fixed depth, built from unit-cube points (splat included)."""

    def __init__(self, depth, unit6):
        self.depth = int(depth)
        self.unit = _f64(unit6, (-1, 6))
        self._h = lib().orc_tree_new(self.depth, _ptr(self.unit), self.unit.shape[0])
        self.n = lib().orc_tree_nodes(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_tree_free(self._h)
            self._h = None

    def normal_field(self):
        nf = np.zeros((self.n, 3))
        w = np.zeros(self.n)
        lib().orc_tree_normal_field(self._h, _ptr(nf), _ptr(w))
        return nf, w

    def rhs(self, pw):
        b = np.zeros(self.n)
        lib().orc_tree_rhs(self._h, float(pw), _ptr(b))
        return b

    def assemble(self, pw):
        nnz = lib().orc_tree_assemble(self._h, float(pw))
        ptr = np.zeros(self.n + 1, dtype=np.uint64)
        col = np.zeros(nnz, dtype=np.uint32)
        val = np.zeros(nnz)
        lib().orc_tree_csr(self._h, _ptr(ptr), _ptr(col), _ptr(val))
        return ptr, col, val

    def spmv(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        if lib().orc_tree_spmv(self._h, _ptr(x), _ptr(y)) != 0:
            raise RuntimeError("assemble() first")
        return y

    def solve_reference(self, pw, cg_iters, acc):
        x = np.zeros(self.n)
        info = np.zeros(2, dtype=np.uint64)
        lib().orc_tree_solve_reference(self._h, float(pw), int(cg_iters), float(acc), _ptr(x), _ptr(info))
        return x, info

    def coarse_rhs(self, pw):
        cd = self.depth - 2 if self.depth > 2 else 0
        out = np.zeros(8 ** cd)
        if lib().orc_tree_coarse_rhs(self._h, float(pw), _ptr(out)) != 0:
            raise RuntimeError("no coarse level")
        return out

    def prolongate(self, coarse_lex, coarse_depth):
        out = np.zeros(self.n)
        lib().orc_tree_prolongate(self._h, _ptr(_f64(coarse_lex)), int(coarse_depth), _ptr(out))
        return out

    def solve_converged(self, pw, tol=1e-12, maxit=100000, x0=None):
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        rr = C.c_double(0.0)
        it = lib().orc_tree_solve_converged(self._h, float(pw), float(tol), int(maxit), _ptr(x), C.byref(rr))
        return x, it, rr.value


    # ---- matrix-free fine operator (depths where the crate's CSR does not fit in host memory)
    def apply_mf(self, x, pw):
        """y = A x with the entries of assemble_system computed on the fly."""
        x = _f64(x)
        y = np.empty(self.n)
        lib().orc_tree_apply_mf(self._h, float(pw), _ptr(x), _ptr(y))
        return y

    def release_field(self):
        """Free the normal field and weights (rhs() needs them; the matrix-free solves do not)."""
        lib().orc_tree_release_field(self._h)

    def cg_mf(self, b, pw, iters, acc, x0=None):
        """The crate's solve_cg (src/solvers.rs:20-69) with the matrix-free operator.
        Returns (x, iterations, delta) with delta[k] = ||r||^2 after k iterations."""
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        delta = np.full(int(iters) + 1, np.nan)
        it = lib().orc_tree_cg_mf(self._h, float(pw), _ptr(_f64(b)), _ptr(x), int(iters), float(acc), _ptr(delta))
        return x, it, delta

    def solve_converged_mf(self, b, pw, tol=1e-12, maxit=100000, x0=None):
        """CG until ||b - A x|| <= tol ||b||, matrix-free, from x0 (default 0)."""
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        rr = C.c_double(0.0)
        it = lib().orc_tree_solve_converged_mf(self._h, float(pw), _ptr(_f64(b)), float(tol), int(maxit), _ptr(x),
                                               C.byref(rr))
        return x, it, rr.value


def evaluate(depth, sol, pts3):
    pts3 = _f64(pts3, (-1, 3))
    out = np.zeros(pts3.shape[0])
    lib().orc_evaluate_many(int(depth), _ptr(_f64(sol)), _ptr(pts3), 3, pts3.shape[0], _ptr(out))
    return out


def iso(depth, sol, unit6):
    unit6 = _f64(unit6, (-1, 6))
    return lib().orc_iso(int(depth), _ptr(_f64(sol)), _ptr(unit6), unit6.shape[0])


def _take_mesh(m):
    v = np.ctypeslib.as_array(m.verts, shape=(m.nv * 3,)).reshape(-1, 3).copy() if m.nv else np.zeros((0, 3))
    t = np.ctypeslib.as_array(m.tris, shape=(m.nt * 3,)).reshape(-1, 3).copy() if m.nt else np.zeros((0, 3), np.uint64)
    lib().orc_mesh_free(C.byref(m))
    return v, t


def extract_surface(depth, sol, iso_value):
    m = OrcMesh()
    lib().orc_extract_surface(int(depth), _ptr(_f64(sol)), float(iso_value), C.byref(m))
    return _take_mesh(m)


def reconstruct(pts6, depth=8, scale=1.1, cg_accuracy=1e-3, cg_iters=500, point_weight=0.0,
                solve_mode=0, target_rel_residual=1e-12, max_iters=200000, want_coeffs=False):
    """reconstructor::reconstruct restated.  solve_mode 0 = the crate's cascadic schedule,
    1 = the same fine system solved to ``target_rel_residual``."""
    pts6 = _f64(pts6, (-1, 6))
    p = OrcParams(depth, scale, cg_accuracy, cg_iters, point_weight, solve_mode,
                  target_rel_residual, max_iters)
    m, st = OrcMesh(), OrcStats()
    coeffs = np.zeros(8 ** depth) if want_coeffs else None
    lib().orc_reconstruct(_ptr(pts6), pts6.shape[0], C.byref(p), C.byref(m), C.byref(st), _ptr(coeffs))
    v, t = _take_mesh(m)
    stats = {f: getattr(st, f) for f, _ in OrcStats._fields_}
    return v, t, stats, coeffs


# ------------------------------------------------------------------ degree 2 (extension)
def deg2_constants():
    """1-D integrals of the quadratic B-spline at offsets -2..2: mass, stiffness, N2' N2."""
    m, s, g = np.zeros(5), np.zeros(5), np.zeros(5)
    lib().orc_deg2_constants(_ptr(m), _ptr(s), _ptr(g))
    return m, s, g


def evaluate2(depth, sol, pts3):
    pts3 = _f64(pts3, (-1, 3))
    sol = _f64(sol)
    return np.array([lib().orc_evaluate2(int(depth), _ptr(sol), *p) for p in pts3])


class Tree2:
    """Degree-2 system on unit-cube points (pw: screening weight)."""

    def __init__(self, depth, unit6, pw):
        self.depth = int(depth)
        self.unit = _f64(unit6, (-1, 6))
        self._h = lib().orc_tree2_new(self.depth, _ptr(self.unit), self.unit.shape[0], float(pw))
        self.n = 8 ** self.depth

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_tree2_free(self._h)
            self._h = None

    def normal_field(self):
        nf, w = np.zeros((self.n, 3)), np.zeros(self.n)
        lib().orc_tree2_normal_field(self._h, _ptr(nf), _ptr(w))
        return nf, w

    def rhs(self):
        b = np.zeros(self.n)
        lib().orc_tree2_rhs(self._h, _ptr(b))
        return b

    def apply(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        lib().orc_tree2_apply(self._h, _ptr(x), _ptr(y))
        return y

    def solve(self, tol=1e-12, maxit=100000):
        x, rr = np.zeros(self.n), C.c_double()
        it = lib().orc_tree2_solve(self._h, float(tol), int(maxit), _ptr(x), C.byref(rr))
        return x, it, rr.value

    def release_field(self):
        """Free the normal field and weights (rhs() needs them; apply() does not)."""
        lib().orc_tree2_release_field(self._h)


class _CG:
    """The crate's CG loop (src/solvers.rs:20-69) on a matrix-free oracle operator, one
    iteration per step() (the CPU baseline's unit of work); from x = 0 with right-hand side b."""

    def step(self):
        """One iteration; returns ||r||^2 after it."""
        return lib().orc_cg_step(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_cg_free(self._h)
            self._h = None


class CG2(_CG):
    def __init__(self, tree2, b):
        self.tree = tree2  # keeps the operator alive
        self._h = lib().orc_cg2_new(tree2._h, _ptr(_f64(b)))


class CG1(_CG):
    def __init__(self, tree, b, pw):
        self.tree = tree
        self._h = lib().orc_cg1_new(tree._h, float(pw), _ptr(_f64(b)))


def loss2(pts6, queries3, depth, point_weight=4.0, scale=1.1, tol=1e-13):
    """Degree-2 forward for finite differences: the unit-cube transform of the points, the
    degree-2 system solved by CG to `tol`, L = mean over the queries (model space, mapped with
    the same transform) of the degree-2 implicit function squared."""
    unit, m = to_unit(pts6, scale)
    x, _, _ = Tree2(depth, unit, point_weight).solve(tol=tol)
    mm = np.asarray(m).reshape(4, 4).T
    qu = np.asarray(queries3, dtype=np.float64) @ mm[:3, :3].T + mm[:3, 3]
    chi = evaluate2(depth, x, qu)
    return float(np.mean(chi ** 2))


def extract_surface2(depth, sol, iso_value):
    m = OrcMesh()
    lib().orc_extract_surface2(int(depth), _ptr(_f64(sol)), float(iso_value), C.byref(m))
    return _take_mesh(m)


def reconstruct2(pts6, depth, scale=1.1, point_weight=4.0, tol=1e-12, maxit=100000):
    """(vertices, triangles, iso, relres, coefficients) of the degree-2 pipeline."""
    pts6 = _f64(pts6, (-1, 6))
    m, iso, rr = OrcMesh(), C.c_double(), C.c_double()
    coeffs = np.zeros(8 ** depth)
    lib().orc_reconstruct2(_ptr(pts6), pts6.shape[0], int(depth), float(scale), float(point_weight), float(tol),
                           int(maxit), C.byref(m), C.byref(iso), C.byref(rr), _ptr(coeffs))
    v, t = _take_mesh(m)
    return v, t, iso.value, rr.value, coeffs


# ------------------------------------------------------------------ adjoint
def loss(pts6, queries3, depth, point_weight=4.0, scale=1.1, dl_dchi=None, tol=1e-13):
    """L = mean chi(q)^2 (or sum g_k chi(q_k) with g = dl_dchi) after a converged FP64 solve;
    the unit-cube transform follows the points' bbox (keep perturbations off its extremes)."""
    pts6 = _f64(pts6, (-1, 6))
    q = _f64(queries3, (-1, 3))
    g = None if dl_dchi is None else _f64(dl_dchi)
    return lib().orc_loss(_ptr(pts6), pts6.shape[0], int(depth), float(point_weight), float(scale), _ptr(q),
                          q.shape[0], _ptr(g), float(tol))


def loss_backward(pts6, queries3, depth, point_weight=4.0, scale=1.1, dl_dchi=None, tol=1e-13):
    """(chi, dL/dpositions, dL/dnormals, L) in model space, the transform held fixed."""
    pts6 = _f64(pts6, (-1, 6))
    q = _f64(queries3, (-1, 3))
    g = None if dl_dchi is None else _f64(dl_dchi)
    n, k = pts6.shape[0], q.shape[0]
    chi, dp, dn, L = np.zeros(k), np.zeros((n, 3)), np.zeros((n, 3)), C.c_double()
    rc = lib().orc_loss_backward(_ptr(pts6), n, int(depth), float(point_weight), float(scale), _ptr(q), k, _ptr(g),
                                 float(tol), _ptr(chi), _ptr(dp), _ptr(dn), C.byref(L))
    if rc != 0:
        raise ValueError("orc_loss_backward: empty input")
    return chi, dp, dn, L.value


# ------------------------------------------------------------------ generic CSR
def csr_cg(ptr, col, val, b, x0, maxit, acc):
    ptr = np.ascontiguousarray(ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    x = _f64(x0).copy()
    it = lib().orc_csr_cg(len(ptr) - 1, _ptr(ptr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(b)), _ptr(x),
                          int(maxit), float(acc))
    return x, it


def csr_spmv(ptr, col, val, x):
    ptr = np.ascontiguousarray(ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    y = np.zeros(len(ptr) - 1)
    lib().orc_csr_spmv(len(ptr) - 1, _ptr(ptr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(x)), _ptr(y))
    return y


def csr_gs_sweep(ptr, col, val, b, x):
    ptr = np.ascontiguousarray(ptr, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    x = _f64(x).copy()
    lib().orc_csr_gs_sweep(len(ptr) - 1, _ptr(ptr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(b)), _ptr(x))
    return x

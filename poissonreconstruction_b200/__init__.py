"""B200-native screened Poisson surface reconstruction.

Python mirror of the reference crate's public path (``poisson_recon::reconstructor``):

    reconstruct(points, params) -> (Mesh, ReconstructStats)       src/reconstructor.rs:25

``points`` is an (N, 6) float64 array of ``x y z nx ny nz`` rows (the crate's
``OrientedPoint``, src/fem_tree.rs:10).  Everything runs in ``libpoisson_recon_b200.so``
through its C ABI (include/poisson_recon.h); there is no CPU fallback: importing works
anywhere, but any computation raises if the library or a B200 is missing.
"""
import ctypes as C
import dataclasses
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpoisson_recon_b200.so")

PR_OK = 0
PR_ERR_INVALID_ARGUMENT = -1
PR_ERR_OUT_OF_MEMORY = -2
PR_ERR_CUDA = -3
PR_ERR_NOT_CONVERGED = -4
PR_ERR_NO_DEVICE = -5
PR_ERR_STATE = -6
PR_ERR_INTERNAL = -7

PR_SOLVE_CONVERGED = 0
PR_SOLVE_REFERENCE_SCHEDULE = 1
PR_PRECISION_MIXED = 0
PR_PRECISION_FP64 = 1
PR_BAND_FULL = 1


class PrParams(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("samples_per_node", C.c_double), ("scale", C.c_double),
                ("cg_accuracy", C.c_double), ("cg_iters", C.c_uint64), ("point_weight", C.c_double),
                ("verbose", C.c_int32), ("solve_mode", C.c_int32), ("precision", C.c_int32),
                ("target_rel_residual", C.c_double), ("max_iters", C.c_uint32), ("smooth_sweeps", C.c_uint32),
                ("inner_rel_tol", C.c_double), ("degree", C.c_uint32), ("coarse_depth", C.c_uint32),
                ("band_flags", C.c_uint32), ("reserved", C.c_uint32 * 5)]


class PrMesh(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_double)), ("n_vertices", C.c_uint64),
                ("triangles", C.POINTER(C.c_uint64)), ("n_triangles", C.c_uint64)]


class PrStats(C.Structure):
    _fields_ = [("time_transform", C.c_double), ("time_tree", C.c_double), ("time_system", C.c_double),
                ("time_solve", C.c_double), ("time_extract", C.c_double), ("time_total", C.c_double),
                ("fem_nodes", C.c_uint64), ("matrix_nnz", C.c_uint64), ("mesh_vertices", C.c_uint64),
                ("mesh_triangles", C.c_uint64), ("iso_value", C.c_double), ("rel_residual", C.c_double),
                ("pcg_iterations", C.c_uint32), ("refinement_steps", C.c_uint32), ("points_in_cube", C.c_uint64),
                ("solve_bytes", C.c_double), ("peak_device_bytes", C.c_double), ("converged", C.c_int32),
                ("reserved_i", C.c_int32), ("time_mesh_copy", C.c_double), ("reserved", C.c_double * 4)]


class PrAdjointStats(C.Structure):
    _fields_ = [("loss", C.c_double), ("rel_residual", C.c_double), ("pcg_iterations", C.c_uint32),
                ("refinement_steps", C.c_uint32), ("converged", C.c_int32), ("queries_off_band", C.c_int32),
                ("time_solve", C.c_double), ("time_total", C.c_double), ("reserved", C.c_double * 4)]


# Every C-ABI entry point and its signature (checked against include/poisson_recon.h by the tests).
_P = C.c_void_p
SIGNATURES = {
    "pr_version": (C.c_char_p, []),
    "pr_abi_layout": (None, [_P]),
    "pr_kernel_launches": (C.c_uint64, [C.POINTER(C.c_uint64)]),
    "pr_autotune_log": (C.c_char_p, []),
    "pr_ctx_apply_operator_device": (C.c_int, [_P, _P, _P, C.c_int]),
    "pr_iso_value_noalloc": (C.c_int, [C.c_uint32, _P, _P, C.c_uint64, _P, _P]),
    "pr_ctx_kernel_bench": (C.c_int, [_P, C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]),
    "pr_last_error": (C.c_char_p, []),
    "pr_params_default": (PrParams, []),
    "pr_reconstruct": (C.c_int, [_P, C.c_uint64, C.POINTER(PrParams), C.POINTER(PrMesh), C.POINTER(PrStats)]),
    "pr_mesh_free": (None, [C.POINTER(PrMesh)]),
    "pr_host_free": (None, [_P]),
    "pr_context_create": (C.c_int, [C.c_int, _P, C.POINTER(_P)]),
    "pr_context_destroy": (C.c_int, [_P]),
    "pr_ctx_reconstruct": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(PrParams), C.POINTER(PrMesh),
                                     C.POINTER(PrStats)]),
    "pr_ctx_reconstruct_device": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(PrParams), C.POINTER(PrStats)]),
    "pr_ctx_mesh_device": (C.c_int, [_P, C.POINTER(_P), C.POINTER(C.c_uint64), C.POINTER(_P),
                                     C.POINTER(C.c_uint64)]),
    "pr_ctx_mesh_copy": (C.c_int, [_P, C.POINTER(PrMesh)]),
    "pr_ctx_synchronize": (C.c_int, [_P]),
    "pr_ctx_info": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), _P]),
    "pr_ctx_get_coefficients": (C.c_int, [_P, _P]),
    "pr_ctx_get_rhs": (C.c_int, [_P, _P]),
    "pr_ctx_get_coarse_rhs": (C.c_int, [_P, C.POINTER(C.c_uint32), _P]),
    "pr_ctx_band_info": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), _P]),
    "pr_ctx_band_get": (C.c_int, [_P, C.c_int, _P]),
    "pr_ctx_band_apply": (C.c_int, [_P, _P, _P]),
    "pr_ctx_cg_reference": (C.c_int, [_P, _P, C.c_uint64, C.c_double, _P, _P, C.POINTER(C.c_uint64)]),
    "pr_ctx_get_unit_points": (C.c_int, [_P, _P]),
    "pr_ctx_get_normal_field": (C.c_int, [_P, _P, _P]),
    "pr_ctx_apply_operator": (C.c_int, [_P, _P, _P, C.c_int]),
    "pr_ctx_evaluate": (C.c_int, [_P, _P, _P, C.c_uint64, _P]),
    "pr_ctx_extract": (C.c_int, [_P, _P, C.c_double, C.POINTER(PrMesh)]),
    "pr_ctx_extract_at_depth": (C.c_int, [_P, C.c_uint32, _P, C.c_double, C.POINTER(PrMesh)]),
    "pr_ctx_reconstruct_batch": (C.c_int, [_P, C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P, _P]),
    "pr_reconstruct_batch": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, _P, _P, _P]),
    "pr_ply_read_points": (C.c_int, [C.c_char_p, C.POINTER(_P), C.POINTER(C.c_uint64)]),
    "pr_ply_write_mesh": (C.c_int, [C.c_char_p, C.POINTER(PrMesh), C.c_int]),
    "pr_ctx_solve": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(PrParams), C.POINTER(PrStats)]),
    "pr_ctx_loss_backward": (C.c_int, [_P, _P, C.c_uint64, _P, _P, _P, _P, C.POINTER(PrAdjointStats)]),
    "pr_loss_backward": (C.c_int, [_P, C.c_uint64, C.POINTER(PrParams), _P, C.c_uint64, _P, _P, _P, _P,
                                   C.POINTER(PrAdjointStats)]),
}

_LIB = None


class ReconstructError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (status %d)" % (msg, code))
        self.code = code


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("%s is missing: run `python -m poissonreconstruction_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _check(rc):
    if rc != PR_OK:
        raise ReconstructError(rc, lib().pr_last_error().decode())


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


@dataclasses.dataclass
class ReconstructParams:
    """src/reconstructor.rs:8-15 (defaults of ReconstructParams::default()) + extensions."""
    depth: int = 8
    samples_per_node: float = 1.5
    scale: float = 1.1
    cg_accuracy: float = 1e-3
    cg_iters: int = 500
    point_weight: float = 0.0
    verbose: bool = False
    solve_mode: int = PR_SOLVE_CONVERGED
    precision: int = PR_PRECISION_MIXED
    target_rel_residual: float = 1e-6
    max_iters: int = 200
    smooth_sweeps: int = 1
    inner_rel_tol: float = 1e-4
    degree: int = 1
    coarse_depth: int = 0
    band_flags: int = 0

    def to_c(self):
        p = PrParams()
        for f in dataclasses.fields(self):
            setattr(p, f.name, int(getattr(self, f.name)) if f.type in (int, bool, "int", "bool")
                    else getattr(self, f.name))
        return p


@dataclasses.dataclass
class Mesh:
    """src/marching_cubes.rs:8-11: (V,3) float64 vertices, (T,3) uint64 vertex indices."""
    vertices: np.ndarray
    triangles: np.ndarray


@dataclasses.dataclass
class ReconstructStats:
    time_transform: float = 0.0
    time_tree: float = 0.0
    time_system: float = 0.0
    time_solve: float = 0.0
    time_extract: float = 0.0
    time_total: float = 0.0
    fem_nodes: int = 0
    matrix_nnz: int = 0
    mesh_vertices: int = 0
    mesh_triangles: int = 0
    iso_value: float = 0.0
    rel_residual: float = 0.0
    pcg_iterations: int = 0
    refinement_steps: int = 0
    points_in_cube: int = 0
    solve_bytes: float = 0.0
    peak_device_bytes: float = 0.0
    converged: int = 0
    time_mesh_copy: float = 0.0

    @classmethod
    def from_c(cls, s):
        return cls(**{f.name: getattr(s, f.name) for f in dataclasses.fields(cls)})


def _owned_array(ptr, count, ctype, dtype):
    """numpy view of a library-allocated mesh array; pr_host_free releases it with the array."""
    if not count:
        return np.zeros((0, 3), dtype=dtype)
    base = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count * 3,))
    weakref.finalize(base, lib().pr_host_free, C.cast(ptr, C.c_void_p).value)
    return base.reshape(-1, 3)


def _take_mesh(m):
    """Take ownership of a pr_mesh's arrays without copying."""
    v = _owned_array(m.vertices, m.n_vertices, C.c_double, np.float64)
    t = _owned_array(m.triangles, m.n_triangles, C.c_uint64, np.uint64)
    m.vertices = None
    m.triangles = None
    m.n_vertices = m.n_triangles = 0
    return Mesh(v, t)


def _points(points):
    pts = np.ascontiguousarray(points, dtype=np.float64)
    if pts.ndim != 2 or pts.shape[1] != 6:
        raise ValueError("points must be an (N, 6) array of x y z nx ny nz")
    return pts


def reconstruct(points, params=None):
    """reconstructor::reconstruct (src/reconstructor.rs:25-70) on the GPU."""
    params = params or ReconstructParams()
    pts = _points(points)
    p, m, s = params.to_c(), PrMesh(), PrStats()
    _check(lib().pr_reconstruct(_ptr(pts), pts.shape[0], C.byref(p), C.byref(m), C.byref(s)))
    return _take_mesh(m), ReconstructStats.from_c(s)


PR_PLY_ASCII = 0
PR_PLY_BINARY = 1
CLI_PATH = os.path.join(_HERE, "poisson-recon")


def read_ply(path):
    """ply::read_oriented_points (src/ply.rs:13-70): an (N, 6) float64 array x y z nx ny nz."""
    p, n = C.c_void_p(), C.c_uint64()
    _check(lib().pr_ply_read_points(os.fsencode(path), C.byref(p), C.byref(n)))
    if n.value == 0:
        return np.zeros((0, 6))
    base = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n.value * 6,))
    out = base.reshape(-1, 6).copy()
    lib().pr_host_free(p)
    return out


def write_ply(path, mesh, binary=False):
    """ply::write_mesh (src/ply.rs:73-107); binary=True writes binary_little_endian."""
    v = np.ascontiguousarray(mesh.vertices, dtype=np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(mesh.triangles, dtype=np.uint64).reshape(-1, 3)
    m = PrMesh(v.ctypes.data_as(C.POINTER(C.c_double)), v.shape[0], t.ctypes.data_as(C.POINTER(C.c_uint64)),
               t.shape[0])
    _check(lib().pr_ply_write_mesh(os.fsencode(path), C.byref(m), PR_PLY_BINARY if binary else PR_PLY_ASCII))


def reconstruct_batch(clouds, params=None, concurrency=4):
    """Reconstruct independent clouds concurrently (no counterpart in the reference crate).

    clouds: sequence of (N_i, 6) arrays; params: one ReconstructParams for all clouds or a
    sequence with one per cloud.  Returns a list of (Mesh, ReconstructStats); raises on the
    lowest-numbered failed cloud."""
    pts = [_points(c) for c in clouds]
    count = len(pts)
    if params is None or isinstance(params, ReconstructParams):
        params = [params or ReconstructParams()] * count
    if len(params) != count:
        raise ValueError("one params entry per cloud")
    ptrs = (C.c_void_p * count)(*[p.ctypes.data for p in pts])
    ns = (C.c_uint64 * count)(*[p.shape[0] for p in pts])
    cps = (PrParams * count)(*[p.to_c() for p in params])
    meshes = (PrMesh * count)()
    stats = (PrStats * count)()
    status = (C.c_int * count)()
    rc = lib().pr_reconstruct_batch(ptrs, ns, count, cps, int(concurrency), meshes, stats, status)
    out = [(_take_mesh(meshes[i]), ReconstructStats.from_c(stats[i])) for i in range(count)]
    _check(rc)
    return out


@dataclasses.dataclass
class AdjointStats:
    loss: float = 0.0
    rel_residual: float = 0.0
    pcg_iterations: int = 0
    refinement_steps: int = 0
    converged: int = 0
    queries_off_band: int = 0
    time_solve: float = 0.0
    time_total: float = 0.0

    @classmethod
    def from_c(cls, s):
        return cls(**{f.name: getattr(s, f.name) for f in dataclasses.fields(cls)})


def _queries(queries, dl_dchi):
    q = np.ascontiguousarray(queries, dtype=np.float64)
    if q.ndim != 2 or q.shape[1] != 3:
        raise ValueError("queries must be a (K, 3) array")
    g = None
    if dl_dchi is not None:
        g = np.ascontiguousarray(dl_dchi, dtype=np.float64).reshape(-1)
        if g.shape[0] != q.shape[0]:
            raise ValueError("dl_dchi must have one entry per query")
    return q, g


def loss_backward(points, queries, params=None, dl_dchi=None):
    """Solve, then differentiate chi at model-space `queries` (no counterpart in the reference).
    Returns (chi, dL/dpositions, dL/dnormals, AdjointStats); with dl_dchi None, L = mean chi^2."""
    params = params or ReconstructParams()
    pts = _points(points)
    q, g = _queries(queries, dl_dchi)
    chi, dp, dn = np.zeros(q.shape[0]), np.zeros((pts.shape[0], 3)), np.zeros((pts.shape[0], 3))
    p, s = params.to_c(), PrAdjointStats()
    _check(lib().pr_loss_backward(_ptr(pts), pts.shape[0], C.byref(p), _ptr(q), q.shape[0], _ptr(g), _ptr(chi),
                                  _ptr(dp), _ptr(dn), C.byref(s)))
    return chi, dp, dn, AdjointStats.from_c(s)


class Context:
    """A device context: owns a CUDA stream (or uses the one given) and the buffers of the
    last reconstruction, whose intermediate state the accessors read."""

    def __init__(self, device=0, stream=None):
        h = C.c_void_p()
        _check(lib().pr_context_create(int(device), C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pr_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- reconstruction
    def reconstruct(self, points, params=None):
        params = params or ReconstructParams()
        pts = _points(points)
        p, m, s = params.to_c(), PrMesh(), PrStats()
        _check(lib().pr_ctx_reconstruct(self._h, _ptr(pts), pts.shape[0], C.byref(p), C.byref(m), C.byref(s)))
        self._n_points = pts.shape[0]
        return _take_mesh(m), ReconstructStats.from_c(s)

    def solve(self, points, params=None):
        """Transform, splat, RHS and solve without marching cubes (state kept for the adjoint)."""
        params = params or ReconstructParams()
        pts = _points(points)
        p, s = params.to_c(), PrStats()
        _check(lib().pr_ctx_solve(self._h, _ptr(pts), pts.shape[0], C.byref(p), C.byref(s)))
        self._n_points = pts.shape[0]
        return ReconstructStats.from_c(s)

    def loss_backward(self, queries, dl_dchi=None, n_points=None):
        """Gradients of the last solve w.r.t. its points: (chi, dL/dpositions, dL/dnormals, stats)."""
        q, g = _queries(queries, dl_dchi)
        n = n_points if n_points is not None else getattr(self, "_n_points", None)
        if n is None:
            raise ValueError("n_points unknown: pass the point count of the last solve")
        chi, dp, dn = np.zeros(q.shape[0]), np.zeros((n, 3)), np.zeros((n, 3))
        s = PrAdjointStats()
        _check(lib().pr_ctx_loss_backward(self._h, _ptr(q), q.shape[0], _ptr(g), _ptr(chi), _ptr(dp), _ptr(dn),
                                          C.byref(s)))
        return chi, dp, dn, AdjointStats.from_c(s)

    def reconstruct_device(self, d_points_ptr, n, params=None):
        """Input already on the device (pointer to n x 6 float64); the mesh stays there."""
        params = params or ReconstructParams()
        p, s = params.to_c(), PrStats()
        _check(lib().pr_ctx_reconstruct_device(self._h, C.c_void_p(d_points_ptr), int(n), C.byref(p), C.byref(s)))
        return ReconstructStats.from_c(s)

    def mesh_device(self):
        dv, dt = C.c_void_p(), C.c_void_p()
        nv, nt = C.c_uint64(), C.c_uint64()
        _check(lib().pr_ctx_mesh_device(self._h, C.byref(dv), C.byref(nv), C.byref(dt), C.byref(nt)))
        return dv.value, nv.value, dt.value, nt.value

    def mesh(self):
        m = PrMesh()
        _check(lib().pr_ctx_mesh_copy(self._h, C.byref(m)))
        return _take_mesh(m)

    def synchronize(self):
        _check(lib().pr_ctx_synchronize(self._h))

    # -- accessors
    def info(self):
        d, n = C.c_uint32(), C.c_uint64()
        m = np.zeros(16)
        _check(lib().pr_ctx_info(self._h, C.byref(d), C.byref(n), _ptr(m)))
        return d.value, n.value, m

    def coefficients(self):
        _, n, _ = self.info()
        out = np.zeros(n)
        _check(lib().pr_ctx_get_coefficients(self._h, _ptr(out)))
        return out

    def rhs(self):
        _, n, _ = self.info()
        out = np.zeros(n)
        _check(lib().pr_ctx_get_rhs(self._h, _ptr(out)))
        return out

    def coarse_rhs(self):
        """Reference schedule: (coarse depth, right-hand side of its coarse system, Morton order)."""
        d = C.c_uint32()
        _check(lib().pr_ctx_get_coarse_rhs(self._h, C.byref(d), None))
        out = np.zeros(8 ** d.value)
        _check(lib().pr_ctx_get_coarse_rhs(self._h, C.byref(d), _ptr(out)))
        return d.value, out

    # ---- adaptive (coarse_depth > 0) state
    def band_info(self):
        """(depth, coarse depth, brick Morton codes (uint32, the band's brick order))."""
        d, dc, nb = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(lib().pr_ctx_band_info(self._h, C.byref(d), C.byref(dc), C.byref(nb), None))
        codes = np.zeros(nb.value, dtype=np.uint32)
        _check(lib().pr_ctx_band_info(self._h, C.byref(d), C.byref(dc), C.byref(nb), _ptr(codes)))
        return d.value, dc.value, codes

    def band_vector(self, which):
        """0: right-hand side, 1: solved coefficients, 2: prolonged coarse solution (512 per brick)."""
        _, _, codes = self.band_info()
        out = np.zeros(512 * len(codes))
        _check(lib().pr_ctx_band_get(self._h, int(which), _ptr(out)))
        return out

    def band_apply(self, x):
        """A_BB x on the band (FP64)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        _check(lib().pr_ctx_band_apply(self._h, _ptr(x), _ptr(y)))
        return y

    def cg_reference(self, iters, accuracy, x0=None):
        """The crate's CG loop on the last degree-1 fine system (FP64, on the device):
        returns (x, iterations, delta) with delta[k] = ||r||^2 after k iterations."""
        _, n, _ = self.info()
        x = np.zeros(n)
        delta = np.full(int(iters) + 1, np.nan)
        it = C.c_uint64()
        x0 = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        _check(lib().pr_ctx_cg_reference(self._h, _ptr(x0) if x0 is not None else None, int(iters), float(accuracy),
                                         _ptr(x), _ptr(delta), C.byref(it)))
        return x, it.value, delta

    def unit_points(self, n_points):
        out = np.zeros((n_points, 6))
        _check(lib().pr_ctx_get_unit_points(self._h, _ptr(out)))
        return out

    def normal_field(self):
        _, n, _ = self.info()
        nf, w = np.zeros((n, 3)), np.zeros(n)
        _check(lib().pr_ctx_get_normal_field(self._h, _ptr(nf), _ptr(w)))
        return nf, w

    def apply_operator(self, x, precision=PR_PRECISION_FP64):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        _check(lib().pr_ctx_apply_operator(self._h, _ptr(x), _ptr(y), int(precision)))
        return y

    def apply_operator_device(self, d_x, d_y, precision=PR_PRECISION_MIXED):
        """Enqueue y = A x on device pointers (no synchronisation)."""
        _check(lib().pr_ctx_apply_operator_device(self._h, C.c_void_p(d_x), C.c_void_p(d_y), int(precision)))

    KERNELS = {"spmv": 0, "spmv_xpby": 1, "smooth_first": 2, "smooth": 3, "smooth_prolong_dot": 4,
               "resid_restrict": 5, "stencil_per_node": 6, "smooth_prolong_dot_coarse": 7,
               "resid_restrict_coarse": 8, "cg_update_presmooth": 9,
               # degree 2 (finest level of the given depth)
               "d2_cheb": 20, "d2_cheb_regs": 21, "d2_apply": 22, "d2_apply_regs": 23, "d2_resid": 24,
               "d2_restrict": 25, "d2_prolong": 26, "d2_cheb_first": 27, "d2_cheb_f": 28, "d2_cheb_pf": 29,
               "d2_cg_dir": 30, "d2_refine": 31}

    def kernel_bench(self, kernel, depth, precision=PR_PRECISION_MIXED, reps=10):
        """(ms per launch, algorithmic bytes per launch) of one solver kernel."""
        ms, by = C.c_double(), C.c_double()
        _check(lib().pr_ctx_kernel_bench(self._h, self.KERNELS[kernel], int(depth), int(precision), int(reps),
                                         C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def evaluate(self, pts3, coefficients=None):
        pts3 = np.ascontiguousarray(pts3, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(pts3.shape[0])
        co = None if coefficients is None else np.ascontiguousarray(coefficients, dtype=np.float64)
        _check(lib().pr_ctx_evaluate(self._h, _ptr(co), _ptr(pts3), pts3.shape[0], _ptr(out)))
        return out

    def extract(self, coefficients, iso, depth=None):
        """Marching cubes of given FP64 coefficients; vertices in unit-cube space."""
        co = np.ascontiguousarray(coefficients, dtype=np.float64)
        m = PrMesh()
        if depth is None:
            _check(lib().pr_ctx_extract(self._h, _ptr(co), float(iso), C.byref(m)))
        else:
            _check(lib().pr_ctx_extract_at_depth(self._h, int(depth), _ptr(co), float(iso), C.byref(m)))
        return _take_mesh(m)


def band_natural_index(codes, depth):
    """Natural grid index (x + res (y + res z)) of every band entry (bricks in `codes` order, 512
    nodes per brick, x fastest inside a brick)."""
    codes = np.asarray(codes, dtype=np.uint64)

    def compact(v):
        v = v & np.uint64(0x09249249)
        v = (v | (v >> np.uint64(2))) & np.uint64(0x030C30C3)
        v = (v | (v >> np.uint64(4))) & np.uint64(0x0300F00F)
        v = (v | (v >> np.uint64(8))) & np.uint64(0x030000FF)
        v = (v | (v >> np.uint64(16))) & np.uint64(0x000003FF)
        return v.astype(np.int64)

    bx, by, bz = compact(codes), compact(codes >> np.uint64(1)), compact(codes >> np.uint64(2))
    loc = np.arange(512)
    lx, ly, lz = loc & 7, (loc >> 3) & 7, loc >> 6
    res = 1 << depth
    gx = (8 * bx[:, None] + lx[None, :]).ravel()
    gy = (8 * by[:, None] + ly[None, :]).ravel()
    gz = (8 * bz[:, None] + lz[None, :]).ravel()
    return gx + res * (gy + res * gz)


def kernel_launches():
    """(own kernel launches, library primitive calls) so far in this process."""
    prim = C.c_uint64()
    n = lib().pr_kernel_launches(C.byref(prim))
    return n, prim.value


__all__ = ["ReconstructParams", "ReconstructStats", "Mesh", "reconstruct", "Context", "ReconstructError", "lib"]


def autotune_log():
    """The z-segment choices of the degree-1 block kernels made so far in this process."""
    return lib().pr_autotune_log().decode()

"""C ABI checks that need no GPU: the library loads, exports every function that
include/poisson_recon.h declares, its struct layouts match the ctypes mirror, and argument
validation / empty input behave like the crate (src/reconstructor.rs:28) before any device
work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import poissonreconstruction_b200 as prb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "poisson_recon.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pr_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    if not os.path.exists(prb.LIB_PATH):
        pytest.skip("library not built (python -m poissonreconstruction_b200.build)")
    return prb.lib()


def test_exports_every_declared_symbol(L):
    funcs = header_functions()
    assert len(funcs) >= 20
    for f in funcs:
        assert hasattr(L, f), f
    assert set(funcs) == set(prb.SIGNATURES), set(funcs) ^ set(prb.SIGNATURES)


def test_struct_layouts(L):
    out = (C.c_uint64 * 4)()
    L.pr_abi_layout(out)
    assert out[0] == C.sizeof(prb.PrParams)
    assert out[1] == C.sizeof(prb.PrMesh)
    assert out[2] == C.sizeof(prb.PrStats)
    assert out[3] == 48


def test_params_default_mirrors_crate(L):
    p = L.pr_params_default()
    # ReconstructParams::default(), src/reconstructor.rs:14
    assert (p.depth, p.samples_per_node, p.scale, p.cg_accuracy, p.cg_iters, p.point_weight, p.verbose) == \
        (8, 1.5, 1.1, 1e-3, 500, 0.0, 0)
    assert p.solve_mode == prb.PR_SOLVE_CONVERGED and p.precision == prb.PR_PRECISION_MIXED
    assert p.target_rel_residual == 1e-6
    py = prb.ReconstructParams()
    assert (py.depth, py.scale, py.cg_accuracy, py.cg_iters, py.point_weight) == (8, 1.1, 1e-3, 500, 0.0)


def test_empty_input_returns_empty_mesh(L):
    mesh, st = prb.reconstruct(np.zeros((0, 6)), prb.ReconstructParams(depth=6))
    assert mesh.vertices.shape == (0, 3) and mesh.triangles.shape == (0, 3)
    assert st.fem_nodes == 0 and st.iso_value == 0.0


@pytest.mark.parametrize("kw,msg", [
    (dict(depth=0), "depth"), (dict(depth=11), "depth"), (dict(scale=0.0), "scale"),
    (dict(point_weight=-1.0), "point_weight"), (dict(solve_mode=7), "solve_mode"),
    (dict(precision=3), "precision"), (dict(target_rel_residual=float("nan")), "target_rel_residual"),
    # adaptive reconstruction: degree 2 only, depth <= 12, at most 4 levels above the coarse one
    (dict(depth=6, coarse_depth=3), "degree 2"), (dict(depth=13, coarse_depth=10, degree=2), "depth"),
    (dict(depth=12, coarse_depth=7, degree=2), "coarse_depth"),
    (dict(depth=8, coarse_depth=5, degree=2, solve_mode=1), "PR_SOLVE_CONVERGED"),
])
def test_invalid_params_rejected(L, kw, msg):
    pts = np.zeros((4, 6))
    with pytest.raises(prb.ReconstructError) as e:
        prb.reconstruct(pts, prb.ReconstructParams(**kw))
    assert e.value.code == prb.PR_ERR_INVALID_ARGUMENT and msg in str(e.value)


def test_null_arguments(L):
    p = L.pr_params_default()
    assert L.pr_reconstruct(None, 5, C.byref(p), C.byref(prb.PrMesh()), None) == prb.PR_ERR_INVALID_ARGUMENT
    assert L.pr_reconstruct(None, 0, None, C.byref(prb.PrMesh()), None) == prb.PR_ERR_INVALID_ARGUMENT
    assert L.pr_context_create(0, None, None) == prb.PR_ERR_INVALID_ARGUMENT
    assert L.pr_ctx_get_rhs(None, None) == prb.PR_ERR_INVALID_ARGUMENT
    L.pr_mesh_free(None)  # no-op


def test_no_device_is_an_error_not_a_fallback(L):
    from tests.conftest import _has_gpu
    if _has_gpu():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert L.pr_context_create(0, None, C.byref(h)) == prb.PR_ERR_NO_DEVICE
    with pytest.raises(prb.ReconstructError) as e:
        prb.reconstruct(np.random.default_rng(0).standard_normal((10, 6)), prb.ReconstructParams(depth=3))
    assert e.value.code == prb.PR_ERR_NO_DEVICE

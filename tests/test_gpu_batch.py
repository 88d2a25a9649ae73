"""Batched reconstruction (pr_reconstruct_batch / pr_ctx_reconstruct_batch) on the GPU: every
cloud's mesh equals the one a single-cloud call produces (the pipeline is deterministic), and
a bad cloud fails alone."""
import ctypes as C

import numpy as np
import pytest

import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

pytestmark = pytest.mark.gpu


def _small_batch(count=10, seed=77):
    rng = np.random.default_rng(seed)
    clouds, params = [], []
    for i in range(count):
        n = int(rng.integers(5_000, 60_000))
        if i % 2:
            pts = synthetic.ellipsoid(n, 1000 + i, radii=tuple(rng.uniform(0.3, 1.0, 3)), noise=0.001, fp32=True)
        else:
            pts = synthetic.torus(n, 1000 + i, R=0.9, r=0.3, noise=0.001, normal_sigma=0.0, fp32=True)
        clouds.append(pts)
        params.append(prb.ReconstructParams(depth=int(rng.integers(5, 8)), point_weight=4.0))
    return clouds, params


def test_batch_matches_single_calls(ctx):
    clouds, params = _small_batch()
    out = prb.reconstruct_batch(clouds, params, concurrency=3)
    assert len(out) == len(clouds)
    for pts, p, (mesh, st) in zip(clouds, params, out):
        m1, st1 = ctx.reconstruct(pts, p)
        assert st.fem_nodes == 8 ** p.depth and st.converged == 1
        assert np.array_equal(mesh.triangles, m1.triangles)
        assert np.array_equal(mesh.vertices, m1.vertices)
        assert st.iso_value == st1.iso_value


def test_batch_reports_the_failed_cloud():
    clouds, params = _small_batch(count=4, seed=5)
    params[2] = prb.ReconstructParams(depth=11, point_weight=4.0)  # outside [1, 10]
    count = len(clouds)
    ptrs = (C.c_void_p * count)(*[c.ctypes.data for c in clouds])
    ns = (C.c_uint64 * count)(*[c.shape[0] for c in clouds])
    cps = (prb.PrParams * count)(*[p.to_c() for p in params])
    meshes, stats, status = (prb.PrMesh * count)(), (prb.PrStats * count)(), (C.c_int * count)()
    rc = prb.lib().pr_reconstruct_batch(ptrs, ns, count, cps, 2, meshes, stats, status)
    assert rc == prb.PR_ERR_INVALID_ARGUMENT
    assert list(status) == [0, 0, prb.PR_ERR_INVALID_ARGUMENT, 0]
    assert b"cloud 2" in prb.lib().pr_last_error()
    for i in (0, 1, 3):
        assert meshes[i].n_triangles > 0
        prb.lib().pr_mesh_free(C.byref(meshes[i]))
    assert meshes[2].n_triangles == 0


def test_batch_empty_and_zero_point_clouds():
    assert prb.reconstruct_batch([]) == []
    out = prb.reconstruct_batch([np.zeros((0, 6)), synthetic.sphere(3000, seed=2)],
                                prb.ReconstructParams(depth=5, point_weight=4.0))
    assert out[0][0].triangles.shape == (0, 3) and out[1][0].triangles.shape[0] > 0


def _mixed_shapes(seed=91):
    """Clouds of depth 5 and 6 whose solves stop after different numbers of iterations: clean and
    noisy surfaces, a few hundred points and tens of thousands."""
    rng = np.random.default_rng(seed)
    clouds, depths = [], []
    for i in range(9):
        n = [300, 2_000, 40_000][i % 3]
        kind = (i // 3) % 3
        if kind == 0:
            pts = synthetic.sphere(n, seed=500 + i)
        elif kind == 1:
            pts = synthetic.torus(n, 600 + i, R=0.8, r=0.25, noise=0.01, normal_sigma=0.3, fp32=True)
        else:
            pts = synthetic.ellipsoid(n, 700 + i, radii=tuple(rng.uniform(0.3, 1.0, 3)), noise=0.02, fp32=True)
        clouds.append(pts)
        depths.append(5 + (i % 2))
    return clouds, depths


@pytest.mark.parametrize("precision", [prb.PR_PRECISION_MIXED, prb.PR_PRECISION_FP64])
def test_packed_solve_matches_single_calls(ctx, precision, monkeypatch, capsys):
    """Clouds of one depth are solved together (one launch per solver step for all of them); packs
    of at most 3 clouds here, so a depth group spans several packs.  Every cloud's coefficients,
    iteration counts, residual and mesh equal a single-cloud call's, also for clouds that stop
    before the others of their pack."""
    monkeypatch.setenv("PR_PACK_MAX_CLOUDS", "3")
    clouds, depths = _mixed_shapes()
    params = [prb.ReconstructParams(depth=d, point_weight=4.0, precision=precision) for d in depths]
    out = prb.reconstruct_batch(clouds, params, concurrency=2)
    iters = {}
    for pts, p, (mesh, st) in zip(clouds, params, out):
        m1, st1 = ctx.reconstruct(pts, p)
        assert st.converged == 1
        assert (st.pcg_iterations, st.refinement_steps) == (st1.pcg_iterations, st1.refinement_steps)
        assert st.rel_residual == st1.rel_residual
        assert st.iso_value == st1.iso_value
        assert np.array_equal(mesh.triangles, m1.triangles)
        assert np.array_equal(mesh.vertices, m1.vertices)
        iters.setdefault(p.depth, []).append((st.pcg_iterations, st.refinement_steps))
    with capsys.disabled():
        print("\npacked batch (%s): iterations per depth %s" % ("FP64" if precision else "mixed", iters))

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

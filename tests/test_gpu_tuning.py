"""The z-segment autotuner of the degree-1 block kernels (SpMV, residual + restriction,
smoother): 2, 4 or 8 z planes per thread compute the same values, so a forced choice, another
forced choice and the tuned one give the same solve and mesh bit for bit, and the tuner logs
what it chose."""
import numpy as np
import pytest

import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [prb.PR_PRECISION_MIXED, prb.PR_PRECISION_FP64])
def test_every_z_segment_gives_the_same_solve(precision, monkeypatch, capsys):
    pts = synthetic.torus(200_000, seed=31)
    p = prb.ReconstructParams(depth=8, point_weight=4.0, precision=precision)
    runs = {}
    with prb.Context(0) as ctx:
        for zt in ("2", "4", "8"):
            monkeypatch.setenv("PR_ZT", zt)
            mesh, st = ctx.reconstruct(pts, p)
            runs[zt] = (ctx.coefficients(), mesh, st)
        monkeypatch.delenv("PR_ZT")
        mesh, st = ctx.reconstruct(pts, p)
        runs["tuned"] = (ctx.coefficients(), mesh, st)
    x0, m0, s0 = runs["4"]
    for k, (x, m, s) in runs.items():
        assert np.array_equal(x, x0), k
        assert np.array_equal(m.triangles, m0.triangles) and np.array_equal(m.vertices, m0.vertices), k
        assert (s.pcg_iterations, s.rel_residual, s.iso_value) == (s0.pcg_iterations, s0.rel_residual, s0.iso_value)
    log = prb.autotune_log()
    if precision == prb.PR_PRECISION_MIXED:
        for fam in ("spmv16", "resid16", "smooth16"):
            assert fam in log
    with capsys.disabled():
        print("\nautotuner choices so far:\n" + log)

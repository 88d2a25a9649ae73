"""pr_iso_value_noalloc: the iso value computed without any device allocation.

Some callers cannot allocate device memory — a host whose caching allocator already holds
the free memory, or a latency-bound loop that must avoid the synchronisation cudaMalloc
implies.  This entry point takes every input and its output as device pointers and keeps
its partial sums in a fixed device array.  The test calls it twice in a row through the C
ABI on the coefficients and points of a degree-1 reconstruction (the only basis it evaluates),
and requires both results to equal, bit for bit, the iso value that pr_ctx_reconstruct computed
for them (the library's own allocating path: same per-point arithmetic, same fixed block grid,
same compensated sums).
This file is collected last, so that a run stopping at the first failure has run every
other test first.
"""
import ctypes as C

import numpy as np
import pytest

import poissonreconstruction_b200 as prb
from poissonreconstruction_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_iso_value_noalloc_matches_reconstruct_twice():
    import torch

    pts = synthetic.torus(30000, seed=31)
    depth = 6
    with prb.Context(0) as ctx:
        _, st = ctx.reconstruct(pts, prb.ReconstructParams(depth=depth, point_weight=4.0))
        coeffs = ctx.coefficients()
        unit = ctx.unit_points(len(pts))
    dev = torch.device("cuda", 0)
    d_x = torch.from_numpy(coeffs).to(dev)
    d_p = torch.from_numpy(np.ascontiguousarray(unit[:, :3])).to(dev)
    d_out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream or None)
    L = prb.lib()
    for k in range(2):  # two calls in a row share the scratch array
        rc = L.pr_iso_value_noalloc(depth, C.c_void_p(d_x.data_ptr()), C.c_void_p(d_p.data_ptr()), len(pts),
                                    C.c_void_p(d_out.data_ptr() + 8 * k), stream)
        assert rc == prb.PR_OK, L.pr_last_error().decode()
    torch.cuda.synchronize(dev)
    got = d_out.cpu().numpy()
    for v in got:
        assert v == st.iso_value, (v, st.iso_value)


def test_iso_value_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    dev = torch.device("cuda", 0)
    d = torch.zeros(8, dtype=torch.float64, device=dev)
    L = prb.lib()
    p = C.c_void_p(d.data_ptr())
    assert L.pr_iso_value_noalloc(1, p, p, (1 << 28) + 1, p, None) == prb.PR_ERR_INVALID_ARGUMENT
    assert "2^28" in L.pr_last_error().decode()
    assert L.pr_iso_value_noalloc(11, p, p, 1, p, None) == prb.PR_ERR_INVALID_ARGUMENT

"""fmma_exact_noalloc_d, the exact sum whose partial sums live in a 16 MiB
static device array, against the exact solver of fmma_solve_d.

This file is collected last so that the GPU cases run both in a fresh
process (this file alone) and after every other test in the same process.
Each case makes two calls in a row into two outputs: both must match the
existing entry point within 1e-12 (rel. L2; only the summation order
differs), agree bit for bit with each other (the chunks are added in a fixed
order), and the second call must leave the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

LIMIT = 262144  # n_tgt * nrhs, 16 MiB of doubles split at least 8 ways

CASES = [
    # dim, kernel, p0, n_tgt, n_src, nrhs (0 = unit weights)
    (3, "inv_r_safe", 0.0, 1000, 300_000, 2),
    (2, "gaussian", 0.01, 4096, 100_000, 1),
    (1, "inv_diff", 0.0, 777, 50_001, 3),
    (3, "multiquadric", 1e-4, 65536, 20_000, 4),  # n_tgt * nrhs at the limit
    (2, "log_r", 0.0, 5, 1000, 0),
    (3, "sum2_over_r2", 0.0, 300, 257, 1),
]


def _noalloc(L, dim, kid, p0, t, s, w, out, stream):
    nrhs = 1 if w is None else (1 if w.ndim == 1 else int(w.shape[0]))
    return L.fmma_exact_noalloc_d(dim, kid, p0, int(t.shape[0]), C.c_void_p(t.data_ptr()), int(s.shape[0]),
                                  C.c_void_p(s.data_ptr()), nrhs, None if w is None else C.c_void_p(w.data_ptr()),
                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("dim,kernel,p0,nt,ns,nrhs", CASES)
def test_noalloc_matches_exact_twice(ctx, dim, kernel, p0, nt, ns, nrhs):
    import torch

    import fmma_b200
    from fmma_b200 import _lib
    L = _lib.load()
    r = np.random.default_rng(nt + ns)
    t = torch.tensor(r.random((nt, dim)), dtype=torch.float64, device="cuda")
    s = torch.tensor(r.random((ns, dim)), dtype=torch.float64, device="cuda")
    if nrhs == 0:
        w = None
        shape = (nt,)
    else:
        w = torch.tensor(r.standard_normal((nrhs, ns)), dtype=torch.float64, device="cuda")
        shape = (nrhs, nt)
    ctx.set_kernel(kernel, p0)
    want, _ = ctx.solve(t, s, w, solver="exact")
    torch.cuda.synchronize()
    kid = fmma_b200.KERNELS[kernel]
    out1 = torch.full(shape, np.nan, dtype=torch.float64, device="cuda")
    out2 = torch.full(shape, np.nan, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_noalloc(L, dim, kid, p0, t, s, w, out1, stream))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _lib.check(_noalloc(L, dim, kid, p0, t, s, w, out2, stream))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    W = want.cpu().numpy()
    for got in (out1, out2):
        g = got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert rel_l2(g, W) <= 1e-12, rel_l2(g, W)
    assert torch.equal(out1, out2)


@pytest.mark.gpu
def test_noalloc_no_sources_clears_ans():
    import torch

    import fmma_b200
    from fmma_b200 import _lib
    L = _lib.load()
    t = torch.rand((100, 3), dtype=torch.float64, device="cuda")
    s = torch.empty((0, 3), dtype=torch.float64, device="cuda")
    out = torch.full((100,), 7.0, dtype=torch.float64, device="cuda")
    _lib.check(L.fmma_exact_noalloc_d(3, fmma_b200.KERNELS["inv_r"], 0.0, 100, C.c_void_p(t.data_ptr()), 0, None, 1,
                                      None, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0


@pytest.mark.parametrize("nt,nrhs", [(LIMIT + 1, 1), (LIMIT // 2 + 1, 2), (1 << 62, 64)])
def test_noalloc_rejects_sizes_beyond_the_scratch(nt, nrhs):
    """Rejected before any device work, so this also runs without a GPU."""
    from fmma_b200 import _lib
    L = _lib.load()
    buf = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = L.fmma_exact_noalloc_d(3, 0, 0.0, nt, buf, 10, buf, nrhs, None, buf, None)
    assert st == _lib.ERR_INVALID_ARG
    msg = L.fmma_last_error().decode()
    assert "fmma_exact_noalloc_d" in msg and str(LIMIT) in msg and "16 MiB" in msg

"""Failure paths, made on the host: a device allocator that refuses a request
turns the solve into FMMA_ERR_OOM (status 3) and leaves the context usable;
the same allocator hook serves the context from PyTorch's caching allocator.
No GPU fault is involved: the refusal happens in host code."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed=1, n=20000):
    r = np.random.default_rng(seed)
    return r.random((n, 3)), r.random((n, 3)), r.uniform(-1, 1, n)


def test_refused_allocation_is_oom_and_context_recovers():
    import fmma_b200
    t, s, w = _case()
    ctx = fmma_b200.Context(0)
    try:
        ctx.set_kernel("inv_r_safe")
        ref, _ = ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        asked = []
        ctx.set_allocator(lambda n, stream: asked.append(n) or 0, lambda p, n, stream: None)
        with pytest.raises(fmma_b200.FmmaError) as e:
            ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        assert e.value.status == 3 and asked, (e.value.status, asked)
        assert "fail" in str(e.value)
        ctx.set_allocator()  # back to cudaMalloc
        out, _ = ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        assert np.array_equal(out, ref)
    finally:
        ctx.close()


def test_misaligned_allocation_is_refused():
    """An allocator block that is not 256-byte aligned (a torch block offset
    by 16 bytes) is given back through the free callback and the solve fails
    with FMMA_ERR_INVALID_ARG before any kernel reads it; with an aligned
    allocator again the same context solves bit-identically."""
    import torch

    import fmma_b200
    t, s, w = _case()
    ctx = fmma_b200.Context(0)
    live = {}

    def alloc(n, stream):
        p = torch.cuda.caching_allocator_alloc(n + 256, 0, stream)
        live[p + 16] = p
        return p + 16

    def free(p, n, stream):
        torch.cuda.caching_allocator_delete(live.pop(p))

    try:
        ctx.set_kernel("inv_r_safe")
        ref, _ = ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        ctx.set_allocator(alloc, free)
        with pytest.raises(fmma_b200.FmmaError) as e:
            ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        assert e.value.status == 1 and "aligned" in str(e.value), (e.value.status, str(e.value))
        assert not live  # every block went back
        ctx.set_allocator()
        out, _ = ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
        assert np.array_equal(out, ref)
    finally:
        ctx.close()


def test_allocation_budget_exhausted_mid_solve():
    """A pool with a byte budget serves the first requests, then refuses: the
    failure comes in the middle of a solve, after kernels have run.  Raising
    the budget, the same context solves correctly."""
    import torch

    import fmma_b200
    t, s, w = _case(2)
    ctx = fmma_b200.Context(0)
    live = {}
    budget = [0]

    def alloc(n, stream):
        if sum(live.values()) + n > budget[0]:
            return 0
        p = torch.cuda.caching_allocator_alloc(n, 0, stream)
        live[p] = n
        return p

    def free(p, n, stream):
        live.pop(p, None)
        torch.cuda.caching_allocator_delete(p)

    try:
        ctx.set_kernel("inv_r_safe")
        ref, _ = ctx.solve(t, s, w, poly_ord=4, depth=5)
        budget[0] = 4 << 20  # enough for the first buffers, not for a solve
        ctx.set_allocator(alloc, free)
        with pytest.raises(fmma_b200.FmmaError) as e:
            ctx.solve(t, s, w, poly_ord=4, depth=5)
        assert e.value.status == 3
        budget[0] = 8 << 30
        out, _ = ctx.solve(t, s, w, poly_ord=4, depth=5)
        assert np.array_equal(out, ref)
        assert live
    finally:
        ctx.close()
    assert not live  # every buffer went back through free


def test_torch_allocator_results_identical():
    import torch

    import fmma_b200
    t, s, w = _case(3, 30000)
    a = fmma_b200.Context(0)
    b = fmma_b200.Context(0)
    try:
        for c in (a, b):
            c.set_kernel("log_r")
        before = torch.cuda.memory_allocated(0)
        b.use_torch_allocator()
        ra, _ = a.solve(t[:, :2].copy(), s[:, :2].copy(), w, poly_ord=5, depth=6, precision="tf32x3")
        rb, _ = b.solve(t[:, :2].copy(), s[:, :2].copy(), w, poly_ord=5, depth=6, precision="tf32x3")
        assert np.array_equal(ra, rb)
        assert torch.cuda.memory_allocated(0) > before  # b's scratch lives in torch's pool
    finally:
        a.close()
        b.close()
    assert torch.cuda.memory_allocated(0) == before


def test_m2l_wait_timeout_reports_and_context_recovers():
    """The tensor-core M2L's MMA issuer waits for a flag that nothing sets,
    bounded at 2e6 SM clocks (~1 ms): the wait gives up, every role of the
    kernel stops at its next wait and drains (gathers and operator copies
    landed, the drain commit of the issuer's MMAs waited for, TMEM freed), and
    the solve returns FMMA_ERR_TIMEOUT (status 5).  With the hook off, the same
    context then solves correctly."""
    import fmma_b200
    t, s, w = _case(4, 30000)
    ctx = fmma_b200.Context(0)
    try:
        ctx.set_kernel("inv_r_safe")
        ref, _ = ctx.solve(t, s, w, poly_ord=5, depth=5, precision="bf16x3")
        ctx.debug_m2l_wait(2_000_000, hold_issuer=True)
        with pytest.raises(fmma_b200.FmmaError) as e:
            ctx.solve(t, s, w, poly_ord=5, depth=5, precision="bf16x3")
        assert e.value.status == 5, e.value
        ctx.debug_m2l_wait()  # defaults
        out, _ = ctx.solve(t, s, w, poly_ord=5, depth=5, precision="bf16x3")
        assert np.array_equal(out, ref)
        # a shorter bound that nothing runs into: the solve is unaffected
        ctx.debug_m2l_wait(200_000_000)
        out2, _ = ctx.solve(t, s, w, poly_ord=5, depth=5, precision="bf16x3")
        assert np.array_equal(out2, ref)
    finally:
        ctx.debug_m2l_wait()
        ctx.close()

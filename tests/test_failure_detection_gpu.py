"""Failure detection without a GPU fault: a kernel waits on a device flag
that nothing sets, gives up after a short clock budget and records
GC_ERR_TIMEOUT in the context's status word -- the path a bounded TMA wait
takes when a tile never arrives.  The host reads it at gc_synchronize, the
status clears, and the context keeps working (bit-exact results after)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(gc, oracle):
    import torch
    ctx = gc.Context(0, torch.cuda.current_stream().cuda_stream)
    assert gc.lib.gc_selftest_bounded_wait(ctx.handle, 200_000_000) == 0   # ~0.1 s at 2 GHz
    with pytest.raises(gc.GcError) as e:
        ctx.synchronize()
    assert e.value.status == "GC_ERR_TIMEOUT" and "bounded device wait" in str(e.value)
    ctx.synchronize()                                   # cleared: no error the second time
    rng = np.random.default_rng(3)
    f = rng.standard_normal((16, 16, 16))
    g = gc.Grid(16, 16, 16)
    out = gc.laplacian(torch.from_numpy(f).cuda(), g, 4, ctx=ctx)
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle.op("laplacian", 4, f))
    assert gc.lib.gc_selftest_bounded_wait(ctx.handle, -1) != 0            # argument checks
    ctx.close()


def test_non_finite_detection(gc):
    """gc_check_finite: a NaN or an infinity planted on the host is found at
    its first flat index, with its component and cell in the message; a
    finite field passes; float fields and vector fields too."""
    import torch
    g = gc.Grid(12, 10, 8)
    f = torch.randn(g.shape, device="cuda", dtype=torch.float64)
    gc.check_finite(f, g)
    f[3, 4, 5] = float("nan")
    f[6, 0, 0] = float("inf")
    with pytest.raises(gc.GcError) as e:
        gc.check_finite(f, g)
    assert e.value.status == "GC_ERR_NONFINITE"
    assert "flat index 413" in str(e.value) and "cell (5, 4, 3)" in str(e.value)   # 3*120 + 4*12 + 5
    v = torch.zeros((3,) + g.shape, device="cuda", dtype=torch.float32)
    gc.check_finite(v, g)
    v[2, 0, 1, 2] = float("-inf")
    with pytest.raises(gc.GcError, match="component 2, cell \\(2, 1, 0\\)"):
        gc.check_finite(v, g)
    # A blown-up trajectory: explicit Euler far beyond its stability limit.
    psi = (0.05 * torch.rand((1, 64, 64), device="cuda", dtype=torch.float64)).contiguous()
    gc.ch_integrate(psi, gc.Grid(64, 64, 1), gc.CahnHilliardRhs(1.0, 1.0, 2), 1.0, 200, gc.ExplicitEuler)
    with pytest.raises(gc.GcError) as e:
        gc.check_finite(psi, gc.Grid(64, 64, 1))
    assert e.value.status == "GC_ERR_NONFINITE"

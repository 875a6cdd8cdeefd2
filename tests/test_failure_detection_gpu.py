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

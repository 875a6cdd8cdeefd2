"""Calls are ordered with the caller's stream: work torch enqueues before a
call is visible to it, and work enqueued after the call sees its results,
with no device-wide synchronisation in between."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _busy(torch):
    a = torch.randn(4096, 4096, device="cuda")
    for _ in range(6):
        a = a @ a / 64.0
    return a


@pytest.mark.parametrize("side", [False, True])
def test_inputs_and_outputs_follow_stream_order(gc, side):
    import torch
    stream = torch.cuda.Stream() if side else torch.cuda.current_stream()
    ctx = gc.Context(0, stream.cuda_stream)
    g = gc.Grid(1024, 1024, 1)
    rng = np.random.default_rng(0)
    pattern = torch.from_numpy(rng.standard_normal(g.shape)).cuda()
    want_lap = gc.laplacian(pattern, g, 2)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        x = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
        _busy(torch)
        x.copy_(pattern)                      # producer on the caller stream
        total = gc.integrate(x, g, ctx=ctx)   # must see the copy
        y = gc.laplacian(x, g, 2, ctx=ctx)
        diff = (y - want_lap).abs().max()     # consumer on the caller stream
        psi = 0.05 * torch.ones(g.shape, dtype=torch.float64, device="cuda")
        gc.ch_integrate(psi, g, gc.CahnHilliardRhs(), 0.01, 20, gc.RK4, ctx=ctx)
        s = psi.sum()
    torch.cuda.synchronize()
    assert total == gc.integrate(pattern, g)
    assert float(diff) == 0.0
    assert abs(float(s) - 0.05 * g.size) < 1e-9 * g.size
    ctx.close()


def test_event_timing_covers_the_work(gc):
    """CUDA events on the caller stream bracket the library's kernels."""
    import time
    import torch
    g = gc.Grid(4096, 4096, 1)
    psi = 0.05 * torch.rand(g.shape, dtype=torch.float64, device="cuda")
    rhs = gc.CahnHilliardRhs()
    gc.ch_integrate(psi, g, rhs, 0.01, 16, gc.RK4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gc.ch_integrate(psi, g, rhs, 0.01, 32, gc.RK4)
    torch.cuda.synchronize()
    host_ms = (time.perf_counter() - t0) * 1e3
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    gc.ch_integrate(psi, g, rhs, 0.01, 32, gc.RK4)
    e.record()
    torch.cuda.synchronize()
    assert s.elapsed_time(e) > 0.5 * host_ms, (s.elapsed_time(e), host_ms)

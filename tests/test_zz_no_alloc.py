"""gc_integrate_noalloc: the pairwise integral for callers that cannot
allocate device memory (their device memory belongs to another allocator,
or their loop forbids allocation once running).  Called through the C ABI
with buffers the caller owns; its result must equal gc_integrate's
(bit-identical: the pairwise tree is exact), on two calls in a row that
share the library's fixed scratch array, and no device memory may be taken
by those calls.  Kept in a file of its own that pytest collects last."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(gc):
    f = gc.lib.gc_integrate_noalloc
    f.argtypes = [C.POINTER(gc.gc_grid), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_integrate_twice(gc):
    import torch
    f = _bind(gc)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    cases = [(gc.Grid(513, 257, 33, 0.5, 0.25, 2.0), torch.float64),
             (gc.Grid(1000, 999, 1), torch.float32),
             (gc.Grid(8192, 4096, 1), torch.float64)]
    result = torch.empty(1, dtype=torch.float64, device="cuda")
    # set-up call (first call on this device), then measure free memory
    x0 = torch.ones(cases[0][0].shape, dtype=torch.float64, device="cuda")
    assert f(C.byref(cases[0][0].c()), 0, x0.data_ptr(), result.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    inputs = [torch.from_numpy(rng.standard_normal(g.shape)).to("cuda", dt) for g, dt in cases]
    want = [gc.integrate(x, g) for x, (g, _) in zip(inputs, cases)]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for rep in range(2):
        for x, (g, dt), w in zip(inputs, cases, want):
            code = 0 if dt == torch.float64 else 1
            assert f(C.byref(g.c()), code, x.data_ptr(), result.data_ptr(), stream) == 0, \
                gc.lib.gc_last_error().decode()
            torch.cuda.synchronize()
            assert float(result.item()) == w, (rep, g, float(result.item()), w)
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_back_to_back_on_one_stream(gc):
    """The usage the header prescribes: calls queued one after another on one
    (non-default) stream, with no host wait between them, each reusing the
    shared array; every result lands in its own element and all equal
    gc_integrate bit for bit after one synchronize."""
    import torch
    f = _bind(gc)
    rng = np.random.default_rng(6)
    cases = [(gc.Grid(300, 200, 7), torch.float64), (gc.Grid(4096, 4096, 1), torch.float64),
             (gc.Grid(77, 1, 1), torch.float32)]
    inputs = [torch.from_numpy(rng.standard_normal(g.shape)).to("cuda", dt) for g, dt in cases]
    want = [gc.integrate(x, g) for x, (g, _) in zip(inputs, cases)]
    side = torch.cuda.Stream()
    results = torch.full((6,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        for rep in range(2):
            for k, (x, (g, dt)) in enumerate(zip(inputs, cases)):
                code = 0 if dt == torch.float64 else 1
                ptr = results.data_ptr() + 8 * (3 * rep + k)
                assert f(C.byref(g.c()), code, x.data_ptr(), ptr, side.cuda_stream) == 0, \
                    gc.lib.gc_last_error().decode()
    side.synchronize()
    got = results.cpu().tolist()
    assert got == want + want, (got, want)


def test_noalloc_rejects_oversized_field(gc):
    import torch
    f = _bind(gc)
    g = gc.Grid(1 << 15, 1 << 15, 1)  # 2^30 cells > 2^29
    result = torch.empty(1, dtype=torch.float64, device="cuda")
    dummy = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = f(C.byref(g.c()), 0, dummy.data_ptr(), result.data_ptr(), None)
    assert rc == 1
    assert "2^29" in gc.lib.gc_last_error().decode()

"""The reference's 31 named partial derivatives (diff/MixedPartial.hpp,
ThirdOrder.hpp, FourthOrder.hpp over diff/detail/MultiIndexDerivative.hpp)
on the GPU: double results bit-identical to the oracle (itself bit-identical
to the reference, pinned by tests/golden), float within stated tolerance,
order 6 (no reference counterpart) by convergence against analytic
derivatives, and the per-axis extent rule."""
import math

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu

GRIDS = [((9, 10, 12), (0.3, 0.25, 0.5)), ((1, 9, 17), (1.0, 1.0, 1.0)), ((8, 8, 40), (0.5, 1.0, 2.0)),
         ((40, 12, 10), (1.0, 1.0, 1.0))]


def run(gc, arr, grid, counts, order, dtype):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr)).to("cuda", dtype)
    out = gc.partial(t, grid, counts, order)
    torch.cuda.synchronize()
    return out.double().cpu().numpy()


@pytest.mark.parametrize("order", [2, 4])
def test_all_31_bit_exact_vs_oracle(gc, oracle, order):
    import torch
    rng = np.random.default_rng(31 + order)
    for shape, h in GRIDS:
        f = rng.standard_normal(shape)
        g = gc.Grid(shape[2], shape[1], shape[0], *h)
        for counts in oracle_lib.PARTIALS:
            try:
                want = oracle.mixed(counts, order, f, h)
            except ValueError:
                continue   # axis too short for this stencil: the error test below covers it
            got = run(gc, f, g, counts, order, torch.float64)
            assert np.array_equal(got, want), (shape, counts, order)


def test_named_functions_and_golden(gc):
    """gc.dxx ... gc.d4dxdydz2 map to the right counts (golden vectors from
    the reference itself)."""
    import os
    import torch
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz"))
    for gname, order in (("aniso3d", 4), ("flat2d", 2)):
        f, h = golden[f"{gname}/f"], tuple(golden[f"{gname}/h"])
        g = gc.Grid(f.shape[2], f.shape[1], f.shape[0], *h)
        for name, c in gc.PARTIALS.items():
            got = getattr(gc, name)(torch.from_numpy(f).cuda(), g, order)
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), golden[f"{gname}/partial{c[0]}{c[1]}{c[2]}_{order}"]), name


def test_float32_within_tolerance(gc, oracle):
    import torch
    rng = np.random.default_rng(5)
    shape, h = (12, 14, 16), (1.0, 1.0, 1.0)
    f = rng.standard_normal(shape)
    g = gc.Grid(16, 14, 12, *h)
    for counts in oracle_lib.PARTIALS:
        want = oracle.mixed(counts, 4, f, h)
        got = run(gc, f.astype(np.float32), g, counts, 4, torch.float32)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < 2e-5, (counts, err)


@pytest.mark.parametrize("counts", [(1, 1, 0), (2, 1, 0), (1, 1, 2), (3, 0, 1), (2, 2, 0)])
def test_order6_convergence(gc, counts):
    """Order 6 against the analytic derivative of a Fourier mode: slope 6."""
    import torch
    errs = []
    kx, ky, kz = 1, 2, 1
    for n in (16, 24, 32):
        h = 1.0 / n
        x = np.arange(n) * h
        Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
        ph = 2 * np.pi * (kx * X + ky * Y + kz * Z)
        f = np.sin(ph)
        total = sum(counts)
        exact = (2 * np.pi * kx) ** counts[0] * (2 * np.pi * ky) ** counts[1] * (2 * np.pi * kz) ** counts[2] * \
            np.sin(ph + total * np.pi / 2)
        got = run(gc, f, gc.Grid(n, n, n, h, h, h), counts, 6, torch.float64)
        errs.append(np.abs(got - exact).max() / np.abs(exact).max())
    slope = math.log(errs[0] / errs[2]) / math.log(32 / 16)
    assert abs(slope - 6) < 0.6, (counts, errs, slope)


def test_per_axis_extent_rule(gc):
    """diff/detail/PreconditionAxisExtent.hpp:64-79 per axis: a count-0 axis
    takes any extent; a differentiated axis with 2 <= N <= 2r is rejected,
    naming the axis."""
    import torch
    t = torch.zeros((3, 4, 16), device="cuda", dtype=torch.float64)
    g = gc.Grid(16, 4, 3)
    gc.partial(t, g, (2, 0, 0), 4)            # y and z not differentiated: any extent
    with pytest.raises(gc.GcError) as e:
        gc.partial(t, g, (1, 1, 0), 4)        # y: radius 2 needs N >= 5
    assert e.value.status == "GC_ERR_AXIS_EXTENT" and "axis y" in str(e.value)
    with pytest.raises(gc.GcError):
        gc.partial(t, g, (0, 0, 0), 2)

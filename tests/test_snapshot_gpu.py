"""Asynchronous snapshots of device fields and checkpoint / resume on the
GPU: a snapshot holds the field as it was when the call returned (later work
may overwrite it at once), files match the synchronous writers, and a run
resumed from a checkpoint is bit-identical to the uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _psi0(n, seed=3):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return (0.05 * (2 * torch.rand((1, n, n), generator=g, device="cuda", dtype=torch.float64) - 1)).contiguous()


def test_snapshot_is_taken_when_called(gc, tmp_path):
    """The field is overwritten right after each call; every file still holds
    the value at the call (slot ring of depth 2 wrapping several times)."""
    import torch
    n = 96
    grid = gc.Grid(n, n, 1)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    psi = _psi0(n)
    kept = []
    with gc.Snapshotter(depth=2) as snap:
        for k in range(6):
            gc.ch_integrate(psi, grid, rhs, 0.01, 20, gc.RK4)
            torch.cuda.synchronize()
            kept.append(psi.cpu().numpy().copy())
            snap.vtk(psi, grid, str(tmp_path / f"psi_{k:06d}.vtk"), "psi", binary=(k % 2 == 1))
            snap.checkpoint(psi, grid, str(tmp_path / f"state_{k}.gcb"), {"chunk": k})
            psi.fill_(float("nan"))                   # overwritten at once
            psi.copy_(torch.from_numpy(kept[-1]).cuda())
        snap.flush()
    for k, want in enumerate(kept):
        gc.write_vtk(want, grid, str(tmp_path / "sync.vtk"), "psi", binary=(k % 2 == 1))
        assert (tmp_path / f"psi_{k:06d}.vtk").read_bytes() == (tmp_path / "sync.vtk").read_bytes(), k
        back, g2, meta = gc.load_checkpoint(str(tmp_path / f"state_{k}.gcb"))
        assert np.array_equal(back, want) and meta == {"chunk": k} and g2 == grid


def test_resume_is_bit_identical(gc, tmp_path):
    """examples/cahn_hilliard.cpp's chunked RK4 loop, stopped half-way,
    checkpointed, loaded into a fresh buffer and continued."""
    import torch
    for shape in ((1, 128, 128), (24, 24, 24)):
        grid = gc.Grid(shape[2], shape[1], shape[0])
        rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
        g = torch.Generator(device="cuda").manual_seed(9)
        psi0 = (0.05 * (2 * torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) - 1)).contiguous()
        whole = psi0.clone()
        gc.ch_integrate(whole, grid, rhs, 0.005, 200, gc.RK4)
        half = psi0.clone()
        gc.ch_integrate(half, grid, rhs, 0.005, 100, gc.RK4)
        with gc.Snapshotter(depth=1) as snap:
            snap.checkpoint(half, grid, str(tmp_path / "mid.gcb"), {"step": 100, "t": 0.5})
        half.fill_(0.0)
        resumed, g2, meta = gc.load_checkpoint(str(tmp_path / "mid.gcb"), device="cuda")
        assert meta == {"step": 100, "t": 0.5} and g2 == grid
        gc.ch_integrate(resumed, g2, rhs, 0.005, 100, gc.RK4)
        torch.cuda.synchronize()
        assert torch.equal(resumed, whole), shape


def test_float_and_vector_fields(gc, tmp_path):
    import torch
    grid = gc.Grid(10, 9, 8)
    u = torch.randn((3,) + grid.shape, device="cuda", dtype=torch.float32)
    with gc.Snapshotter() as snap:
        snap.checkpoint(u, grid, str(tmp_path / "u.gcb"))
        snap.vtk(u[1].contiguous(), grid, str(tmp_path / "u1.vtk"), "uy")
    back, _, _ = gc.load_checkpoint(str(tmp_path / "u.gcb"), device="cuda")
    assert back.dtype == torch.float32 and torch.equal(back, u)
    gc.write_vtk(u[1].cpu().numpy(), grid, str(tmp_path / "sync.vtk"), "uy")
    assert (tmp_path / "u1.vtk").read_bytes() == (tmp_path / "sync.vtk").read_bytes()


def test_write_failure_reported_at_flush(gc, tmp_path):
    grid = gc.Grid(8, 8, 1)
    psi = _psi0(8)
    snap = gc.Snapshotter()
    snap.vtk(psi, grid, str(tmp_path / "missing_dir" / "x.vtk"))
    with pytest.raises(ValueError, match="cannot open"):
        snap.flush()
    snap.vtk(psi, grid, str(tmp_path / "ok.vtk"))   # usable again after the error was reported
    snap.close()
    assert (tmp_path / "ok.vtk").exists()

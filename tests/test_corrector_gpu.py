"""Learned coarse-step corrector: the library's BF16 tensor-core forward and
backward kernels against a CPU float64 restatement of the same network, the
loss going down under the library's own Adam training, what the trained
network gains over the coarse scheme without it, and the plain-RK4 fallback.

Tolerances: BF16 weights and activations carry ~3 significant digits through
six layers, so the forward correction and the gradient are compared with the
float64 network in relative L2 (forward < 3e-2, gradient < 6e-2, cosine
> 0.995)."""
import numpy as np
import pytest

import corrector_ref

pytestmark = pytest.mark.gpu


def _ch_pairs(gc, n, size, steps_between, seed, warm=0):
    """Pairs (c(t), c(t + 16 dt)) of the plain GPU solver, dt = 0.01."""
    import torch
    rng = np.random.default_rng(seed)
    g = gc.Grid(size, size, 1)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    ins, outs = [], []
    for _ in range(n):
        c = torch.from_numpy(rng.uniform(-0.3, 0.3) + 0.05 * (2 * rng.random((1, size, size)) - 1)).cuda()
        gc.ch_integrate(c, g, rhs, 0.01, warm + int(rng.integers(0, steps_between)), gc.RK4)
        a = c.clone()
        gc.ch_integrate(c, g, rhs, 0.01, 16, gc.RK4)
        ins.append(a[0])
        outs.append(c[0].clone())
    return torch.stack(ins), torch.stack(outs)


def test_forward_matches_cpu_network(gc):
    import torch
    params = gc.corrector_init_params(seed=1, last_scale=1.0)
    rng = np.random.default_rng(2)
    c = rng.uniform(-1, 1, (2, 40, 56))
    net = gc.Corrector(40, 56, max_batch=2)
    net.set_params(params, s_out=0.05)
    got = net.forward(torch.from_numpy(c).float().cuda()).double().cpu().numpy()
    want = corrector_ref.delta(params, c.astype(np.float32), 0.05)
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel < 3e-2, rel
    assert np.abs(got.mean(axis=(1, 2))).max() < 1e-6   # zero-mean projection
    net.close()


def test_gradient_matches_cpu_network(gc):
    import torch
    params = gc.corrector_init_params(seed=3, last_scale=1.0)
    rng = np.random.default_rng(4)
    c = rng.uniform(-1, 1, (2, 32, 48)).astype(np.float32)
    target = (c + 0.02 * rng.standard_normal(c.shape)).astype(np.float32)
    net = gc.Corrector(32, 48, max_batch=2)
    net.set_params(params, s_out=0.05)
    g_gpu, loss_gpu = net.gradient(torch.from_numpy(c).cuda(), torch.from_numpy(target).cuda())
    loss_cpu, g_cpu = corrector_ref.loss_and_grad(params, c, target, 0.05)
    assert abs(loss_gpu - loss_cpu) / loss_cpu < 1e-2, (loss_gpu, loss_cpu)
    rel = np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu)
    cos = float(g_gpu @ g_cpu / (np.linalg.norm(g_gpu) * np.linalg.norm(g_cpu)))
    assert rel < 6e-2 and cos > 0.995, (rel, cos)
    # per-layer: every layer's gradient agrees, not just the total
    per = 9 * 32 * 32 + 32
    for layer in range(6):
        a, b = g_gpu[layer * per:(layer + 1) * per], g_cpu[layer * per:(layer + 1) * per]
        assert np.linalg.norm(a - b) <= 0.1 * np.linalg.norm(b) + 1e-12, layer
    net.close()


def _base_features(gc, c, dt, stages=6):
    """B(c), [u, e] and rho: u = (B - c)/rms, e = est/rms, rho = rms(est),
    est = (B - c)/dt - (f(c) + f(B))/2, from the library's own RKC2 step and
    RHS (FP64)."""
    import torch
    h, w = c.shape[1:]
    g = gc.Grid(w, h, 1)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    ct = torch.from_numpy(c).cuda()
    base = ct.clone()
    est = torch.empty_like(ct)
    for b in range(c.shape[0]):
        gc.ch_rkc(base[b], g, rhs, dt, 1, stages)
        est[b] = (base[b] - ct[b]) / dt - 0.5 * (gc.ch_rhs(ct[b], g, rhs)[0] + gc.ch_rhs(base[b], g, rhs)[0])
    base, est = base.cpu().numpy(), est.cpu().numpy()
    incr = base - c
    sigma = np.sqrt((incr ** 2).mean(axis=(1, 2)))
    rho = np.sqrt((est ** 2).mean(axis=(1, 2)))
    return base, [incr / sigma[:, None, None], est / rho[:, None, None]], rho


def test_base_step_and_normalized_loss_match_cpu_network(gc):
    """With an RKC2 base step B: input channels (B(c) - c) and the base step's
    trapezoid residual est, each at unit RMS; output scaled by Dt rms(est);
    coarse step B(c) + delta; loss normalised by the base step's error.
    Against the float64 network fed the same features (B and f from the
    library's gc_ch_rkc and gc_ch_rhs, bit-identical to their CPU
    restatements)."""
    import torch
    params = gc.corrector_init_params(seed=6, last_scale=1.0, inputs=3)
    rng = np.random.default_rng(8)
    h, w, dtc = 32, 40, 0.16
    c = rng.uniform(-1, 1, (2, h, w))
    base, feats, rho = _base_features(gc, c, dtc)
    net = gc.Corrector(h, w, max_batch=2)
    net.set_params(params, s_out=0.5)
    net.set_base(gc.CahnHilliardRhs(1.0, 1.0, 2), dtc, 6)
    ct = torch.from_numpy(c).cuda()
    got = net.forward(ct).double().cpu().numpy() - (base - c)          # the network's part
    want = corrector_ref.delta(params, c, 0.5, feats, dtc * rho)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 3e-2
    assert np.abs(got.mean(axis=(1, 2))).max() < 1e-5 * np.abs(want).max()
    no_feat = corrector_ref.delta(params, c, 0.5, (), dtc * rho)
    assert np.linalg.norm(no_feat - want) > 0.1 * np.linalg.norm(want)   # the features matter
    target = base + 0.3 * dtc * rho[:, None, None] * rng.standard_normal(c.shape)
    net.set_loss(True)
    g_gpu, loss_gpu = net.gradient(ct, torch.from_numpy(target).cuda())
    loss_cpu, g_cpu = corrector_ref.loss_and_grad(params, c, target, 0.5, feats, dtc * rho, start=base,
                                                  normalized=True)
    assert abs(loss_gpu - loss_cpu) / loss_cpu < 1e-2, (loss_gpu, loss_cpu)
    cos = float(g_gpu @ g_cpu / (np.linalg.norm(g_gpu) * np.linalg.norm(g_cpu)))
    assert np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu) < 6e-2 and cos > 0.995, cos
    net.set_base(None)
    got_off = net.forward(ct).double().cpu().numpy()
    without = corrector_ref.delta(params, c, 0.5)
    assert np.linalg.norm(got_off - without) / np.linalg.norm(without) < 3e-2
    net.close()


def test_training_gains_over_the_scheme_without_network(gc):
    """Trained on solver pairs at 64 x 64, the network's coarse step c + delta
    is closer to 16 fine RK4 steps than the coarse step without it (c), on
    held-out pairs; plain RK4 at the coarse dt = 0.16 is unstable."""
    import torch
    size = 64
    xin, xout = _ch_pairs(gc, 48, size, 400, seed=10, warm=100)
    vin, vout = _ch_pairs(gc, 8, size, 400, seed=99, warm=100)
    net = gc.Corrector(size, size, max_batch=16)
    net.set_params(gc.corrector_init_params(seed=5, last_scale=0.1), s_out=0.05)
    xin32, xout32 = xin.float(), xout.float()
    losses = []
    for it in range(400):
        k = (it * 16) % 48
        losses.append(net.train_step(xin32[k:k + 16], xout32[k:k + 16], lr=2e-3 if it < 300 else 5e-4))
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
    delta = net.forward(vin.float()).double()
    err_net = float(((vin + delta - vout) ** 2).mean())
    err_without = float(((vin - vout) ** 2).mean())
    assert err_net < 0.5 * err_without, (err_net, err_without)
    # The coarse step as one plain RK4 step of dt = 0.16: unstable.
    c = vin[:1].clone()
    g = gc.Grid(size, size, 1)
    gc.ch_integrate(c, g, gc.CahnHilliardRhs(1.0, 1.0, 2), 0.16, 20, gc.RK4)
    assert not bool(torch.isfinite(c).all()) or float(c.abs().max()) > 10.0
    net.close()


def test_rejected_steps_fall_back_to_plain_rk4_exactly(gc, oracle):
    """A network that proposes no change (all-zero weights) leaves the
    trapezoid residual at 1, so every coarse step is rejected and taken by
    16 plain RK4 steps: the state is bit-identical to the fine solver."""
    import torch
    size = 48
    rng = np.random.default_rng(7)
    psi0 = 0.05 * (2 * rng.random((1, size, size)) - 1)
    net = gc.Corrector(size, size)
    net.set_params(np.zeros(net.n_params, dtype=np.float32))
    t = torch.from_numpy(psi0[0].copy()).cuda()
    g = gc.Grid(size, size, 1)
    stats = net.advance(t, g, gc.CahnHilliardRhs(1.0, 1.0, 2), n_coarse=5, residual_tol=0.5)
    assert stats["fallbacks"] == 5 and stats["accepted"] == 0
    # By cause: an unchanged proposal keeps F (energy check passes) but its
    # residual is 1 > 0.5.
    assert stats["rejected_residual"] == 5 and stats["rejected_energy"] == 0
    torch.cuda.synchronize()
    want = oracle.ch_integrate(2, 1.0, 1.0, psi0, 0.01, 80)
    assert np.array_equal(t.cpu().numpy(), want[0])
    net.close()


def test_parameters_save_and_load(gc, tmp_path):
    """Corrector.save / load: FP32 master parameters, s_out, the base step and
    the loss setting survive a round trip through the checkpoint format; the
    restored network gives the same increment."""
    import torch
    net = gc.Corrector(32, 32, max_batch=1)
    net.set_params(gc.corrector_init_params(seed=4, last_scale=0.5, inputs=3), s_out=0.7)
    net.set_base(gc.CahnHilliardRhs(1.0, 0.8, 2), 0.16, 6)
    net.set_loss(True)
    path = str(tmp_path / "net.gcb")
    net.save(path, {"trained_on": "unit test"})
    c = (0.1 * torch.rand((1, 32, 32), device="cuda", dtype=torch.float64)).contiguous()
    want = net.forward(c)
    other = gc.Corrector(32, 32, max_batch=1)
    meta = other.load(path)
    assert meta["trained_on"] == "unit test" and meta["s_out"] == 0.7
    assert np.array_equal(other.get_params(), net.get_params())
    assert torch.equal(other.forward(c), want)
    with pytest.raises(ValueError, match="does not hold"):
        gc.save_checkpoint(np.zeros(10, dtype=np.float32), gc.Grid(10, 1, 1), str(tmp_path / "x.gcb"))
        other.load(str(tmp_path / "x.gcb"))
    net.close()
    other.close()


def test_batch_size_does_not_change_results(gc):
    """A 512^2 sample alone and as each of three copies in one batch (the
    persistent convolution then splits the tiles differently over its CTAs
    and pipeline slots): every sample's increment is bit-identical."""
    import torch
    net = gc.Corrector(512, 512, max_batch=3)
    net.set_params(gc.corrector_init_params(seed=2, last_scale=0.3, inputs=1), s_out=0.5)
    c = (0.3 * torch.rand((1, 512, 512), device="cuda", dtype=torch.float64) - 0.15).contiguous()
    one = net.forward(c)
    three = net.forward(c.repeat(3, 1, 1).contiguous())
    torch.cuda.synchronize()
    for b in range(3):
        assert torch.equal(three[b], one[0]), b
    net.close()

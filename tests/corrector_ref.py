"""CPU float64 restatement of the corrector network (test infrastructure):
the same 6-layer periodic 3x3 CNN, GELU (tanh form), zero-mean output, with
torch autograd for the reference gradient of the loss (see loss_and_grad).
Inputs: channel 0 = c, channels 1, 2 = the features (zero when absent)."""
import numpy as np
import torch
import torch.nn.functional as F

LAYERS, CH = 6, 32


def unpack(params):
    p = torch.as_tensor(np.asarray(params, dtype=np.float64))
    per = 9 * CH * CH + CH
    out = []
    for layer in range(LAYERS):
        blk = p[layer * per:(layer + 1) * per]
        w = blk[:9 * CH * CH].reshape(9, CH, CH)   # t, ci, co
        b = blk[9 * CH * CH:]
        out.append((w, b))
    return out


def forward(params_t, c, s_out, features=(), scale=None):
    """params_t: list of (W[t][ci][co], b) float64 tensors; c and each of
    `features` (at most 2): (B, H, W); scale: (B,) output scale per sample
    (1 when absent)."""
    feats = list(features) + [torch.zeros_like(c)] * (2 - len(features))
    x = torch.stack([c] + feats, dim=1)
    for layer, (w, b) in enumerate(params_t):
        k = w.reshape(3, 3, CH, CH).permute(3, 2, 0, 1)  # co, ci, ky, kx
        if layer == 0:
            k = k[:, :3]
        z = F.conv2d(F.pad(x, (1, 1, 1, 1), mode="circular"), k) + b[None, :, None, None]
        x = F.gelu(z, approximate="tanh") if layer + 1 < LAYERS else z
    z6 = x[:, 0]
    d = s_out * (z6 - z6.mean(dim=(1, 2), keepdim=True))
    return d if scale is None else d * scale[:, None, None]


def _t(a):
    return None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float64))


def delta(params, c, s_out, features=(), scale=None):
    with torch.no_grad():
        return forward(unpack(params), _t(c), s_out, [_t(f) for f in features], _t(scale)).numpy()


def loss_and_grad(params, c, target, s_out, features=(), scale=None, start=None, normalized=False):
    """Loss sum_b sum_p r^2 / (N den_b), r = start + delta - target (start = c
    when absent), N all cells, den_b = mean_p((target - start)^2) of sample b
    when normalized else 1."""
    pt = [(w.clone().requires_grad_(True), b.clone().requires_grad_(True)) for w, b in unpack(params)]
    ct, tt = _t(c), _t(target)
    st = ct if start is None else _t(start)
    d = forward(pt, ct, s_out, [_t(f) for f in features], _t(scale))
    r2 = (st + d - tt) ** 2
    if normalized:
        den = ((tt - st) ** 2).mean(dim=(1, 2), keepdim=True)
        loss = (r2 / den).sum() / r2.numel()
    else:
        loss = r2.mean()
    loss.backward()
    grads = []
    for w, b in pt:
        grads.append(w.grad.reshape(-1))
        grads.append(b.grad)
    return float(loss.detach()), torch.cat(grads).numpy()

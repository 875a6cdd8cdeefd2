"""CPU float64 restatement of the corrector network (test infrastructure):
the same 6-layer periodic 3x3 CNN, GELU (erf form), zero-mean output, with
torch autograd for the reference gradient of mean((c + delta - target)^2)."""
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


def forward(params_t, c, s_out):
    """params_t: list of (W[t][ci][co], b) float64 tensors; c: (B, H, W)."""
    x = c[:, None]
    for layer, (w, b) in enumerate(params_t):
        k = w.reshape(3, 3, CH, CH).permute(3, 2, 0, 1)  # co, ci, ky, kx
        if layer == 0:
            k = k[:, :1]
        z = F.conv2d(F.pad(x, (1, 1, 1, 1), mode="circular"), k) + b[None, :, None, None]
        x = F.gelu(z) if layer + 1 < LAYERS else z
    z6 = x[:, 0]
    return s_out * (z6 - z6.mean(dim=(1, 2), keepdim=True))


def delta(params, c, s_out):
    with torch.no_grad():
        return forward(unpack(params), torch.as_tensor(np.asarray(c, dtype=np.float64)), s_out).numpy()


def loss_and_grad(params, c, target, s_out):
    pt = [(w.clone().requires_grad_(True), b.clone().requires_grad_(True)) for w, b in unpack(params)]
    ct = torch.as_tensor(np.asarray(c, dtype=np.float64))
    tt = torch.as_tensor(np.asarray(target, dtype=np.float64))
    d = forward(pt, ct, s_out)
    loss = ((ct + d - tt) ** 2).mean()
    loss.backward()
    grads = []
    for w, b in pt:
        grads.append(w.grad.reshape(-1))
        grads.append(b.grad)
    return float(loss.detach()), torch.cat(grads).numpy()

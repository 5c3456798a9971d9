"""CPU float64 restatement of the restoration U-Net (TEST INFRASTRUCTURE ONLY).

The network has no upstream counterpart (the upstream toolkit has no learned component); this
file restates, with torch float64 autograd on the CPU, the network that
cuda_ultrasound_toolkit_b200/csrc/unet.cu computes with its tcgen05 kernels, so that tests
can check the GPU forward pass and every parameter gradient against it. Only tests import it.

Parameters come as the library's master vector (FP32 [cout][27][cin] weights and [cout] biases
per layer, at the offsets the library reports) and are used exactly, in float64.
"""
import numpy as np
import torch
import torch.nn.functional as F


def _conv(p, layer, x, relu=True):
    cin, cout = layer["cin"], layer["cout"]
    if not isinstance(p, torch.Tensor):
        p = torch.as_tensor(np.asarray(p, dtype=np.float64))
    w = p[layer["w_off"]:layer["w_off"] + cout * 27 * cin].reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
    b = p[layer["b_off"]:layer["b_off"] + cout]
    y = F.conv3d(x, w, b, padding=1)
    return F.relu(y) if relu else y


def forward(p, layers, vol, target=None):
    """vol, target: complex [n][Z][Y][X]. Returns (restored volume, loss or None), where
    loss = sum |vol/s + f - target/s|^2 / (n * voxels), s the per-volume RMS of vol."""
    vol = torch.as_tensor(vol).to(torch.complex128)
    n = vol.shape[0]
    s = torch.sqrt(torch.mean(vol.real ** 2 + vol.imag ** 2, dim=(1, 2, 3)))  # [n]
    sv = s.reshape(n, 1, 1, 1)
    u = torch.stack([vol.real, vol.imag], dim=1) / sv.unsqueeze(1)
    x0 = torch.cat([u, torch.zeros((n, 14) + tuple(vol.shape[1:]), dtype=torch.float64)], dim=1)
    L = layers
    e0a = _conv(p, L[0], x0)
    e0b = _conv(p, L[1], e0a)
    e1a = _conv(p, L[2], F.avg_pool3d(e0b, 2))
    e1b = _conv(p, L[3], e1a)
    e2a = _conv(p, L[4], F.avg_pool3d(e1b, 2))
    e2b = _conv(p, L[5], e2a)
    bt = _conv(p, L[6], F.avg_pool3d(e2b, 2))
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")  # noqa: E731
    d2 = _conv(p, L[7], torch.cat([e2b, up(bt)], dim=1))
    d1 = _conv(p, L[8], torch.cat([e1b, up(d2)], dim=1))
    d0 = _conv(p, L[9], torch.cat([e0b, up(d1)], dim=1))
    f = _conv(p, L[10], d0, relu=False)[:, :2]
    out = vol + sv * torch.complex(f[:, 0], f[:, 1])
    loss = None
    if target is not None:
        t = torch.as_tensor(target).to(torch.complex128)
        tn = torch.stack([t.real, t.imag], dim=1) / sv.unsqueeze(1)
        diff = u + f - tn
        loss = torch.sum(diff * diff) / (n * vol[0].numel())
    return out, loss


def gradients(p, layers, vol, target):
    """(loss, d loss / d p) with p the master vector (float64 autograd)."""
    pt = torch.tensor(np.asarray(p, dtype=np.float64), requires_grad=True)
    _, loss = forward(pt, layers, vol, target)
    loss.backward()
    return float(loss.detach()), pt.grad.numpy()

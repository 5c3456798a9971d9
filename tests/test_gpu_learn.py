"""Tensor-core 3-D convolutions and the restoration U-Net against CPU float64 references.

Single convolutions use BF16-exact inputs, so the reference is exact up to the kernel's FP32
accumulation and (forward) the BF16 rounding of the output. The U-Net keeps every activation
and gradient in BF16 between layers, so its forward output and parameter gradients are
compared with the float64 restatement in oracle/unet_ref.py by relative L2 error.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from cuda_ultrasound_toolkit_b200 import learn

pytestmark = pytest.mark.gpu

TOL_CONV_OUT = 6e-3      # BF16 output rounding (2^-9 relative) over a whole volume
TOL_WGRAD = 2e-5         # FP32 accumulation order of BF16-exact products
TOL_UNET_OUT = 5e-3      # restored volume (the residual branch is a small correction)
TOL_UNET_GRAD = 6e-2     # parameter gradients through 22 BF16-stored activations/gradients


def rel_l2(a, b):
    a, b = torch.as_tensor(a).cpu(), torch.as_tensor(b).cpu()
    if a.is_complex() or b.is_complex():
        a = torch.view_as_real(a.to(torch.complex128))
        b = torch.view_as_real(b.to(torch.complex128))
    a, b = a.to(torch.float64), b.to(torch.float64)
    return float(torch.linalg.norm((a - b).ravel()) / max(float(torch.linalg.norm(b.ravel())), 1e-300))


def bf16_exact(*shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen, dtype=torch.float64) * scale).to(torch.bfloat16).to(torch.float64)


# (cin, cout) pairs the library instantiates
INSTANTIATED = {(16, 16), (16, 32), (16, 64), (32, 16), (32, 32), (32, 64), (32, 128), (64, 16), (64, 32), (64, 64),
                (128, 32), (128, 64)}

CONV_CASES = [
    # (cin, cout, Z, Y, X, n)
    (16, 16, 8, 16, 128, 1),
    (16, 32, 16, 16, 32, 2),
    (32, 64, 8, 8, 32, 1),
    (64, 64, 4, 8, 16, 1),
    (128, 32, 8, 8, 8, 1),
    (32, 128, 4, 8, 8, 1),
    (16, 16, 4, 4, 4, 1),      # smaller than one 128-voxel tile
    (64, 16, 16, 8, 16, 2),
    # 128-wide volumes: the halo kernel (two channel blocks per stage, cout <= 32)
    (32, 16, 4, 8, 128, 2),
    (16, 32, 2, 2, 128, 1),
    (64, 16, 2, 4, 128, 1),
]


@pytest.mark.parametrize("cin,cout,Z,Y,X,n", [c for c in CONV_CASES if c[4] == 128])
def test_conv3d_halo_kernel_matches_tap_kernel(cin, cout, Z, Y, X, n):
    """The halo kernel and the per-tap kernel compute the same sums (FP32 accumulation order may differ)."""
    g = torch.Generator().manual_seed(cin + cout + Z + Y)
    x = bf16_exact(n, cin, Z, Y, X, gen=g)
    w = bf16_exact(cout, cin, 3, 3, 3, gen=g, scale=(1.0 / (27 * cin)) ** 0.5)
    wf, _ = learn.relayout(learn.master_weight(w).float().cuda(), cin, cout)
    xc = learn.to_c8(x.float().cuda())
    a = learn.from_c8(learn.conv3d(xc, wf, None, cout)).float()
    learn.force_tap_kernel(True)
    try:
        b = learn.from_c8(learn.conv3d(xc, wf, None, cout)).float()
    finally:
        learn.force_tap_kernel(False)
    assert rel_l2(a.cpu(), b.cpu()) < 4e-3


@pytest.mark.parametrize("cin,cout,Z,Y,X,n", CONV_CASES)
def test_conv3d_forward(cin, cout, Z, Y, X, n):
    g = torch.Generator().manual_seed(cin * 1000 + cout + Z)
    x = bf16_exact(n, cin, Z, Y, X, gen=g)
    w = bf16_exact(cout, cin, 3, 3, 3, gen=g, scale=(1.0 / (27 * cin)) ** 0.5)
    b = torch.randn(cout, generator=g, dtype=torch.float64) * 0.1
    ref = F.relu(F.conv3d(x, w, b, padding=1))
    wf, _ = learn.relayout(learn.master_weight(w).float().cuda(), cin, cout)
    out = learn.conv3d(learn.to_c8(x.float().cuda()), wf, b.float().cuda(), cout, relu=True)
    got = learn.from_c8(out).float().cpu()
    assert rel_l2(got, ref) < TOL_CONV_OUT
    assert float((got.double() - ref).abs().max()) < 1e-2 * float(ref.abs().max()) + 1e-3


@pytest.mark.parametrize("cin,cout,Z,Y,X,n", CONV_CASES)
def test_conv3d_input_gradient(cin, cout, Z, Y, X, n):
    """The input gradient is the forward kernel with the flipped, transposed filter."""
    if (cout, cin) not in INSTANTIATED:
        pytest.skip("channel pair not instantiated for the transposed convolution")
    g = torch.Generator().manual_seed(cin + 7 * cout + Z)
    dy = bf16_exact(n, cout, Z, Y, X, gen=g)
    w = bf16_exact(cout, cin, 3, 3, 3, gen=g, scale=(1.0 / (27 * cout)) ** 0.5)
    ref = torch.nn.grad.conv3d_input((n, cin, Z, Y, X), w, dy, padding=1)
    _, wb = learn.relayout(learn.master_weight(w).float().cuda(), cin, cout)
    out = learn.conv3d(learn.to_c8(dy.float().cuda()), wb, None, cin, relu=False)
    assert rel_l2(learn.from_c8(out).float().cpu(), ref) < TOL_CONV_OUT


@pytest.mark.parametrize("cin,cout,Z,Y,X,n", CONV_CASES)
def test_conv3d_weight_gradient(cin, cout, Z, Y, X, n):
    g = torch.Generator().manual_seed(3 * cin + cout + X)
    x = bf16_exact(n, cin, Z, Y, X, gen=g)
    dy = bf16_exact(n, cout, Z, Y, X, gen=g)
    ref = torch.nn.grad.conv3d_weight(x, (cout, cin, 3, 3, 3), dy, padding=1)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    dw = learn.conv3d_weight_grad(learn.to_c8(x.float().cuda()), learn.to_c8(dy.float().cuda()), status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    got = learn.torch_weight(dw.cpu(), cin, cout)
    assert rel_l2(got, ref) < TOL_WGRAD


def _unet_case(shape, seed, nb=1):
    net = learn.UNet(shape, max_batch=nb, seed=seed)
    p = net.get_params()
    rng = np.random.default_rng(seed)
    # Give the (zero-initialised) output layer and the biases values, so every path is exercised.
    w, b = net.layer_params(p, 10)
    w[:2] = rng.normal(0, 0.05, w[:2].shape)
    b[:2] = rng.normal(0, 0.01, 2)
    for i in range(10):
        _, bi = net.layer_params(p, i)
        bi[:] = rng.normal(0, 0.02, bi.shape)
    # The library computes with BF16 weights: give the reference the same values.
    p = torch.tensor(p).to(torch.bfloat16).float().numpy()
    net.set_params(p)
    vol = rng.normal(size=(nb,) + shape) + 1j * rng.normal(size=(nb,) + shape)
    vol[:, shape[0] // 2, shape[1] // 2, shape[2] // 2] += 20.0
    tgt = vol * 0.8 + 0.3 * (rng.normal(size=vol.shape) + 1j * rng.normal(size=vol.shape))
    return net, p, vol.astype(np.complex64), tgt.astype(np.complex64)


@pytest.mark.parametrize("shape,nb", [((16, 16, 16), 1), ((32, 32, 32), 2), ((16, 32, 64), 1), ((16, 16, 128), 2)])
def test_unet_forward_matches_reference(shape, nb):
    from oracle import unet_ref
    net, p, vol, _ = _unet_case(shape, 11, nb)
    out = net.forward(torch.from_numpy(vol).cuda()).cpu().numpy()
    net.check()
    ref, _ = unet_ref.forward(p, net.layers, vol)
    assert rel_l2(torch.from_numpy(out), ref) < TOL_UNET_OUT
    # The residual the network adds, on its own, to a looser bar.
    assert rel_l2(torch.from_numpy(out - vol), ref - torch.from_numpy(vol).to(torch.complex128)) < 3e-2


@pytest.mark.parametrize("shape,nb", [((16, 16, 16), 1), ((32, 32, 32), 2), ((16, 16, 128), 1)])
def test_unet_gradients_match_reference(shape, nb):
    from oracle import unet_ref
    net, p, vol, tgt = _unet_case(shape, 5, nb)
    net.compute_gradients(torch.from_numpy(vol).cuda(), torch.from_numpy(tgt).cuda())
    loss = net.last_loss()
    grads = net.get_gradients()
    ref_loss, ref_g = unet_ref.gradients(p, net.layers, vol, tgt)
    # last_loss is the mean over real components; the reference loss is that times 2.
    assert abs(2 * loss - ref_loss) < 5e-3 * ref_loss
    for i, l in enumerate(net.layers):
        gw, gb = net.layer_params(grads, i)
        rw, rb = net.layer_params(ref_g, i)
        rw = rw[:l["cout_real"], :, :l["cin_real"]]
        assert rel_l2(gw[:l["cout_real"], :, :l["cin_real"]], rw) < TOL_UNET_GRAD, f"layer {i} weights"
        assert rel_l2(gb[:l["cout_real"]], rb[:l["cout_real"]]) < TOL_UNET_GRAD, f"layer {i} bias"
        # padded weights receive exactly zero gradient
        assert np.all(gw[l["cout_real"]:] == 0) and np.all(gw[:, :, l["cin_real"]:] == 0)


def test_unet_untrained_is_identity():
    net = learn.UNet((16, 16, 32), max_batch=1, seed=3)
    rng = np.random.default_rng(0)
    vol = (rng.normal(size=(1, 16, 16, 32)) + 1j * rng.normal(size=(1, 16, 16, 32))).astype(np.complex64)
    out = net.forward(torch.from_numpy(vol).cuda()).cpu().numpy()
    assert np.array_equal(out, vol)


def test_unet_training_reduces_loss():
    """A few Adam steps on a fixed pair: the loss must fall well below its start."""
    shape = (32, 32, 32)
    net = learn.UNet(shape, max_batch=2, seed=9)
    rng = np.random.default_rng(1)
    vol = rng.normal(size=(2,) + shape) + 1j * rng.normal(size=(2,) + shape)
    # target: the input smoothed along x (a task the convolutions can represent)
    tgt = (vol + np.roll(vol, 1, axis=3) + np.roll(vol, -1, axis=3)) / 3
    v = torch.from_numpy(vol.astype(np.complex64)).cuda()
    t = torch.from_numpy(tgt.astype(np.complex64)).cuda()
    net.compute_gradients(v, t)
    first = net.last_loss()
    for _ in range(60):
        net.train_step(v, t, 2e-3)
    net.compute_gradients(v, t)
    last = net.last_loss()
    assert last < 0.5 * first, (first, last)

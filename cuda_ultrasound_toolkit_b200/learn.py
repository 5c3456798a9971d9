"""Learned sparse-transmit restoration: the 3-D U-Net of csrc/unet.cu, trained and run by the
library's own tcgen05 convolution kernels (csrc/conv3d.cu), plus the C8 volume helpers the
tests use to drive single convolutions.

C8 layout: [n][c / 8][z][y][x][c % 8] BF16. Master weights: FP32 [cout][27][cin] with
tap = (kz * 3 + ky) * 3 + kx for the offsets (kz - 1, ky - 1, kx - 1).
"""
import ctypes

import numpy as np
import torch

from .api import _check, _stream_handle, lib

_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        vp, sz, u, b, f = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_bool, ctypes.c_float
        ull = ctypes.c_ulonglong
        fp = ctypes.POINTER(ctypes.c_float)
        sig = {
            "cutb_unet_create": ([u, u, u, u, ull], vp),
            "cutb_unet_destroy": ([vp], None),
            "cutb_unet_param_buffer_size": ([vp], sz),
            "cutb_unet_param_count": ([vp], sz),
            "cutb_unet_layer_count": ([], u),
            "cutb_unet_layer_info": ([vp, u, ctypes.POINTER(ull)], b),
            "cutb_unet_get_params": ([vp, fp], b),
            "cutb_unet_set_params": ([vp, fp], b),
            "cutb_unet_get_gradients": ([vp, fp], b),
            "cutb_unet_forward": ([vp, vp, vp, u, vp], b),
            "cutb_unet_compute_gradients": ([vp, vp, vp, u, vp], b),
            "cutb_unet_train_step": ([vp, vp, vp, u, f, vp], b),
            "cutb_unet_last_loss": ([vp, ctypes.POINTER(ctypes.c_double)], b),
            "cutb_unet_check": ([vp], b),
            "cutb_conv3d_relayout": ([vp, u, u, vp, vp, vp], b),
            "cutb_conv3d_forward": ([vp, vp, vp, vp, u, u, u, u, u, u, ctypes.c_int, vp, vp], b),
            "cutb_conv3d_weight_grad": ([vp, vp, vp, u, u, u, u, u, u, vp, vp], b),
            "cutb_debug_conv3d_force_tap_kernel": ([ctypes.c_int], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _bound = True
    return L


# ---- C8 layout -----------------------------------------------------------------------------------
def to_c8(t):
    """[n][C][Z][Y][X] (C a multiple of 8) -> C8 BF16 tensor [n][C/8][Z][Y][X][8] on t's device."""
    n, C, Z, Y, X = t.shape
    return t.reshape(n, C // 8, 8, Z, Y, X).permute(0, 1, 3, 4, 5, 2).contiguous().to(torch.bfloat16)


def from_c8(t):
    """C8 [n][CB][Z][Y][X][8] -> [n][CB*8][Z][Y][X] (same dtype)."""
    n, CB, Z, Y, X, _ = t.shape
    return t.permute(0, 1, 5, 2, 3, 4).reshape(n, CB * 8, Z, Y, X)


def torch_weight(w, cin, cout):
    """Master [cout][27][cin] -> torch Conv3d weight [cout][cin][3][3][3]."""
    return w.reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)


def master_weight(wt):
    """torch Conv3d weight [cout][cin][3][3][3] -> master [cout][27][cin]."""
    cout, cin = wt.shape[:2]
    return wt.permute(0, 2, 3, 4, 1).reshape(cout, 27, cin)


def relayout(w_master, cin, cout, stream=None):
    """BF16 forward and input-gradient weight relayouts of an FP32 master weight (device)."""
    w = w_master.contiguous().float()
    wf = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=w.device)
    wb = torch.empty_like(wf)
    _check(_lib().cutb_conv3d_relayout(w.data_ptr(), cin, cout, wf.data_ptr(), wb.data_ptr(), _stream_handle(stream)),
           "cutb_conv3d_relayout")
    return wf, wb


def conv3d(x_c8, wf, bias, cout, relu=False, status=None, stream=None):
    """One tensor-core 3x3x3 convolution on a C8 volume; returns the C8 output."""
    n, CB, Z, Y, X, _ = x_c8.shape
    out = torch.empty((n, cout // 8, Z, Y, X, 8), dtype=torch.bfloat16, device=x_c8.device)
    st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=x_c8.device)
    _check(_lib().cutb_conv3d_forward(x_c8.data_ptr(), wf.data_ptr(), bias.data_ptr() if bias is not None else None,
                                      out.data_ptr(), X, Y, Z, n, CB * 8, cout, int(relu), st.data_ptr(),
                                      _stream_handle(stream)), "cutb_conv3d_forward")
    return out


def force_tap_kernel(on):
    """Test hook: route every forward convolution through the per-tap kernel."""
    _lib().cutb_debug_conv3d_force_tap_kernel(int(bool(on)))


def conv3d_weight_grad(x_c8, dout_c8, status=None, stream=None):
    """FP32 weight gradient [cout][27][cin] of a 3x3x3 convolution (tensor cores)."""
    n, CB, Z, Y, X, _ = x_c8.shape
    cout = dout_c8.shape[1] * 8
    dw = torch.zeros((cout, 27, CB * 8), dtype=torch.float32, device=x_c8.device)
    st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=x_c8.device)
    _check(_lib().cutb_conv3d_weight_grad(x_c8.data_ptr(), dout_c8.data_ptr(), dw.data_ptr(), X, Y, Z, n, CB * 8, cout,
                                          st.data_ptr(), _stream_handle(stream)), "cutb_conv3d_weight_grad")
    return dw


class UNet:
    """The restoration network on one GPU (device buffers for up to ``max_batch`` volumes)."""

    def __init__(self, shape_zyx, max_batch=1, seed=1):
        Z, Y, X = shape_zyx
        L = _lib()
        self.shape = (Z, Y, X)
        self.max_batch = max_batch
        self._h = L.cutb_unet_create(X, Y, Z, max_batch, seed)
        if not self._h:
            _check(False, "cutb_unet_create")
        self.size = L.cutb_unet_param_buffer_size(self._h)
        self.layers = []
        info = (ctypes.c_ulonglong * 7)()
        for i in range(L.cutb_unet_layer_count()):
            _check(L.cutb_unet_layer_info(self._h, i, info), "cutb_unet_layer_info")
            cin, cout, cin_r, cout_r, level, w_off, b_off = list(info)
            self.layers.append(dict(cin=cin, cout=cout, cin_real=cin_r, cout_real=cout_r, level=level, w_off=w_off,
                                    b_off=b_off))

    def close(self):
        if self._h:
            _lib().cutb_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def param_count(self):
        return _lib().cutb_unet_param_count(self._h)

    def get_params(self):
        out = np.empty(self.size, dtype=np.float32)
        _check(_lib().cutb_unet_get_params(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "cutb_unet_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.size
        _check(_lib().cutb_unet_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "cutb_unet_set_params")

    def get_gradients(self):
        out = np.empty(self.size, dtype=np.float32)
        _check(_lib().cutb_unet_get_gradients(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "cutb_unet_get_gradients")
        return out

    def layer_params(self, p, i):
        """(weight [cout][27][cin], bias [cout]) views of layer i in a master vector."""
        l = self.layers[i]
        w = p[l["w_off"]:l["w_off"] + l["cout"] * 27 * l["cin"]].reshape(l["cout"], 27, l["cin"])
        b = p[l["b_off"]:l["b_off"] + l["cout"]]
        return w, b

    def _vol(self, t):
        assert t.is_cuda and t.dtype == torch.complex64 and t.is_contiguous() and tuple(t.shape[1:]) == self.shape
        assert 1 <= t.shape[0] <= self.max_batch
        return t

    def forward(self, vol, out=None, stream=None):
        """Restored volumes for complex64 device volumes [n][Z][Y][X]."""
        vol = self._vol(vol)
        if out is None:
            out = torch.empty_like(vol)
        _check(_lib().cutb_unet_forward(self._h, vol.data_ptr(), out.data_ptr(), vol.shape[0], _stream_handle(stream)),
               "cutb_unet_forward")
        return out

    def compute_gradients(self, vol, target, stream=None):
        vol, target = self._vol(vol), self._vol(target)
        _check(_lib().cutb_unet_compute_gradients(self._h, vol.data_ptr(), target.data_ptr(), vol.shape[0],
                                                  _stream_handle(stream)), "cutb_unet_compute_gradients")

    def train_step(self, vol, target, lr, stream=None):
        vol, target = self._vol(vol), self._vol(target)
        _check(_lib().cutb_unet_train_step(self._h, vol.data_ptr(), target.data_ptr(), vol.shape[0], float(lr),
                                           _stream_handle(stream)), "cutb_unet_train_step")

    def last_loss(self):
        """Mean squared normalised residual of the last gradient pass (synchronises)."""
        v = ctypes.c_double()
        _check(_lib().cutb_unet_last_loss(self._h, ctypes.byref(v)), "cutb_unet_last_loss")
        return v.value

    def check(self):
        _check(_lib().cutb_unet_check(self._h), "cutb_unet_check")

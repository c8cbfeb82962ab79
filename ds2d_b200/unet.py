"""Python mirror of the U-Net preconditioner C ABI (ds2d_unet_*): BF16 tensor-core inference and
training on the GPU; parameters are one flat FP32 vector in the oracle's layer order."""
import ctypes

import numpy as np

from ._lib import DS2DError, load


def layer_shapes(base=32):
    """(name, w shape [k][k][cout][cin], b shape [cout]) in the flat parameter order."""
    c = [base, 2 * base, 4 * base, 8 * base]
    out = []
    prev = 1
    for l in range(4):
        out.append((f"e{l + 1}a", (3, 3, c[l], prev), (c[l],)))
        out.append((f"e{l + 1}b", (3, 3, c[l], c[l]), (c[l],)))
        prev = c[l]
    for l in (2, 1, 0):
        out.append((f"d{l + 1}a", (3, 3, c[l], prev + c[l]), (c[l],)))
        out.append((f"d{l + 1}b", (3, 3, c[l], c[l]), (c[l],)))
        prev = c[l]
    out.append(("out", (1, 1, 1, c[0]), (1,)))
    return out


def flatten(params, base=32):
    """dict name.w / name.b -> flat FP32 vector."""
    parts = []
    for name, ws, bs in layer_shapes(base):
        parts.append(np.asarray(params[name + ".w"], np.float64).reshape(ws).ravel())
        parts.append(np.asarray(params[name + ".b"], np.float64).reshape(bs).ravel())
    return np.concatenate(parts).astype(np.float32)


def he_normal(seed, base=32):
    """Initial parameters as one flat FP32 vector: He-normal 3x3 weights (std sqrt(2 / fan_in)),
    std sqrt(1 / fan_in) for the 1x1 output layer, zero biases; seeded, in layer_shapes order."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, ws, bs in layer_shapes(base):
        k, _, cout, cin = ws
        fan_in = cin * k * k
        std = np.sqrt((1.0 if name == "out" else 2.0) / fan_in)
        parts.append((rng.standard_normal(ws) * std).ravel())
        parts.append(np.zeros(bs).ravel())
    return np.concatenate(parts).astype(np.float32)


def unflatten(vec, base=32):
    out, off = {}, 0
    for name, ws, bs in layer_shapes(base):
        nw, nb = int(np.prod(ws)), int(np.prod(bs))
        out[name + ".w"] = vec[off:off + nw].reshape(ws)
        off += nw
        out[name + ".b"] = vec[off:off + nb].reshape(bs)
        off += nb
    return out


class UNet:
    def __init__(self, base=32, max_n=4, max_h=512, max_w=256, device=0):
        self.lib = load()
        self.base = base
        h = ctypes.c_void_p()
        rc = self.lib.ds2d_unet_create(base, max_n, max_h, max_w, device, ctypes.byref(h))
        if rc:
            raise DS2DError(rc, self.lib.ds2d_unet_last_error(None).decode())
        self.h = h
        self.n = int(self.lib.ds2d_unet_num_params(self.h))

    def close(self):
        if self.h:
            self.lib.ds2d_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            raise DS2DError(rc, self.lib.ds2d_unet_last_error(self.h).decode())

    def set_option(self, key, value):
        """"tcgen05": 1 = 3x3 convolutions on tcgen05 / TMEM, 0 = mma.sync; "tcgen05_wgrad": 0
        keeps the weight gradient on mma.sync; "tcgen05_tma": 1 = convolution operands by tiled
        bulk-tensor loads through a ring of "tcgen05_stages" (2 or 3) stages, 0 = staged by the
        threads; "tcgen05_rows": output rows per CTA (1, 2 or 4); "tcgen05_wgrad_tma": 1 = weight-gradient operands MN-major by bulk-tensor boxes,
        0 = transposed through the threads."""
        self._check(self.lib.ds2d_unet_set_option(self.h, key.encode(), int(value)))

    def set_stream(self, stream_handle):
        self._check(self.lib.ds2d_unet_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def set_params(self, vec):
        v = np.ascontiguousarray(vec, np.float32)
        self._check(self.lib.ds2d_unet_set_params(
            self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), v.size))

    def get_params(self):
        v = np.zeros(self.n, np.float32)
        self._check(self.lib.ds2d_unet_get_params(
            self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), v.size))
        return v

    def forward(self, x_ptr, y_ptr, n, h, w):
        """y = net(x) on device pointers (FP32 [n][h][w])."""
        self._check(self.lib.ds2d_unet_forward(self.h, ctypes.c_void_p(x_ptr),
                                               ctypes.c_void_p(y_ptr), n, h, w))

    def loss_grad(self, x_ptr, t_ptr, n, h, w, want_grads=False):
        loss = ctypes.c_double(0.0)
        g = np.zeros(self.n, np.float32) if want_grads else None
        gp = g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if want_grads else None
        self._check(self.lib.ds2d_unet_loss_grad(self.h, ctypes.c_void_p(x_ptr),
                                                 ctypes.c_void_p(t_ptr), n, h, w,
                                                 ctypes.byref(loss), gp))
        return (loss.value, g) if want_grads else loss.value

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self._check(self.lib.ds2d_unet_adam_step(self.h, lr, beta1, beta2, eps))

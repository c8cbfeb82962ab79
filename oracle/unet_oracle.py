"""FP64 numpy oracle of the image-domain U-Net preconditioner (test infrastructure only).

The reference has no learned component: this network is the project's own extension (an
approximate inverse Hessian mapping an RTM image to reflectivity).  This file is the ground truth
its sm_100a BF16 tensor-core kernels are checked against: forward activations, the loss, and the
gradient of every parameter (the oracle's gradients are in turn pinned by finite differences in
the CPU test suite).

Network (all tensors NHWC, channels last):
  encoder  level l = 1..4 with C = 32, 64, 128, 256:  conv3x3 -> ReLU -> conv3x3 -> ReLU
           (levels 1-3 keep the result as a skip, then 2x2 average pooling)
  decoder  level l = 3..1: nearest 2x upsampling, concat [upsampled, skip_l] on channels,
           conv3x3 -> ReLU -> conv3x3 -> ReLU
  output   1x1 convolution 32 -> 1 (no activation)
Every convolution has a bias; 3x3 convolutions are 'same' with zero padding.  Weights are stored
as W[ky][kx][cout][cin] (the layout the CUDA kernels read).
"""
import numpy as np

LEVELS = (32, 64, 128, 256)


def layer_specs(base=32, cin=1):
    """(name, cin, cout, k) of every convolution in execution order."""
    c = [base, 2 * base, 4 * base, 8 * base]
    specs = []
    prev = cin
    for l in range(4):
        specs.append((f"e{l + 1}a", prev, c[l], 3))
        specs.append((f"e{l + 1}b", c[l], c[l], 3))
        prev = c[l]
    for l in (2, 1, 0):
        specs.append((f"d{l + 1}a", prev + c[l], c[l], 3))
        specs.append((f"d{l + 1}b", c[l], c[l], 3))
        prev = c[l]
    specs.append(("out", c[0], 1, 1))
    return specs


def init_params(seed, base=32, cin=1):
    """He-normal weights, zero biases (FP64)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, ci, co, k in layer_specs(base, cin):
        std = np.sqrt(2.0 / (ci * k * k)) if name != "out" else np.sqrt(1.0 / ci)
        p[name + ".w"] = rng.standard_normal((k, k, co, ci)) * std
        p[name + ".b"] = np.zeros(co)
    return p


def conv(x, w, b):
    """'same' convolution, x [N][H][W][Ci], w [k][k][Co][Ci] -> [N][H][W][Co]."""
    k = w.shape[0]
    r = k // 2
    n, h, wd, ci = x.shape
    xp = np.pad(x, ((0, 0), (r, r), (r, r), (0, 0)))
    y = np.zeros((n, h, wd, w.shape[2])) + b
    for ky in range(k):
        for kx in range(k):
            y += np.einsum("nhwc,oc->nhwo", xp[:, ky:ky + h, kx:kx + wd, :], w[ky, kx])
    return y


def conv_grads(x, w, dy):
    """Gradients of conv(x, w, b) given dy: (dx, dw, db)."""
    k = w.shape[0]
    r = k // 2
    n, h, wd, ci = x.shape
    xp = np.pad(x, ((0, 0), (r, r), (r, r), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ky in range(k):
        for kx in range(k):
            dw[ky, kx] = np.einsum("nhwo,nhwc->oc", dy, xp[:, ky:ky + h, kx:kx + wd, :])
            dxp[:, ky:ky + h, kx:kx + wd, :] += np.einsum("nhwo,oc->nhwc", dy, w[ky, kx])
    dx = dxp[:, r:r + h, r:r + wd, :]
    return dx, dw, dy.sum(axis=(0, 1, 2))


def pool(x):
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def pool_grad(dy):
    return np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_grad(dy):
    n, h, w, c = dy.shape
    return dy.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


def forward(p, x, base=32):
    """x [N][H][W][1] -> (y [N][H][W][1], cache)."""
    specs = {s[0]: s for s in layer_specs(base, x.shape[3])}
    cache = {}

    def cv(name, inp, relu=True):
        z = conv(inp, p[name + ".w"], p[name + ".b"])
        cache[name] = (inp, z)
        return np.maximum(z, 0.0) if relu else z

    skips = []
    h = x
    for l in range(4):
        h = cv(f"e{l + 1}a", h)
        h = cv(f"e{l + 1}b", h)
        if l < 3:
            skips.append(h)
            h = pool(h)
    for l in (2, 1, 0):
        h = np.concatenate([up(h), skips[l]], axis=3)
        h = cv(f"d{l + 1}a", h)
        h = cv(f"d{l + 1}b", h)
    y = cv("out", h, relu=False)
    del specs
    return y, cache


def loss_and_grads(p, x, target, base=32):
    """Mean-squared error over all pixels and its gradient for every parameter."""
    y, cache = forward(p, x, base)
    diff = y - target
    loss = float(np.mean(diff ** 2))
    dy = 2.0 * diff / diff.size
    g = {}

    def back(name, dout, relu=True):
        inp, z = cache[name]
        if relu:
            dout = dout * (z > 0)
        dx, dw, db = conv_grads(inp, p[name + ".w"], dout)
        g[name + ".w"] = dw
        g[name + ".b"] = db
        return dx

    c = [base, 2 * base, 4 * base, 8 * base]
    dh = back("out", dy, relu=False)
    dskips = [None, None, None]
    for l in (0, 1, 2):
        dh = back(f"d{l + 1}b", dh)
        dh = back(f"d{l + 1}a", dh)
        cup = dh.shape[3] - c[l]
        dskips[l] = dh[..., cup:]
        dh = up_grad(dh[..., :cup])
    for l in (3, 2, 1, 0):
        if l < 3:
            dh = pool_grad(dh) + dskips[l]
        dh = back(f"e{l + 1}b", dh)
        dh = back(f"e{l + 1}a", dh)
    return loss, g, y

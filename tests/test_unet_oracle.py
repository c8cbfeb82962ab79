"""Pins the FP64 U-Net oracle: its analytic gradients against central finite differences, and the
flat parameter layout shared with the C ABI."""
import numpy as np

from ds2d_b200.unet import flatten, layer_shapes, unflatten
from oracle import unet_oracle as uo


def test_oracle_gradients_match_finite_differences():
    base = 4
    p = uo.init_params(0, base=base)
    rng = np.random.default_rng(1)
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.standard_normal(p[k].shape) * 0.05
    x = rng.standard_normal((2, 16, 8, 1))
    t = rng.standard_normal((2, 16, 8, 1))
    _, g, _ = uo.loss_and_grads(p, x, t, base=base)
    checked = 0
    for name in sorted(p):
        a = p[name]
        for _ in range(2):
            idx = tuple(int(rng.integers(0, s)) for s in a.shape)
            old = a[idx]
            h = 1e-6
            a[idx] = old + h
            lp = uo.loss_and_grads(p, x, t, base=base)[0]
            a[idx] = old - h
            lm = uo.loss_and_grads(p, x, t, base=base)[0]
            a[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(g[name][idx] - fd) <= 1e-6 * max(1e-3, abs(fd)), (name, idx, g[name][idx], fd)
            checked += 1
    assert checked == 2 * len(p)


def test_flat_parameter_layout_round_trips():
    p = uo.init_params(3)
    v = flatten(p)
    assert v.size == sum(int(np.prod(ws)) + int(np.prod(bs)) for _, ws, bs in layer_shapes())
    q = unflatten(v)
    for k in p:
        np.testing.assert_allclose(q[k], p[k], rtol=1e-6, atol=1e-7)
    names = [s[0] for s in uo.layer_specs()]
    assert names == [s[0] for s in layer_shapes()]

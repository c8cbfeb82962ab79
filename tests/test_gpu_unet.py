"""U-Net preconditioner kernels (BF16 tensor cores, FP32 accumulate) against the FP64 oracle.

Tolerances follow from BF16 storage of activations, weights and activation gradients (8-bit
significand, relative rounding 2^-9 = 2e-3 per value) compounded through 15 convolution layers:
the forward output and the gradients are gated at a few percent relative L2."""
import numpy as np
import pytest

from oracle import unet_oracle as uo
from tests.helpers import rel

pytestmark = pytest.mark.gpu

FWD_GATE = 3e-2
GRAD_GATE_TOTAL = 5e-2
GRAD_GATE_LAYER = 1.5e-1


def _case(n=2, h=32, w=64, seed=0):
    rng = np.random.default_rng(seed)
    p = uo.init_params(seed)
    for k in p:  # non-zero biases so their paths are exercised
        if k.endswith(".b"):
            p[k] = rng.standard_normal(p[k].shape) * 0.05
    x = rng.standard_normal((n, h, w, 1))
    t = rng.standard_normal((n, h, w, 1)) * 0.5
    return p, x, t


@pytest.mark.parametrize("tcgen05", [0, 1])
def test_unet_forward_matches_oracle(cuda_device, tcgen05):
    import torch
    from ds2d_b200.unet import UNet, flatten
    p, x, t = _case()
    n, h, w = x.shape[:3]
    want, _ = uo.forward(p, x)
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_option("tcgen05", tcgen05)
        net.set_params(flatten(p))
        dx = torch.from_numpy(x[..., 0].astype(np.float32)).cuda()
        dy = torch.zeros_like(dx)
        net.forward(dx.data_ptr(), dy.data_ptr(), n, h, w)
        torch.cuda.synchronize()
        got = dy.cpu().numpy()
        # same parameters back
        np.testing.assert_array_equal(net.get_params(), flatten(p))
    assert rel(got, want[..., 0]) < FWD_GATE, rel(got, want[..., 0])


@pytest.mark.parametrize("tcgen05", [0, 1])
def test_unet_gradients_match_oracle(cuda_device, tcgen05):
    import torch
    from ds2d_b200.unet import UNet, flatten, unflatten
    p, x, t = _case(seed=1)
    n, h, w = x.shape[:3]
    loss_want, g_want, _ = uo.loss_and_grads(p, x, t)
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_option("tcgen05", tcgen05)
        net.set_params(flatten(p))
        dx = torch.from_numpy(x[..., 0].astype(np.float32)).cuda()
        dt = torch.from_numpy(t[..., 0].astype(np.float32)).cuda()
        loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w, want_grads=True)
    assert abs(loss - loss_want) <= 2e-2 * loss_want, (loss, loss_want)
    gw = flatten(g_want)
    assert rel(g, gw) < GRAD_GATE_TOTAL, rel(g, gw)
    got = unflatten(g)
    for k, v in g_want.items():
        if np.linalg.norm(v) > 0:
            assert rel(got[k], v) < GRAD_GATE_LAYER, (k, rel(got[k], v))


def test_unet_adam_training_reduces_loss(cuda_device):
    import torch
    from ds2d_b200.unet import UNet, flatten
    p, x, _ = _case(seed=2)
    n, h, w = x.shape[:3]
    # learn a fixed smoothing of the input: reachable by the network
    t = 0.5 * (x + np.roll(x, 1, axis=1))
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        dx = torch.from_numpy(x[..., 0].astype(np.float32)).cuda()
        dt = torch.from_numpy(t[..., 0].astype(np.float32)).cuda()
        first = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
        for _ in range(60):
            net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
            net.adam_step(lr=1e-3)
        last = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    assert last < 0.3 * first, (first, last)


def test_unet_tcgen05_and_mma_sync_agree_on_a_wide_image(cuda_device):
    """Rows wider than one 128-pixel tensor-core tile, several channel groups: the two tensor-core
    paths give the same forward output up to FP32 summation order and BF16 rounding."""
    import torch
    from ds2d_b200.unet import UNet, flatten
    p = uo.init_params(4)
    rng = np.random.default_rng(4)
    n, h, w = 2, 24, 200
    x = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    out = []
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        for tc in (0, 1):
            net.set_option("tcgen05", tc)
            y = torch.zeros_like(x)
            net.forward(x.data_ptr(), y.data_ptr(), n, h, w)
            torch.cuda.synchronize()
            out.append(y.cpu().numpy())
    assert rel(out[1], out[0]) < 1e-2, rel(out[1], out[0])


def test_unet_tcgen05_weight_gradients_agree_with_mma_sync(cuda_device):
    """The weight gradients of every layer from the tcgen05 kernel (64-pixel chunks split over
    CTAs, 128-channel tiles, TMEM accumulators) against the mma.sync kernel on a wide image, with
    the forward and backward-data products on tcgen05 in both runs: the two sum the same BF16
    products in FP32, so they agree up to summation order."""
    import torch
    from ds2d_b200.unet import UNet, flatten, unflatten
    p = uo.init_params(6)
    rng = np.random.default_rng(6)
    n, h, w = 2, 24, 200
    x = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32) * 0.5).cuda()
    grads = []
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        net.set_option("tcgen05", 1)
        net.set_option("tcgen05_wgrad_tma", 0)  # the kernel that transposes through the threads
        for tc in (0, 1):
            net.set_option("tcgen05_wgrad", tc)
            _, g = net.loss_grad(x.data_ptr(), t.data_ptr(), n, h, w, want_grads=True)
            grads.append(unflatten(g))
    for k, v in grads[0].items():
        if np.linalg.norm(v) > 0:
            assert rel(grads[1][k], v) < 1e-4, (k, rel(grads[1][k], v))


def test_unet_tcgen05_two_rows_per_cta_equal_one(cuda_device):
    """The tcgen05 convolution with two (or four) output rows per CTA (the staged weights of a chunk shared
    by both rows, one TMEM accumulator tile per row) against one row per CTA: every output sums
    the same products in the same order, so the forward pass agrees bit for bit, and the
    gradients up to the order of the weight gradient's split-K atomics; an odd row count at the
    coarsest level leaves its last CTA one row past the image."""
    import torch
    from ds2d_b200.unet import UNet, flatten
    p = uo.init_params(7)
    rng = np.random.default_rng(7)
    n, h, w = 2, 40, 200  # 40, 20, 10, 5 rows at the four levels
    x = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32) * 0.5).cuda()
    out, grads = [], []
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        net.set_option("tcgen05", 1)
        net.set_option("tcgen05_tma", 0)  # rows per CTA of the thread-staged kernel
        for rows in (1, 2, 4):
            net.set_option("tcgen05_rows", rows)
            y = torch.zeros_like(x)
            net.forward(x.data_ptr(), y.data_ptr(), n, h, w)
            torch.cuda.synchronize()
            out.append(y.cpu().numpy())
            _, g = net.loss_grad(x.data_ptr(), t.data_ptr(), n, h, w, want_grads=True)
            grads.append(g)
    for k in (1, 2):
        np.testing.assert_array_equal(out[k], out[0])
        assert rel(grads[k], grads[0]) < 1e-5, (k, rel(grads[k], grads[0]))


def test_unet_tcgen05_tma_pipeline_equals_staged(cuda_device):
    """The tcgen05 convolution fed by tiled bulk-tensor loads through a 3-stage mbarrier ring
    (option tcgen05_tma; the copy engine fills the pixels outside the image with zeros; two or
    four rows per CTA, two or three ring stages) against the same convolution staged by the
    threads: the same products summed in the same order, so
    the forward pass agrees bit for bit and the gradients up to the weight gradient's split-K
    atomics; then the pipelined network's gradients against the FP64 oracle."""
    import torch
    from ds2d_b200.unet import UNet, flatten, unflatten
    p = uo.init_params(8)
    rng = np.random.default_rng(8)
    n, h, w = 2, 40, 200
    x = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32) * 0.5).cuda()
    out, grads = [], []
    # (bulk-tensor loads, rows per CTA, ring stages): the thread-staged kernel first
    variants = ((0, 2, 3), (1, 2, 3), (1, 2, 2), (1, 4, 3), (1, 4, 2))
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        net.set_option("tcgen05", 1)
        for tma, rows, stages in variants:
            net.set_option("tcgen05_tma", tma)
            net.set_option("tcgen05_rows", rows)
            net.set_option("tcgen05_stages", stages)
            y = torch.zeros_like(x)
            net.forward(x.data_ptr(), y.data_ptr(), n, h, w)
            torch.cuda.synchronize()
            out.append(y.cpu().numpy())
            _, g = net.loss_grad(x.data_ptr(), t.data_ptr(), n, h, w, want_grads=True)
            grads.append(g)
    for k in range(1, len(variants)):
        np.testing.assert_array_equal(out[k], out[0], err_msg=str(variants[k]))
        assert rel(grads[k], grads[0]) < 1e-5, (variants[k], rel(grads[k], grads[0]))
    ps, xs, ts = _case(seed=9)
    ns, hs, ws = xs.shape[:3]
    _, g_want, _ = uo.loss_and_grads(ps, xs, ts)
    with UNet(max_n=ns, max_h=hs, max_w=ws) as net:
        net.set_option("tcgen05_tma", 1)
        net.set_params(flatten(ps))
        dx = torch.from_numpy(xs[..., 0].astype(np.float32)).cuda()
        dt = torch.from_numpy(ts[..., 0].astype(np.float32)).cuda()
        _, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), ns, hs, ws, want_grads=True)
    assert rel(g, flatten(g_want)) < GRAD_GATE_TOTAL, rel(g, flatten(g_want))


def test_unet_mn_major_weight_gradients_agree_with_mma_sync(cuda_device):
    """The weight and bias gradients of every layer from the tcgen05 kernel fed MN-major by tiled
    bulk-tensor boxes (option tcgen05_wgrad_tma: input-channel tiles of 16, 32, 64 and 128 over
    the network's layers, two 128-channel output tiles on the 256-channel layers, 64-pixel chunks
    with a ragged last one on the 200-pixel rows) against the mma.sync kernel: the same BF16
    products summed in FP32, equal up to summation order."""
    import torch
    from ds2d_b200.unet import UNet, flatten, unflatten
    p = uo.init_params(10)
    rng = np.random.default_rng(10)
    n, h, w = 2, 24, 200
    x = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((n, h, w)).astype(np.float32) * 0.5).cuda()
    grads = []
    with UNet(max_n=n, max_h=h, max_w=w) as net:
        net.set_params(flatten(p))
        net.set_option("tcgen05", 1)
        for tc, tma in ((0, 0), (1, 1)):
            net.set_option("tcgen05_wgrad", tc)
            net.set_option("tcgen05_wgrad_tma", tma)
            _, g = net.loss_grad(x.data_ptr(), t.data_ptr(), n, h, w, want_grads=True)
            grads.append(unflatten(g))
    for k, v in grads[0].items():
        if np.linalg.norm(v) > 0:
            assert rel(grads[1][k], v) < 1e-4, (k, rel(grads[1][k], v))

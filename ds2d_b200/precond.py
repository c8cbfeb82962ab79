"""Learned preconditioner for acoustic CG-LSRTM (no counterpart in the reference).

Pipeline, all on the GPU through this package's own kernels:
  1. training pairs: seeded random reflectivity m (sparse spikes, dipping reflectors, band-limited
     fields) on a smooth background -> Born data L m -> RTM image L^T L m (ds2d_ac_normal);
  2. training: the U-Net (ds2d_b200.unet, BF16 tensor-core kernels) learns image -> band-limited
     reflectivity on random crops of per-sample RMS-normalised pairs with Adam;
  3. application: ds2d_lsrtm_pcg with the trained network as the preconditioner P against the
     same call with P = I (plain CG), both judged by the relative Born-data residual.
"""
import time

import numpy as np

from . import synth


def background(allnx, allnz, vtop=1800.0, vbot=4500.0, seed=0, lateral=0.03, sigma=20.0):
    """Smooth vp increasing linearly with depth plus a smooth +-`lateral` lateral variation."""
    rng = np.random.default_rng(seed)
    z = np.linspace(0.0, 1.0, allnz)[None, :]
    vp = vtop + (vbot - vtop) * z + np.zeros((allnx, 1))
    pert = synth.smooth(rng.uniform(-1, 1, (allnx, allnz)).astype(np.float32), sigma)
    pert = pert / max(float(np.abs(pert).max()), 1e-12)
    return (vp * (1.0 + lateral * pert)).astype(np.float32)


def random_reflectivity(allnx, allnz, rng, density=0.05, amp=0.05, reflectors=4, top=8):
    """Sparse spikes (`density` of the cells, N(0, amp)) plus `reflectors` dipping reflector
    lines of random amplitude; zero in the top `top` rows (source and receiver depth)."""
    m = np.zeros((allnx, allnz), np.float32)
    mask = rng.random((allnx, allnz)) < density
    m[mask] = rng.normal(0.0, amp, int(mask.sum()))
    x = np.arange(allnx)
    for _ in range(reflectors):
        z0 = rng.uniform(top + 4, allnz - 4)
        dip = rng.uniform(-0.25, 0.25)
        zz = np.round(z0 + dip * (x - allnx / 2)).astype(int)
        ok = (zz >= top) & (zz < allnz)
        m[x[ok], zz[ok]] += rng.normal(0.0, 2 * amp)
    m[:, :top] = 0.0
    return m


def training_reflectivity(allnx, allnz, rng, top=8):
    """A varied training model: sparse spikes of random density, 0-6 dipping reflectors, and a
    band-limited random field of random scale, under a random depth trend of the amplitude.  The
    variety makes the network meet inputs like the CG gradients it preconditions later (the
    remaining error of an iterate is smoother and deeper than a fresh reflectivity)."""
    m = random_reflectivity(allnx, allnz, rng, density=rng.uniform(0.01, 0.08),
                            reflectors=int(rng.integers(0, 7)), top=top)
    if rng.random() < 0.7:
        field = synth.smooth(rng.standard_normal((allnx, allnz)).astype(np.float32),
                             rng.uniform(1.0, 6.0))
        field *= rng.uniform(0.2, 1.0) * 0.05 / max(float(field.std()), 1e-12)
        m += field
    z = np.linspace(0.0, 1.0, allnz)[None, :]
    m *= (1.0 + rng.uniform(-0.7, 2.0) * z).astype(np.float32)
    m[:, :top] = 0.0
    return m.astype(np.float32)


def make_pairs(ctx, shots, npairs, seed, device="cuda", log=None, generator=None):
    """(images, reflectivities) as torch FP32 tensors [npairs][allnx][allnz] on the device."""
    import torch
    rng = np.random.default_rng(seed)
    gen = generator or training_reflectivity
    nx, nz = ctx.allnx, ctx.allnz
    X = torch.zeros((npairs, nx, nz), dtype=torch.float32, device=device)
    Y = torch.zeros_like(X)
    t0 = time.perf_counter()
    for i in range(npairs):
        m = torch.from_numpy(gen(nx, nz, rng)).to(device)
        Y[i] = m
        ctx.ac_normal_device(shots, Y[i].data_ptr(), X[i].data_ptr())
        if log and (i + 1) % max(1, npairs // 8) == 0:
            log(f"pairs {i + 1}/{npairs} {time.perf_counter() - t0:.1f} s")
    return X, Y


def make_trajectory_pairs(ctx, shots, nmodels, iters, seed, device="cuda", log=None,
                          generator=None):
    """Training pairs along plain CG-LSRTM trajectories: for each seeded model m, run `iters`
    iterations of CGLS on d = L m and keep, at every iterate m_k, the pair (g_k = L^T (d - L m_k),
    e_k = m - m_k).  g_0 is the RTM image of m and e_0 = m itself; later pairs show the network the
    smoother, deeper, poorly illuminated errors that the CG leaves behind, i.e. the inputs it meets
    as a preconditioner.  Each iteration costs one L and one L^T, the price of one ordinary pair.
    Returns (g, e) as torch FP32 tensors [nmodels * iters][allnx][allnz]."""
    import torch
    rng = np.random.default_rng(seed)
    gen = generator or training_reflectivity
    nx, nz = ctx.allnx, ctx.allnz
    ntr = sum(s.ntr for s in shots)
    G = torch.zeros((nmodels * iters, nx, nz), dtype=torch.float32, device=device)
    E = torch.zeros_like(G)
    dz = torch.zeros((ntr, ctx.nt), dtype=torch.float32, device=device)
    dx = torch.zeros_like(dz)
    qz, qx = torch.zeros_like(dz), torch.zeros_like(dz)
    t0 = time.perf_counter()
    for j in range(nmodels):
        m_true = torch.from_numpy(gen(nx, nz, rng)).to(device)
        ctx.ac_born_device(shots, m_true.data_ptr(), dz.data_ptr(), dx.data_ptr())
        rz, rx = dz.clone(), dx.clone()
        m = torch.zeros_like(m_true)
        g = torch.zeros_like(m_true)
        ctx.ac_born_adj_device(shots, rz.data_ptr(), rx.data_ptr(), g.data_ptr())
        p = g.clone()
        gamma = float(g.double().pow(2).sum())
        for k in range(iters):
            G[j * iters + k] = g
            E[j * iters + k] = m_true - m
            if k + 1 == iters:
                break
            ctx.ac_born_device(shots, p.data_ptr(), qz.data_ptr(), qx.data_ptr())
            delta = float(qz.double().pow(2).sum() + qx.double().pow(2).sum())
            alpha = gamma / delta
            m += alpha * p
            rz -= alpha * qz
            rx -= alpha * qx
            ctx.ac_born_adj_device(shots, rz.data_ptr(), rx.data_ptr(), g.data_ptr())
            gnew = float(g.double().pow(2).sum())
            p = g + (gnew / gamma) * p
            gamma = gnew
        if log:
            log(f"trajectory {j + 1}/{nmodels} {time.perf_counter() - t0:.1f} s")
    return G, E


def normalise(t):
    """Per-sample RMS normalisation of a [n][h][w] tensor."""
    r = t.pow(2).mean(dim=(1, 2), keepdim=True).sqrt().clamp_min(1e-30)
    return t / r


def pad8(t):
    """Zero-pad the last two dims of [n][h][w] to multiples of 8 (the network's constraint)."""
    import torch.nn.functional as F
    h, w = t.shape[-2:]
    return F.pad(t, (0, (-w) % 8, 0, (-h) % 8))


def band_limit(Y, sigma=1.0):
    """Training target: the reflectivity smoothed by a Gaussian of `sigma` cells, i.e. the part of
    it a 15 Hz survey can resolve (the network is not asked to invent unrecoverable spikes)."""
    import torch
    import torch.nn.functional as F
    r = int(3 * sigma + 0.5)
    k = torch.exp(-0.5 * (torch.arange(-r, r + 1, dtype=torch.float32, device=Y.device) / sigma) ** 2)
    k = k / k.sum()
    y = Y[:, None]
    y = F.conv2d(F.pad(y, (0, 0, r, r), mode="reflect"), k.view(1, 1, -1, 1))
    y = F.conv2d(F.pad(y, (r, r, 0, 0), mode="reflect"), k.view(1, 1, 1, -1))
    return y[:, 0].contiguous()


def train(net, X, Y, steps=2000, batch=8, crop=(128, None), lr=1e-3, seed=0, log=None):
    """Adam on MSE(net(x), y) over random lateral crops (full depth by default, so the network
    sees where a feature sits between the surface and the bottom, and with random lateral flips)
    of the per-sample RMS-normalised pairs (x = image, y = band-limited reflectivity); the
    learning rate decays linearly to lr/10.  Returns the mean loss of every tenth of the run."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    Xn, Yn = normalise(X).contiguous(), normalise(band_limit(Y)).contiguous()
    n, h, w = Xn.shape
    ch = min(crop[0] or h, h) // 8 * 8
    cw = min(crop[1] or w, w) // 8 * 8
    xb = torch.empty((batch, ch, cw), dtype=torch.float32, device=X.device)
    yb = torch.empty_like(xb)
    hist, tot, cnt = [], 0.0, 0
    t0 = time.perf_counter()
    for step in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g)
        i0 = torch.randint(0, h - ch + 1, (batch,), generator=g)
        j0 = torch.randint(0, w - cw + 1, (batch,), generator=g)
        flip = torch.rand(batch, generator=g) < 0.5
        for b in range(batch):
            xs = Xn[idx[b], i0[b]:i0[b] + ch, j0[b]:j0[b] + cw]
            ys = Yn[idx[b], i0[b]:i0[b] + ch, j0[b]:j0[b] + cw]
            if flip[b]:
                xs, ys = xs.flip(0), ys.flip(0)
            xb[b].copy_(xs)
            yb[b].copy_(ys)
        tot += net.loss_grad(xb.data_ptr(), yb.data_ptr(), batch, ch, cw)
        cnt += 1
        net.adam_step(lr=lr * (1.0 - 0.9 * step / max(1, steps - 1)))
        if (step + 1) % max(1, steps // 10) == 0:
            hist.append(tot / cnt)
            if log:
                log(f"step {step + 1}/{steps} loss {hist[-1]:.4f} {time.perf_counter() - t0:.1f} s")
            tot, cnt = 0.0, 0
    return hist


def evaluate(net, X, Y):
    """Relative L2 error against the normalised band-limited reflectivity of (a) the network's estimate and
    (b) the best scalar multiple of the RTM image (the method without the network), both after
    an optimal scalar fit, averaged over the samples."""
    import torch
    Xn, Yn = pad8(normalise(X)).contiguous(), pad8(normalise(band_limit(Y))).contiguous()
    n, h, w = Xn.shape
    out = torch.zeros_like(Xn)
    for i in range(n):
        net.forward(Xn[i].data_ptr(), out[i].data_ptr(), 1, h, w)
    torch.cuda.synchronize()

    def fit_err(a, b):
        s = (a * b).sum() / (a * a).sum().clamp_min(1e-30)
        return float(((s * a - b).norm() / b.norm()).item())

    e_net = np.mean([fit_err(out[i], Yn[i]) for i in range(n)])
    e_rtm = np.mean([fit_err(Xn[i], Yn[i]) for i in range(n)])
    return {"net": e_net, "rtm": e_rtm}

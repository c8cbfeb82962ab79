"""Seeded synthetic models and acquisition geometry for the DS2D workloads.

No public dataset is involved: every workload here is a synthetic model generated from a seed
with the sizes and value ranges of the configuration it stands for.
"""
import numpy as np
from scipy.ndimage import gaussian_filter

from .api import ShotGeom


def ricker(nt, f0, dt):
    """Ricker wavelet as main.cpp:461-473 (ricker1): t0 = 1/f, kt = (int)(t0/dt)."""
    pi = np.float32(3.14159265358979)
    f = np.float32(f0)
    dtf = np.float32(dt)
    kt = int(np.float32(1) / f / dtf)
    i = np.arange(nt, dtype=np.float32)
    tt = (i * dtf - np.float32(kt) * dtf).astype(np.float32)
    sp = (pi * f * tt).astype(np.float32)
    sp2 = (-sp * sp).astype(np.float32)
    return (np.exp(sp2.astype(np.float64)) * (1.0 - 2.0 * sp.astype(np.float64) ** 2)).astype(np.float32)


def gardner(vp):
    """Gardner density, rho = 0.31 vp^0.25 g/cc, in kg/m^3."""
    return (310.0 * np.power(vp, 0.25)).astype(np.float32)


def layered(allnx, allnz, seed, layers=4, vmin=2500.0, vmax=5500.0, sigma=5.0, pert=0.05):
    """Flat layers vmin..vmax plus a Gaussian-smoothed +-pert uniform perturbation."""
    rng = np.random.default_rng(seed)
    z = np.arange(allnz)
    bounds = np.linspace(0, allnz, layers + 1)[1:-1]
    idx = np.searchsorted(bounds, z, side="right")
    vel = np.linspace(vmin, vmax, layers)[idx]
    vp = np.broadcast_to(vel, (allnx, allnz)).astype(np.float64)
    noise = gaussian_filter(rng.uniform(-1, 1, (allnx, allnz)), sigma)
    noise /= max(np.abs(noise).max(), 1e-12)
    vp = vp * (1.0 + pert * noise)
    vs = vp / 1.73
    return vp.astype(np.float32), vs.astype(np.float32)


def dipping_lenses(allnx, allnz, seed, layers=8, vmin=2000.0, vmax=6000.0, lenses=3):
    """Dipping layers vmin..vmax plus Gaussian lenses (true model of the RTM workload)."""
    rng = np.random.default_rng(seed)
    x = np.arange(allnx)[:, None].astype(np.float64)
    z = np.arange(allnz)[None, :].astype(np.float64)
    dip = rng.uniform(-0.08, 0.08)
    depth = z - dip * (x - allnx / 2)
    bounds = np.sort(rng.uniform(0.05, 0.95, layers - 1)) * allnz
    idx = np.searchsorted(bounds, depth.ravel(), side="right").reshape(depth.shape)
    vp = np.linspace(vmin, vmax, layers)[idx]
    for _ in range(lenses):
        cx, cz = rng.uniform(0.15, 0.85) * allnx, rng.uniform(0.25, 0.85) * allnz
        r = rng.uniform(0.03, 0.08) * allnx
        amp = rng.uniform(-0.12, 0.12)
        vp = vp * (1 + amp * np.exp(-((x - cx) ** 2 + (z - cz) ** 2) / (2 * r * r)))
    vp = np.clip(vp, vmin, vmax)
    vs = vp / 1.73
    return vp.astype(np.float32), vs.astype(np.float32)


def smooth(v, sigma):
    return gaussian_filter(v.astype(np.float64), sigma, mode="nearest").astype(np.float32)


def reflectivity(allnx, allnz, seed, density=0.05, std=0.05):
    """Sparse random reflectivity: `density` of the cells nonzero, N(0, std)."""
    rng = np.random.default_rng(seed)
    m = np.zeros((allnx, allnz), np.float32)
    mask = rng.uniform(size=m.shape) < density
    m[mask] = rng.normal(0, std, mask.sum())
    return m


def uneven_shots(allnx, pml, nshots, wmin, wmax, seed, sz=0, gz=2):
    """Shots with their own aperture: width ~ U[wmin, wmax] cells, centred on the source and
    clipped to the model, receivers on every column of the window (batched-uneven workload)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0, allnx - 1, nshots).round().astype(int)
    shots = []
    for sx in xs:
        w = int(min(rng.integers(wmin, wmax + 1), allnx))
        wl = int(np.clip(sx - w // 2, 0, allnx - w))
        igx = np.arange(pml, pml + w, dtype=np.int32)
        shots.append(ShotGeom(win_left=wl, isx=pml + int(sx - wl), isz=pml + sz, igz=pml + gz,
                              igx=igx, nx=w))
    return shots


def surface_shots(allnx, nx, pml, nshots, sz=0, gz=2, receivers_every=1, first=None, last=None):
    """Shots evenly spread along the surface, each with an nx-wide window centred on the source
    (clipped to the model), receivers on every `receivers_every`-th interior column at depth gz."""
    first = 0 if first is None else first
    last = allnx - 1 if last is None else last
    xs = np.linspace(first, last, nshots).round().astype(int) if nshots > 1 else np.array([(first + last) // 2])
    shots = []
    for sx in xs:
        wl = int(np.clip(sx - nx // 2, 0, allnx - nx))
        igx = np.arange(pml, pml + nx, receivers_every, dtype=np.int32)
        shots.append(ShotGeom(win_left=wl, isx=pml + int(sx - wl), isz=pml + sz, igz=pml + gz, igx=igx))
    return shots

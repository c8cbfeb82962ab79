"""Generates the golden fixtures of tests/golden/ by running the reference's own CUDA build
(oracle/_ref/libds2dref.so, built by oracle/build_ref.sh) on a GPU.

    python tests/golden/make_golden.py [outdir] [--only name,name...]

Each fixture is an .npz holding the inputs (model, wavelet, geometry, image, data) and the
reference outputs.  Sizes are small so that the CPU oracle replays every case in seconds, except
forward_c1.npz, which is the first benchmark configuration at its full size (251x101, 20-cell
PML, nt 2000; records of every fifth receiver are kept to bound the file).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ds2d_b200 import synth  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

# Small elastic case: 80 x 40 model, 64-wide windows, 10-cell PML, 400 steps of 0.8 ms.
CASE = dict(allnx=80, allnz=40, nx=64, pml=10, nt=400, dx=10.0, dz=10.0, dt=0.0008, f0=15.0)


def geometry():
    c = CASE
    return synth.surface_shots(c["allnx"], c["nx"], c["pml"], 2, sz=0, gz=2)


def models():
    c = CASE
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=11)
    vp_mig, vs_mig = synth.smooth(vp, 3.0), synth.smooth(vs, 3.0)
    return vp, vs, vp_mig, vs_mig


def shot_arrays(shots):
    return dict(win_left=np.array([s.win_left for s in shots], np.int32),
                isx=np.array([s.isx for s in shots], np.int32),
                isz=np.array([s.isz for s in shots], np.int32),
                igz=np.array([s.igz for s in shots], np.int32),
                igx=np.stack([s.igx for s in shots]).astype(np.int32))


# First benchmark configuration: plain elastic forward modelling, one shot at the surface centre.
C1 = dict(allnx=251, allnz=101, nx=251, pml=20, nt=2000, dx=10.0, dz=10.0, dt=0.0008, f0=15.0)
C1_TRACE_STEP = 5


def make_c1(outdir):
    """Config 1 at full size: 4 flat layers 2500-5500 m/s + smoothed 5 % perturbation, vs =
    vp / 1.73, rho = 2000 (the reference's), 15 Hz Ricker at (125, 0), receivers on every column
    at depth 2; the reference's PML forward modelling records vx and vz."""
    c = C1
    g = (c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=101)
    w = synth.ricker(c["nt"], c["f0"], c["dt"])
    shot = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 1, sz=0, gz=2)[0]
    rz, rx = po.ref_forward(*g, vp, vs, w, shot)
    keep = np.arange(0, shot.ntr, C1_TRACE_STEP)
    np.savez_compressed(os.path.join(outdir, "forward_c1.npz"), vp=vp, vs=vs, wavelet=w,
                        case=np.array([c[k] for k in ("allnx", "allnz", "nx", "pml", "nt")], np.int32),
                        steps=np.array([c["dx"], c["dz"], c["dt"], c["f0"]], np.float32),
                        traces=keep.astype(np.int32), rec_vz=rz[keep], rec_vx=rx[keep],
                        **shot_arrays([shot]))


def make_born(outdir):
    """First-order Born records by the reference's own born_modeling (mode 1), small case, two
    shots each: vs = 0 (the acoustic Born operator of the elastic scheme, mu = 0) with an injected
    random band and zero damping, and with the reference's PML; the elastic model with the PML."""
    c = CASE
    g = (c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    shots = geometry()
    vp, vs, vp_mig, vs_mig = models()
    w = synth.ricker(c["nt"], c["f0"], c["dt"])
    img_pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    img_ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    common = dict(case=np.array([c[k] for k in ("allnx", "allnz", "nx", "pml", "nt")], np.int32),
                  steps=np.array([c["dx"], c["dz"], c["dt"], c["f0"]], np.float32), wavelet=w,
                  img_pp=img_pp, **shot_arrays(shots))
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    # acoustic: vs = 0, band injected (seed 1234), the perturbation is img_pp only
    vs0 = np.zeros_like(vp_mig)
    zero = np.zeros_like(img_pp)
    pads = [po.build_model(st, vp_mig, vs0, None, s.win_left, rbc=1, seed=1234, shot_id=i)
            for i, s in enumerate(shots)]
    recs = [po.ref_born(*g, vp_mig, vs0, w, img_pp, zero, s, rbc=1, vp_pad=p[0], vs_pad=p[1])
            for s, p in zip(shots, pads)]
    np.savez_compressed(os.path.join(outdir, "born_acoustic_random.npz"), vp=vp_mig, vs=vs0,
                        seed=np.uint64(1234), vp_pad=np.stack([p[0] for p in pads]),
                        rec_vz=np.stack([r[0] for r in recs]), rec_vx=np.stack([r[1] for r in recs]),
                        **common)
    # acoustic with the reference's PML (vs = 0)
    recs = [po.ref_born(*g, vp_mig, vs0, w, img_pp, zero, s) for s in shots]
    np.savez_compressed(os.path.join(outdir, "born_acoustic_pml.npz"), vp=vp_mig, vs=vs0,
                        rec_vz=np.stack([r[0] for r in recs]), rec_vx=np.stack([r[1] for r in recs]),
                        **common)
    # elastic with PML, both perturbations
    recs = [po.ref_born(*g, vp_mig, vs_mig, w, img_pp, img_ps, s) for s in shots]
    np.savez_compressed(os.path.join(outdir, "born_elastic_pml.npz"), vp=vp_mig, vs=vs_mig,
                        img_ps=img_ps, rec_vz=np.stack([r[0] for r in recs]),
                        rec_vx=np.stack([r[1] for r in recs]), **common)


BANDPASS_CASES = [(80, 40, 0, 8), (81, 41, 3, 12), (121, 41, 0, 10)]  # nx, nz, z1, z2


def make_bandpass(outdir):
    """The reference's bandpass_filter (cuFFT) on seeded random images: even and odd sizes, the
    low-pass (z1 = 0) and band-pass forms."""
    rng = np.random.default_rng(41)
    out = {}
    for i, (nx, nz, z1, z2) in enumerate(BANDPASS_CASES):
        pp = rng.standard_normal((nx, nz)).astype(np.float32)
        ps = rng.standard_normal((nx, nz)).astype(np.float32)
        fpp, fps = po.ref_bandpass(pp, ps, z1, z2)
        out.update({f"in_pp{i}": pp, f"in_ps{i}": ps, f"out_pp{i}": fpp, f"out_ps{i}": fps})
    np.savez_compressed(os.path.join(outdir, "bandpass.npz"),
                        cases=np.array(BANDPASS_CASES, np.int32), **out)


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    c = CASE
    g = (c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    shots = geometry()
    vp, vs, vp_mig, vs_mig = models()
    w = synth.ricker(c["nt"], c["f0"], c["dt"])
    common = dict(case=np.array([c[k] for k in ("allnx", "allnz", "nx", "pml", "nt")], np.int32),
                  steps=np.array([c["dx"], c["dz"], c["dt"], c["f0"]], np.float32), wavelet=w,
                  **shot_arrays(shots))

    # 1. background forward modelling on the true model (observed data), both shots.
    obs = [po.ref_forward(*g, vp, vs, w, s) for s in shots]
    np.savez_compressed(os.path.join(outdir, "forward_pml.npz"), vp=vp, vs=vs,
                        rec_vz=np.stack([o[0] for o in obs]), rec_vx=np.stack([o[1] for o in obs]),
                        **common)
    obs_vz = np.stack([o[0] for o in obs])
    obs_vx = np.stack([o[1] for o in obs])

    # 2. reference-mode ELSRTM on the migration model, iterations 0 and 1, shot 0.
    img_pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    img_ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    for it in (0, 1):
        r = po.ref_elsrtm(*g, vp_mig, vs_mig, w, img_pp, img_ps, shots[0], obs_vz[0], obs_vx[0], it)
        np.savez_compressed(os.path.join(outdir, f"elsrtm_iter{it}.npz"), vp=vp_mig, vs=vs_mig,
                            img_pp=img_pp, img_ps=img_ps, obs_vz=obs_vz[0], obs_vx=obs_vx[0],
                            iteration=np.int32(it), res_vz=r["res_vz"], res_vx=r["res_vx"],
                            images=np.stack(r["images"]), misfit=np.float64(r["misfit"]),
                            **common)

    # 3. RTM with boundary strips (PML) and with an injected random band, two shots each.
    for rbc in (0, 1):
        vp_pad = vs_pad = None
        extra = {}
        if rbc:
            st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
            pads = [po.build_model(st, vp_mig, vs_mig, None, s.win_left, rbc=1, seed=1234,
                                   shot_id=i) for i, s in enumerate(shots)]
            vp_pad = np.stack([p[0] for p in pads])
            vs_pad = np.stack([p[1] for p in pads])
            extra = dict(vp_pad=vp_pad, vs_pad=vs_pad, seed=np.uint64(1234))
        imgs, ms = po.ref_rtm(*g, vp_mig, vs_mig, w, shots, obs_vz, obs_vx, rbc=rbc,
                              vp_pad=vp_pad, vs_pad=vs_pad)
        name = "rtm_random.npz" if rbc else "rtm_pml.npz"
        np.savez_compressed(os.path.join(outdir, name), vp=vp_mig, vs=vs_mig, adj_vz=obs_vz,
                            adj_vx=obs_vx, images=np.stack(imgs), rbc=np.int32(rbc), **extra,
                            **common)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only")]
    only = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
    out = args[0] if args else os.path.dirname(os.path.abspath(__file__))
    makers = {"base": main, "c1": make_c1, "born": make_born, "bandpass": make_bandpass}
    for name in (only.split(",") if only else list(makers)):
        makers[name](out)
    print("golden fixtures written to", out)

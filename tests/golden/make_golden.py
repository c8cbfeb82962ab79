"""Generates the golden fixtures of tests/golden/ by running the reference's own CUDA build
(oracle/_ref/libds2dref.so, built by oracle/build_ref.sh) on a GPU.

    python tests/golden/make_golden.py [outdir]

Each fixture is an .npz holding the inputs (model, wavelet, geometry, image, data) and the
reference outputs.  Sizes are small so that the CPU oracle replays every case in seconds.
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
    print("golden fixtures written to", outdir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))

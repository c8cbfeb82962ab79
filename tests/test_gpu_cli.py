"""The C++ host driver (ds2d_b200/ds2d_elsrtm) on a parameters file and SU gathers, end to end,
against the same iterations driven through the Python API."""
import os
import subprocess

import numpy as np
import pytest

from ds2d_b200 import Elastic2D, ShotGeom, synth
from ds2d_b200.su import read_su, write_su
from tests.helpers import rel

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ds2d_b200",
                   "ds2d_elsrtm")


def test_cli_matches_api(cuda_device, tmp_path):
    allnx, allnz, pml, nt, dx, dt, f0 = 60, 30, 10, 250, 10.0, 0.0006, 15.0
    nshot, sy, gy = 3, 0, 2
    vp, vs = synth.layered(allnx, allnz, seed=7)
    vpm, vsm = synth.smooth(vp, 2.0), synth.smooth(vs, 2.0)
    # every shot records on all columns: window = whole model, source positions in metres
    sxs = [10 * int(x) for x in np.linspace(5, allnx - 6, nshot).round()]
    shots = [ShotGeom(0, pml + sx // 10, pml + sy, pml + gy, np.arange(pml, pml + allnx, dtype=np.int32))
             for sx in sxs]
    w = synth.ricker(nt, f0, dt)
    with Elastic2D(allnx, allnz, allnx, pml, nt, dx, dx, dt, max_shots=nshot, max_ntr=allnx) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward(shots)
    gx = np.tile(np.arange(allnx) * 10, nshot)
    sx = np.repeat(sxs, allnx)
    write_su(tmp_path / "vz.su", oz, sx, gx, dt)
    write_su(tmp_path / "vx.su", ox, sx, gx, dt)
    d2, sx2, gx2, dt2 = read_su(tmp_path / "vz.su")
    np.testing.assert_array_equal(d2, oz)
    assert dt2 == pytest.approx(dt)
    vpm.tofile(tmp_path / "vp.bin")
    vsm.tofile(tmp_path / "vs.bin")
    maxiter = 2
    (tmp_path / "parameters").write_text(
        f"{dx:g} {dx:g} {pml} {allnx} {allnz} 1 {nshot}\n./vp.bin\n./vs.bin\n./vz.su\n./vx.su\n"
        f"./image\n{f0:g} {maxiter}\n{sy} {gy}\n1 0 0 1000\n")
    r = subprocess.run([BIN, "parameters", "max_shots=2"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    # Same iterations through the Python API: ELSRTM + the Adam-like update of main.cpp:1092-1131.
    pp = np.zeros((allnx, allnz), np.float32)
    ps = np.zeros((allnx, allnz), np.float32)
    f32 = np.float32
    b1, b2, al, eps, ga = f32(0.8), f32(0.999), f32(3e-5), f32(5e8), f32(0.99)
    sp = np.zeros_like(pp); ss = np.zeros_like(pp); rp = np.zeros_like(pp); rs = np.zeros_like(pp)
    with Elastic2D(allnx, allnz, allnx, pml, nt, dx, dx, dt, max_shots=nshot, max_ntr=allnx) as e:
        e.set_models(vpm, vsm)
        e.set_wavelet(w)
        for it in range(maxiter):
            e.set_image(pp, ps)
            e.elsrtm(shots, oz, ox, it)
            g = e.read_images()
            ak = al if it == 0 else f32((al / 2) * np.float64(ga) ** it)
            gp = g["pp_grad"] + g["b_pp"] + g["b_pp2"]
            gs = g["ps_grad"] + g["b_ps"] + g["b_ps2"]
            sp = b1 * sp + (1 - b1) * gp
            ss = b1 * ss + (1 - b1) * gs
            rp = b2 * rp + (1 - b2) * (gp * gp)
            rs = b2 * rs + (1 - b2) * (gs * gs)
            k = it + 1
            mp = (sp / (1 - np.float64(b1) ** k)).astype(f32)
            ms = (ss / (1 - np.float64(b1) ** k)).astype(f32)
            vpk = (rp / (1 - np.float64(b2) ** k)).astype(f32)
            vsk = (rs / (1 - np.float64(b2) ** k)).astype(f32)
            pp = pp - ak * (mp / (np.sqrt(vpk) + eps))
            ps = ps - ak * (ms / (np.sqrt(vsk) + eps))
            got = np.fromfile(tmp_path / "image" / f"sum_image_pp_{it}_{allnx}_{allnz}.dat", np.float32)
            assert rel(got.reshape(allnx, allnz), pp) < 1e-4
            gotg = np.fromfile(tmp_path / "image" / f"all_grad_pp_{it}_{allnx}_{allnz}.dat", np.float32)
            assert rel(gotg.reshape(allnx, allnz), gp) < 1e-5
    assert len((tmp_path / "image" / "misfit.txt").read_text().splitlines()) == maxiter

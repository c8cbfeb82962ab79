"""Time-blocked forward launches (k_fwd_tb: several time steps per launch, random boundary)
against the one-step ring kernels and the FP64 oracle, through the C ABI."""
import numpy as np
import pytest

from ds2d_b200 import Elastic2D, synth
from oracle import pyoracle as po
from tests.helpers import GATE, gate, rel, small_case

pytestmark = pytest.mark.gpu

# The time-blocked kernel evaluates every stage with the one-step kernel's expressions; its
# receiver records agree with k_fwd_ring's to FP32 rounding of the same sums.
TB_GATE = 1e-6


def _run(c, shots, vp, vs, w, obs, **opts):
    with Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="random", seed=5, max_shots=len(shots),
                   max_ntr=max(s.ntr for s in shots)) as e:
        for k, v in opts.items():
            e.set_option(k, v)
        e.set_models(vp, vs)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
        e.rtm(shots, obs[0], obs[1])
        return rz, rx, e.read_images()


def _case(allnz, nt):
    c, _, _, w, _ = small_case(nt=nt)
    c["allnz"] = allnz
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=4)
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    rng = np.random.default_rng(7)
    ntr = sum(s.ntr for s in shots)
    obs = (rng.normal(size=(ntr, nt)).astype(np.float32) * 1e-3,
           rng.normal(size=(ntr, nt)).astype(np.float32) * 1e-3)
    return c, vp, vs, w, shots, obs


# (depth, CTA width, rows per CTA, model depth, operand rows by bulk copy): 320 padded rows give
# 256-thread CTAs two z-strips (one inner edge each), 460 give depth 3-4 three strips (an inner
# strip with two halos), 512 threads cover the 320 rows in one strip; xr 24 gives each shot
# several row blocks.  nt 203 is no multiple of the depth, so the last block of a pass is shorter.
# Depth 1-2 run with bulk-copied operand rows (the default) and with per-thread cp.async; depth
# 3-4 have only the latter.
CASES = [(1, 256, 0, 300, 1), (2, 256, 24, 300, 1), (3, 256, 24, 300, 0), (4, 256, 0, 300, 0),
         (1, 512, 24, 300, 1), (2, 512, 0, 300, 1), (3, 256, 24, 440, 0), (4, 256, 24, 440, 0),
         (1, 256, 24, 300, 0), (2, 256, 0, 300, 0), (2, 512, 24, 300, 0), (2, 256, 24, 440, 1)]


_FLOOR = {}


def _image_floor(c, vp, vs, w, shots, obs):
    """FP32 floor of the RTM images on this case: the oracle's FP32 replay against its FP64 one
    (the reconstruction from the final state carries every rounding difference of the forward
    pass into the images, so kernels with different FMA contractions agree only to this floor)."""
    if c["allnz"] not in _FLOOR:
        st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
        ntr = shots[0].ntr
        tot = {p: np.zeros((3, c["allnx"], c["allnz"])) for p in ("f32", "f64")}
        for i, s in enumerate(shots):
            m = po.build_model(st, vp, vs, None, s.win_left, rbc=1, seed=5, shot_id=i)
            sl = slice(i * ntr, (i + 1) * ntr)
            for p in tot:
                o = po.rtm(st, m, w, s, obs[0][sl], obs[1][sl], 1, p)
                for k in range(3):
                    tot[p][k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
        _FLOOR[c["allnz"]] = [rel(tot["f32"][k], tot["f64"][k]) for k in range(3)]
    return _FLOOR[c["allnz"]]


@pytest.mark.parametrize("depth,cta,xr,allnz,bulk", CASES)
def test_time_blocked_forward_matches_one_step(cuda_device, depth, cta, xr, allnz, bulk):
    """Receiver records of the forward modelling (to 1e-6) and the RTM images (to the FP32 floor
    of the images) with the forward pass on the time-blocked kernel against the one-step ring
    kernels."""
    c, vp, vs, w, shots, obs = _case(allnz, nt=203)
    ref = _run(c, shots, vp, vs, w, obs, tb=0, pair=0)
    got = _run(c, shots, vp, vs, w, obs, tb=depth, tb_cta=cta, pair_xr=xr, tb_bulk=bulk)
    assert np.abs(got[0]).max() > 0
    for j in range(2):
        err = rel(got[j], ref[j])
        assert err < TB_GATE, (j, err, "bit-identical" if np.array_equal(got[j], ref[j]) else "")
    floor = _image_floor(c, vp, vs, w, shots, obs)
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        err = rel(got[2][key], ref[2][key])
        assert err < gate(floor[k]), (key, err, f"FP32 floor {floor[k]:.3e}")


def test_time_blocked_uneven_windows_vs_oracle(cuda_device):
    """Shots of different aperture in one batch, two time steps per launch, against the FP64
    oracle's forward records."""
    c, vp, vs, w, _ = small_case(nt=150)
    shots = synth.uneven_shots(c["allnx"], c["pml"], 4, 20, c["allnx"], seed=9)
    wmax = max(s.nx for s in shots)
    with Elastic2D(c["allnx"], c["allnz"], wmax, c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="random", seed=8, max_shots=len(shots), max_ntr=wmax) as e:
        e.set_option("tb", 2)
        e.set_option("pair_xr", 16)
        e.set_models(vp, vs)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
    off = 0
    for i, s in enumerate(shots):
        st = po.Setup(c["allnx"], c["allnz"], s.nx, c["pml"], c["dx"], c["dz"], c["dt"])
        m = po.build_model(st, vp, vs, None, s.win_left, rbc=1, seed=8, shot_id=i)
        oz, ox = po.forward(st, m, w, s, "f64")
        assert rel(rz[off:off + s.ntr], oz) < GATE, (i, rel(rz[off:off + s.ntr], oz))
        assert rel(rx[off:off + s.ntr], ox) < GATE, (i, rel(rx[off:off + s.ntr], ox))
        off += s.ntr

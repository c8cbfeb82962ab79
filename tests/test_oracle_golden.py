"""Pins the CPU oracle against the reference's own CUDA build: every golden fixture in
tests/golden/ (made by tests/golden/make_golden.py on a B200) is replayed by the oracle in FP64
and FP32 on the same inputs."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import case_of, gate, load, rel, shots_of


def _setup(fx):
    c = case_of(fx)
    return c, po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])


def _need(name):
    fx = load(name)
    if fx is None:
        pytest.fail(f"golden fixture {name} missing (run tests/golden/make_golden.py on a GPU)")
    return fx


def test_forward_golden():
    fx = _need("forward_pml.npz")
    c, st = _setup(fx)
    for i, s in enumerate(shots_of(fx)):
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
        rz, rx = po.forward(st, m, fx["wavelet"], s, "f64")
        assert rel(fx["rec_vz"][i], rz) < gate() and rel(fx["rec_vx"][i], rx) < gate()


@pytest.mark.parametrize("it", [0, 1])
def test_elsrtm_golden(it):
    fx = _need(f"elsrtm_iter{it}.npz")
    c, st = _setup(fx)
    s = shots_of(fx)[0]
    m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
    dmp = po.window_image(st, fx["img_pp"], s.win_left)
    dms = po.window_image(st, fx["img_ps"], s.win_left)
    args = (st, m, dmp, dms, fx["wavelet"], s, fx["obs_vz"], fx["obs_vx"], it)
    r64 = po.elsrtm(*args, precision="f64")
    r32 = po.elsrtm(*args, precision="f32")
    for key in ("res_vz", "res_vx"):
        floor = rel(r32[key], r64[key])
        assert rel(fx[key], r64[key]) < gate(floor), key
    for k in range(7):
        full64 = po.place(r64["images"][k], c["allnx"], c["allnz"], s.win_left)
        full32 = po.place(r32["images"][k], c["allnx"], c["allnz"], s.win_left)
        floor = rel(full32, full64)
        assert rel(fx["images"][k], full64) < gate(floor), (k, rel(fx["images"][k], full64), floor)
    if it > 0:
        assert fx["misfit"] == pytest.approx(r64["misfit"], rel=1e-4)


@pytest.mark.parametrize("name", ["rtm_pml.npz", "rtm_random.npz"])
def test_rtm_golden(name):
    fx = _need(name)
    c, st = _setup(fx)
    rbc = int(fx["rbc"])
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    tot32 = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots_of(fx)):
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left, rbc=rbc,
                           seed=int(fx.get("seed", 0)), shot_id=i)
        if rbc:
            np.testing.assert_array_equal(m[0], fx["vp_pad"][i])
        for tot, prec in ((tot64, "f64"), (tot32, "f32")):
            imgs = po.rtm(st, m, fx["wavelet"], s, fx["adj_vz"][i], fx["adj_vx"][i], rbc, prec)
            for k in range(3):
                tot[k] += po.place(imgs[k], c["allnx"], c["allnz"], s.win_left)
    for k in range(3):
        floor = rel(tot32[k], tot64[k])
        assert rel(fx["images"][k], tot64[k]) < gate(floor), (k, rel(fx["images"][k], tot64[k]), floor)


def test_forward_c1_golden():
    """First benchmark configuration at full size (251x101, 20-cell PML, nt 2000): the FP64 oracle
    against the reference's records at every fifth receiver."""
    fx = _need("forward_c1.npz")
    c, st = _setup(fx)
    s = shots_of(fx)[0]
    m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
    rz, rx = po.forward(st, m, fx["wavelet"], s, "f64")
    keep = fx["traces"]
    ez, ex = rel(fx["rec_vz"], rz[keep]), rel(fx["rec_vx"], rx[keep])
    assert ez < gate() and ex < gate(), (ez, ex)


@pytest.mark.parametrize("name", ["born_acoustic_random.npz", "born_acoustic_pml.npz",
                                  "born_elastic_pml.npz"])
def test_born_golden(name):
    """First-order Born records of the reference's born_modeling (mode 1) against the oracle's
    restatement; for vs = 0 also against the acoustic Born oracle, which must be the same operator
    (mu = 0 removes every shear term of the elastic scheme)."""
    fx = _need(name)
    c, st = _setup(fx)
    acoustic = "acoustic" in name
    img_ps = np.zeros_like(fx["img_pp"]) if acoustic else fx["img_ps"]
    for i, s in enumerate(shots_of(fx)):
        rbc = 1 if "random" in name else 0
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left, rbc=rbc,
                           seed=int(fx.get("seed", 0)), shot_id=i)
        if rbc:
            np.testing.assert_array_equal(m[0], fx["vp_pad"][i])
        dmp = po.window_image(st, fx["img_pp"], s.win_left)
        dms = po.window_image(st, img_ps, s.win_left)
        b64 = po.born(st, m, dmp, dms, fx["wavelet"], s, "f64")
        b32 = po.born(st, m, dmp, dms, fx["wavelet"], s, "f32")
        for j in range(2):
            floor = rel(b32[j], b64[j])
            got = rel(fx["rec_vz" if j == 0 else "rec_vx"][i], b64[j])
            assert got < gate(floor), (i, j, got, floor)
        if acoustic:
            az, ax = po.ac_born(st, m, fx["wavelet"], s, dmp)
            assert rel(az, b64[0]) < 1e-10 and rel(ax, b64[1]) < 1e-10


def test_bandpass_golden():
    """The FP64 restatement of the reference's band-pass filter against its cuFFT results."""
    fx = _need("bandpass.npz")
    for i, (nx, nz, z1, z2) in enumerate(fx["cases"]):
        for key in ("pp", "ps"):
            got = po.bandpass(fx[f"in_{key}{i}"], int(z1), int(z2))
            assert rel(got, fx[f"out_{key}{i}"]) < 1e-6, (i, key, rel(got, fx[f"out_{key}{i}"]))


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
def test_reference_cpu_stepper_runs():
    """The reference's own CPU acoustic stepper (the acoustic CPU baseline) builds and propagates:
    in a homogeneous medium the wavefield stays finite, non-zero and mirror-symmetric about the
    source column (its update is symmetric in x up to the staggering)."""
    nx, nz, pml = 81, 61, 10
    vp = np.full((nx, nz), 2500.0, np.float32)
    rho = np.full((nx, nz), 2000.0, np.float32)
    damp = np.zeros((nx, nz), np.float32)
    from ds2d_b200 import synth
    w = synth.ricker(150, 15.0, 0.0008)
    p, sec = po.ref_cpu_acoustic(vp, rho, damp, w, 40, 30, 0.0008, 10.0, 10.0)
    assert np.isfinite(p).all() and np.abs(p).max() > 0 and sec > 0
    assert np.abs(p[40:30:-1, 30]).max() > 0

"""CPU tests of the oracle itself: reference formulas, model set-up and size-independent
properties (linearity, precision agreement, NCC identities)."""
import numpy as np
import pytest

from ds2d_b200 import synth
from oracle import pyoracle as po
from tests.helpers import rel, small_case


@pytest.fixture(scope="module")
def case():
    c, vp, vs, w, shots = small_case()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    model = po.build_model(st, vp, vs, None, shots[0].win_left)
    return c, vp, vs, w, shots, st, model


def test_ricker_matches_main_cpp(case):
    c, *_ = case
    np.testing.assert_array_equal(po.ricker(c["nt"], 15.0, c["dt"]), synth.ricker(c["nt"], 15.0, c["dt"]))


def test_model_window_edges_and_moduli(case):
    c, vp, vs, w, shots, st, model = case
    mvp, mvs, rho, lam, mu, dampx, dampz = model
    pml, wl, nx = c["pml"], shots[0].win_left, c["nx"]
    # interior is the model window, the PML replicates the edges (FD2DGPU.cu:122-138, 234-250)
    np.testing.assert_array_equal(mvp[pml:pml + nx, pml:-pml], vp[wl:wl + nx])
    np.testing.assert_array_equal(mvp[0, pml:-pml], vp[wl])
    np.testing.assert_array_equal(mvp[pml + 3, 0], vp[wl + 3, 0])
    np.testing.assert_array_equal(mvp[-1, -1], vp[wl + nx - 1, -1])
    assert np.all(rho == 2000.0)
    np.testing.assert_array_equal(lam, (np.float32(2000) * (mvp * mvp - np.float32(2) * (mvs * mvs))))
    # damping: zero in the interior, strict '>' at the far edges (FD2DGPU.cu:464, 490)
    assert np.all(dampx[pml:-pml] == 0) and np.all(dampz[:, pml:-pml] == 0)
    nxp = mvp.shape[0]
    assert np.all(dampx[nxp - pml] == 0) and np.all(dampx[nxp - pml + 1] > 0)
    assert np.all(dampx[:pml] > 0) and np.all(dampz[:, :pml] > 0)
    ix, iz = 2, pml + 5
    expect = np.log10(np.float64(np.float32(1) / np.float32(0.001))) * (5.0 * np.float64(mvp[ix, iz]) / (2.0 * pml)) * ((pml - ix) / pml) ** 4
    assert dampx[ix, iz] == pytest.approx(expect, rel=1e-6)


def test_random_band(case):
    c, vp, vs, w, shots, st, model = case
    rb = po.build_model(st, vp, vs, None, shots[0].win_left, rbc=1, seed=99, shot_id=4)
    pml = c["pml"]
    f = rb[0] / model[0]
    assert np.allclose(f[pml:-pml, pml:-pml], 1.0)
    band = np.ones_like(f, bool)
    band[pml:-pml, pml:-pml] = False
    assert f[band].min() >= 0.6 - 1e-6 and f[band].max() < 1.0 + 1e-6
    assert np.allclose(rb[1][band] / model[1][band], f[band], rtol=1e-6)
    assert np.all(rb[5] == 0) and np.all(rb[6] == 0)
    rb2 = po.build_model(st, vp, vs, None, shots[0].win_left, rbc=1, seed=99, shot_id=4)
    np.testing.assert_array_equal(rb[0], rb2[0])


def test_forward_precisions_agree(case):
    c, vp, vs, w, shots, st, model = case
    a = po.forward(st, model, w, shots[0], "f64")
    b = po.forward(st, model, w, shots[0], "f32")
    assert rel(b[0], a[0]) < 1e-5 and rel(b[1], a[1]) < 1e-5


def test_forward_linear_in_wavelet(case):
    c, vp, vs, w, shots, st, model = case
    a = po.forward(st, model, w, shots[0])
    b = po.forward(st, model, 2 * w, shots[0])
    assert rel(b[0], 2 * a[0]) < 1e-12


def test_rtm_linear_in_adjoint_source(case):
    c, vp, vs, w, shots, st, model = case
    rz, rx = po.forward(st, model, w, shots[0])
    for rbc in (0, 1):
        i1 = po.rtm(st, model, w, shots[0], rz, rx, rbc)
        i2 = po.rtm(st, model, w, shots[0], 3 * rz.astype(np.float32), 3 * rx.astype(np.float32), rbc)
        assert rel(i2[0], 3 * i1[0]) < 1e-6 and rel(i2[1], 3 * i1[1]) < 1e-6
        assert rel(i2[2], i1[2]) < 1e-12  # illumination depends on the source side only


def test_ncc_identities():
    rng = np.random.default_rng(0)
    d = rng.normal(size=(5, 50)).astype(np.float32)
    dx = rng.normal(size=(5, 50)).astype(np.float32)
    rz, rx, mis = po.ncc_residual(d, dx, d, dx, 0)
    np.testing.assert_allclose(rz, -d / (np.float64(d) ** 2).sum(1, keepdims=True), rtol=1e-6)
    assert mis == 0.0
    rz, rx, mis = po.ncc_residual(d, dx, d, dx, 1)
    assert mis == pytest.approx(-1.0, abs=1e-6)  # perfect correlation on every trace
    assert np.abs(rz).max() < 1e-6              # zero residual


def test_elsrtm_zero_image_has_no_scattering(case):
    c, vp, vs, w, shots, st, model = case
    rz, rx = po.forward(st, model, w, shots[0])
    z = np.zeros(st.shape, np.float32)
    r = po.elsrtm(st, model, z, z, w, shots[0], rz, rx, 0)
    assert np.abs(r["lm_vz"]).max() == 0 and np.abs(r["lm_vx"]).max() == 0
    for k in (3, 4, 5, 6):
        assert np.abs(r["images"][k]).max() == 0
    assert np.abs(r["images"][0]).max() > 0


def test_adam_update_matches_main_cpp():
    rng = np.random.default_rng(1)
    n = 64
    grads = [rng.normal(size=n).astype(np.float32) for _ in range(6)]
    pp = rng.normal(size=n).astype(np.float32)
    ps = rng.normal(size=n).astype(np.float32)
    pp0, ps0 = pp.copy(), ps.copy()
    st = [np.zeros(n) for _ in range(4)]
    import ctypes
    gp = (po.fp * 6)(*[g.ctypes.data_as(po.fp) for g in grads])
    for it in range(2):
        po.lib().orc_adam_update(n, it, gp, pp.ctypes.data_as(po.fp), ps.ctypes.data_as(po.fp),
                                 *[s.ctypes.data_as(po.dp) for s in st])
    # restatement of main.cpp:1092-1131 in numpy
    b1, b2, al, eps, ga = 0.8, 0.999, 3e-5, 5e8, 0.99
    b1, b2, al, eps, ga = (float(np.float32(v)) for v in (b1, b2, al, eps, ga))
    g = grads[0].astype(np.float64) + grads[2] + grads[4]
    s = r = 0
    x = pp0.astype(np.float64)
    for it in range(2):
        ak = al if it == 0 else (al / 2) * ga ** it
        s = b1 * s + (1 - b1) * g
        r = b2 * r + (1 - b2) * g * g
        k = it + 1
        x = (x - ak * ((s / (1 - b1 ** k)) / (np.sqrt(r / (1 - b2 ** k)) + eps))).astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(pp, x, rtol=1e-6)

"""Parity of the sm_100a path (through the C ABI) with the reference's CUDA build (golden fixtures
and, when oracle/_ref is present, live runs) and with the FP64 CPU oracle."""
import numpy as np
import pytest

from ds2d_b200 import Elastic2D, synth
from oracle import pyoracle as po
from tests.helpers import GATE, case_of, gate, load, rel, shots_of, small_case

pytestmark = pytest.mark.gpu


def _ctx(c, shots, **kw):
    return Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                     max_shots=kw.pop("max_shots", len(shots)), max_ntr=max(s.ntr for s in shots), **kw)


def _need(name):
    fx = load(name)
    if fx is None:
        pytest.fail(f"golden fixture {name} missing")
    return fx


def test_forward_vs_golden(cuda_device):
    fx = _need("forward_pml.npz")
    c = case_of(fx)
    shots = shots_of(fx)
    with _ctx(c, shots) as e:
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        rz, rx = e.forward(shots)
    ntr = shots[0].ntr
    for i in range(len(shots)):
        assert rel(rz[i * ntr:(i + 1) * ntr], fx["rec_vz"][i]) < gate()
        assert rel(rx[i * ntr:(i + 1) * ntr], fx["rec_vx"][i]) < gate()


def test_forward_batch_vs_oracle_f64(cuda_device):
    c, vp, vs, w, shots = small_case()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    rho = synth.gardner(vp)
    with _ctx(c, shots) as e:
        e.set_models(vp, vs, rho)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
        assert e.last_cell_updates == len(shots) * (c["nx"] + 2 * c["pml"]) * (c["allnz"] + 2 * c["pml"]) * c["nt"]
    ntr = shots[0].ntr
    for i, s in enumerate(shots):
        m = po.build_model(st, vp, vs, rho, s.win_left)
        oz, ox = po.forward(st, m, w, s, "f64")
        assert rel(rz[i * ntr:(i + 1) * ntr], oz) < gate()
        assert rel(rx[i * ntr:(i + 1) * ntr], ox) < gate()


@pytest.mark.parametrize("name", ["rtm_pml.npz", "rtm_random.npz"])
def test_rtm_vs_golden_and_oracle(cuda_device, name):
    fx = _need(name)
    c = case_of(fx)
    shots = shots_of(fx)
    rbc = int(fx["rbc"])
    seed = int(fx.get("seed", 0))
    with _ctx(c, shots, boundary="random" if rbc else "pml", seed=seed) as e:
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        e.rtm(shots, fx["adj_vz"].reshape(-1, c["nt"]), fx["adj_vx"].reshape(-1, c["nt"]))
        imgs = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    tot32 = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left, rbc=rbc, seed=seed, shot_id=i)
        for tot, prec in ((tot64, "f64"), (tot32, "f32")):
            o = po.rtm(st, m, fx["wavelet"], s, fx["adj_vz"][i], fx["adj_vx"][i], rbc, prec)
            for k in range(3):
                tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        floor = rel(tot32[k], tot64[k])
        assert rel(imgs[key], fx["images"][k]) < gate(floor), (key, rel(imgs[key], fx["images"][k]))
        assert rel(imgs[key], tot64[k]) < gate(floor), (key, rel(imgs[key], tot64[k]))


@pytest.mark.parametrize("it", [0, 1])
def test_elsrtm_vs_golden_and_oracle(cuda_device, it):
    fx = _need(f"elsrtm_iter{it}.npz")
    c = case_of(fx)
    s = shots_of(fx)[0]
    with _ctx(c, [s]) as e:
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        e.set_image(fx["img_pp"], fx["img_ps"])
        mis, (lz, lx, rz, rx) = e.elsrtm([s], fx["obs_vz"], fx["obs_vx"], it, want_records=True)
        imgs = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
    dmp = po.window_image(st, fx["img_pp"], s.win_left)
    dms = po.window_image(st, fx["img_ps"], s.win_left)
    args = (st, m, dmp, dms, fx["wavelet"], s, fx["obs_vz"], fx["obs_vx"], it)
    r64 = po.elsrtm(*args, precision="f64")
    r32 = po.elsrtm(*args, precision="f32")
    for got, key in ((rz, "res_vz"), (rx, "res_vx")):
        floor = rel(r32[key], r64[key])
        assert rel(got, fx[key]) < gate(floor), (key, rel(got, fx[key]), floor)
        assert rel(got, r64[key]) < gate(floor)
    floor = rel(r32["lm_vz"], r64["lm_vz"])
    assert rel(lz, r64["lm_vz"]) < gate(floor)
    for k, key in enumerate(Elastic2D.IMAGE_NAMES):
        full64 = po.place(r64["images"][k], c["allnx"], c["allnz"], s.win_left)
        full32 = po.place(r32["images"][k], c["allnx"], c["allnz"], s.win_left)
        floor = rel(full32, full64)
        assert rel(imgs[key], fx["images"][k]) < gate(floor), (key, rel(imgs[key], fx["images"][k]), floor)
        assert rel(imgs[key], full64) < gate(floor), (key, rel(imgs[key], full64), floor)
    if it > 0:
        assert mis == pytest.approx(fx["misfit"], rel=1e-4)


@pytest.mark.parametrize("boundary", ["pml", "random"])
def test_elsrtm_fused_matches_half_steps(cuda_device, boundary):
    """Reference-mode ELSRTM on the fused ring kernels (Born sources computed inside the
    background and first-order steps) against the half-step path and the FP64 oracle, three
    shots in one batch."""
    c, vp, vs, w, shots = small_case(nt=300)
    vpm, vsm = synth.smooth(vp, 3.0), synth.smooth(vs, 3.0)
    img_pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    img_ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    with _ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward(shots)
    rbc = int(boundary == "random")
    out = {}
    for fused in (0, 1):
        with _ctx(c, shots, boundary=boundary, seed=5) as e:
            e.set_option("fused", fused)
            e.set_models(vpm, vsm)
            e.set_wavelet(w)
            e.set_image(img_pp, img_ps)
            mis, recs = e.elsrtm(shots, oz, ox, 1, want_records=True)
            out[fused] = (mis, recs, e.read_images())
    # Same formulas, but the ring kernels round a few products differently (their expressions
    # contract into FMAs differently from the half-step kernels').  With the PML the two paths
    # agree to about 1e-6; the undamped random band keeps every rounding difference in the grid,
    # so there both are held to the FP32-vs-FP64 spread of the oracle.
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    ntr = shots[0].ntr
    tot64 = np.zeros((5, c["allnx"], c["allnz"]))
    tot32 = np.zeros((5, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        m = po.build_model(st, vpm, vsm, None, s.win_left, rbc=rbc, seed=5, shot_id=i)
        dmp = po.window_image(st, img_pp, s.win_left)
        dms = po.window_image(st, img_ps, s.win_left)
        sl = slice(i * ntr, (i + 1) * ntr)
        args = (st, m, dmp, dms, w, s, oz[sl], ox[sl], 1)
        r64 = po.elsrtm(*args, rbc=rbc, precision="f64")
        r32 = po.elsrtm(*args, rbc=rbc, precision="f32")
        for j, key in enumerate(("lm_vz", "lm_vx", "res_vz", "res_vx")):
            tol = gate(rel(r32[key], r64[key]))
            assert np.abs(r64[key]).max() > 0
            for fused in (0, 1):
                assert rel(out[fused][1][j][sl], r64[key]) < tol, (key, fused)
            assert rel(out[1][1][j][sl], out[0][1][j][sl]) < tol, key
        for k in range(5):
            tot64[k] += po.place(r64["images"][k], c["allnx"], c["allnz"], s.win_left)
            tot32[k] += po.place(r32["images"][k], c["allnx"], c["allnz"], s.win_left)
    for k, key in enumerate(Elastic2D.IMAGE_NAMES[:5]):
        tol = gate(rel(tot32[k], tot64[k]))
        for fused in (0, 1):
            assert rel(out[fused][2][key], tot64[k]) < tol, (key, fused)


def test_elsrtm_adjoint_born_as_written(cuda_device):
    """The scattered-adjoint term the reference's runs never execute (its launch exceeds the
    register limit), evaluated as written, against the FP64 oracle doing the same."""
    fx = _need("elsrtm_iter1.npz")
    c = case_of(fx)
    s = shots_of(fx)[0]
    with _ctx(c, [s]) as e:
        e.set_option("adjoint_born", 1)
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        e.set_image(fx["img_pp"], fx["img_ps"])
        e.elsrtm([s], fx["obs_vz"], fx["obs_vx"], 1)
        imgs = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
    dmp = po.window_image(st, fx["img_pp"], s.win_left)
    dms = po.window_image(st, fx["img_ps"], s.win_left)
    args = (st, m, dmp, dms, fx["wavelet"], s, fx["obs_vz"], fx["obs_vx"], 1)
    r64 = po.elsrtm(*args, precision="f64", adjoint_born=1)
    r32 = po.elsrtm(*args, precision="f32", adjoint_born=1)
    for k in (5, 6):
        key = Elastic2D.IMAGE_NAMES[k]
        full64 = po.place(r64["images"][k], c["allnx"], c["allnz"], s.win_left)
        full32 = po.place(r32["images"][k], c["allnx"], c["allnz"], s.win_left)
        assert np.abs(full64).max() > 0
        assert rel(imgs[key], full64) < gate(rel(full32, full64)), key


@pytest.mark.parametrize("boundary", ["pml", "random"])
@pytest.mark.parametrize("xr", [16, 64])
@pytest.mark.parametrize("ring", [0, 2, 4, 8])
def test_fused_step_matches_half_steps(cuda_device, boundary, xr, ring):
    c, vp, vs, w, shots = small_case(nt=300)
    out = {}
    for fused in (0, 1):
        with _ctx(c, shots, boundary=boundary, seed=5) as e:
            e.set_option("pair", 0)  # the one-column kernels (the pair kernels have their own test)
            e.set_option("tb", 0)  # one forward step per launch
            e.set_option("fused", fused)
            e.set_option("ring", ring)
            e.set_option("xr", xr)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            rz, rx = e.forward(shots)
            e.rtm(shots, rz, rx)
            out[fused] = (rz, rx, e.read_images())
    # Every path multiplies by 1 / (1 + dt d / 2) in PML cells and by 1 / dx, 1 / dz for strains.
    # The ring kernels also take each pair of adjoint-velocity derivatives of one stencil as a
    # single derivative of the summed operand (linearity): they agree with the half-step path at
    # the FP32 parity gate (1e-5), not bit for bit.  Without the ring the fused kernels keep the
    # half steps' operation order.
    tol = 1e-6 if ring == 0 else GATE
    assert rel(out[1][0], out[0][0]) < tol and rel(out[1][1], out[0][1]) < tol
    for key in ("pp_grad", "ps_grad", "illumination"):
        err = rel(out[1][2][key], out[0][2][key])
        assert err < tol, (key, err)


@pytest.mark.parametrize("boundary", ["pml", "random"])
def test_ring_occupancy_variants_agree(cuda_device, boundary):
    """Register-capped ring kernels (8 forward / 4 backward CTAs per SM) against the default."""
    c, vp, vs, w, shots = small_case(nt=300)
    out = {}
    for occ in (0, 1):
        with _ctx(c, shots, boundary=boundary, seed=5) as e:
            e.set_option("pair", 0)
            e.set_option("tb", 0)  # one forward step per launch
            e.set_option("occ", occ)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            rz, rx = e.forward(shots)
            e.rtm(shots, rz, rx)
            out[occ] = (rz, rx, e.read_images())
    assert rel(out[1][0], out[0][0]) < 1e-6 and rel(out[1][1], out[0][1]) < 1e-6
    for key in ("pp_grad", "ps_grad", "illumination"):
        assert rel(out[1][2][key], out[0][2][key]) < 1e-6, key


@pytest.mark.parametrize("boundary", ["pml", "random"])
def test_ring_cta_widths_agree(cuda_device, boundary):
    """192-thread ring CTAs (2 z-strips of 160 columns) against 128-thread ones (3 strips of
    107) on a 320-cell-deep grid: every cell does the same arithmetic, so the results are equal
    bit for bit."""
    c, _, _, w, _ = small_case(nt=200)
    c["allnz"] = 300
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=4)
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    out = {}
    for cta in (128, 192):
        with _ctx(c, shots, boundary=boundary, seed=5) as e:
            e.set_option("pair", 0)
            e.set_option("tb", 0)  # one forward step per launch
            e.set_option("cta", cta)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            rz, rx = e.forward(shots)
            e.rtm(shots, rz, rx)
            out[cta] = (rz, rx, e.read_images())
    assert np.abs(out[128][0]).max() > 0
    assert np.array_equal(out[192][0], out[128][0]) and np.array_equal(out[192][1], out[128][1])
    for key in ("pp_grad", "ps_grad", "illumination"):
        assert np.array_equal(out[192][2][key], out[128][2][key]), key


@pytest.mark.parametrize("fused", [0, 1])
def test_uneven_windows_vs_oracle(cuda_device, fused):
    """Shots of different aperture widths in one batch (per-slot window sizes)."""
    c, vp, vs, w, _ = small_case(nt=200)
    shots = synth.uneven_shots(c["allnx"], c["pml"], 4, 20, c["allnx"], seed=9)
    wmax = max(s.nx for s in shots)
    with Elastic2D(c["allnx"], c["allnz"], wmax, c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   max_shots=len(shots), max_ntr=wmax) as e:
        e.set_option("fused", fused)
        e.set_models(vp, vs)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
        e.rtm(shots, rz, rx)
        imgs = e.read_images()
    off = 0
    tot = np.zeros((3, c["allnx"], c["allnz"]))
    for s in shots:
        st = po.Setup(c["allnx"], c["allnz"], s.nx, c["pml"], c["dx"], c["dz"], c["dt"])
        m = po.build_model(st, vp, vs, None, s.win_left)
        oz, ox = po.forward(st, m, w, s)
        assert rel(rz[off:off + s.ntr], oz) < gate()
        o = po.rtm(st, m, w, s, rz[off:off + s.ntr], rx[off:off + s.ntr], 0)
        for k in range(3):
            tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
        off += s.ntr
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        assert rel(imgs[key], tot[k]) < 1e-4, (key, rel(imgs[key], tot[k]))


def test_graph_replay_matches_direct_launches(cuda_device):
    """Batches captured into CUDA graphs (first call) and replayed (later calls) give the same
    bits as direct launches."""
    import torch
    c, vp, vs, w, shots = small_case(nt=150)
    stream = torch.cuda.Stream()
    out = {}
    for graph in (0, 1):
        with _ctx(c, shots, boundary="random", seed=3) as e:
            e.set_option("graph", graph)
            e.set_stream(stream.cuda_stream)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            rz, rx = e.forward(shots)
            rz2, rx2 = e.forward(shots)  # replay
            np.testing.assert_array_equal(rz, rz2)
            for _ in range(2):  # capture, then replay
                e.rtm(shots, rz, rx)
                out[graph, _] = e.read_images()
            out[graph, "rec"] = rz
    np.testing.assert_array_equal(out[0, "rec"], out[1, "rec"])
    for key in ("pp_grad", "ps_grad", "illumination"):
        np.testing.assert_array_equal(out[1, 0][key], out[0, 0][key])
        np.testing.assert_array_equal(out[1, 1][key], out[0, 0][key])


def test_batched_equals_one_by_one(cuda_device):
    c, vp, vs, w, shots = small_case(nt=200)
    rz, rx = None, None
    with _ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
        e.rtm(shots, rz, rx)
        batched = e.read_images()
    with _ctx(c, shots, max_shots=1) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        ntr = shots[0].ntr
        for i, s in enumerate(shots):
            e.rtm([s], rz[i * ntr:(i + 1) * ntr], rx[i * ntr:(i + 1) * ntr])
        single = e.read_images()
    for key in ("pp_grad", "ps_grad", "illumination"):
        np.testing.assert_array_equal(batched[key], single[key])


def test_elsrtm_batched_equals_one_by_one(cuda_device):
    """Reference-mode ELSRTM of three shots in one batch and one shot per batch: every shot runs
    the same kernels on its own slot and the images are reduced in shot order, so the gradients
    and the misfit agree bit for bit."""
    c, vp, vs, w, shots = small_case(nt=200)
    vpm, vsm = synth.smooth(vp, 3.0), synth.smooth(vs, 3.0)
    img_pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    img_ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    with _ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward(shots)
    out = {}
    for max_shots in (len(shots), 1):
        with _ctx(c, shots, max_shots=max_shots) as e:
            e.set_models(vpm, vsm)
            e.set_wavelet(w)
            e.set_image(img_pp, img_ps)
            mis = e.elsrtm(shots, oz, ox, 1)
            out[max_shots] = (mis, e.read_images())
    assert out[1][0] == out[len(shots)][0]
    for key in Elastic2D.IMAGE_NAMES:
        np.testing.assert_array_equal(out[1][1][key], out[len(shots)][1][key])


@pytest.mark.parametrize("strips", ["f16", "bf16"])
def test_half_precision_strips(cuda_device, strips):
    """RTM with the PML and the source field rebuilt from FP16 / BF16 boundary strips (one FP32
    scale per 32-cell segment) against the FP64 oracle, which keeps its strips exact: the error
    the storage format adds to the images (gates: FP16 2e-3, BF16 2e-2 relative L2), next to the
    FP32-strip run's own distance from the oracle."""
    fx = _need("rtm_pml.npz")
    c = case_of(fx)
    shots = shots_of(fx)
    out = {}
    for prec in ("f32", strips):
        with _ctx(c, shots, strips=prec) as e:
            e.set_models(fx["vp"], fx["vs"])
            e.set_wavelet(fx["wavelet"])
            e.rtm(shots, fx["adj_vz"].reshape(-1, c["nt"]), fx["adj_vx"].reshape(-1, c["nt"]))
            out[prec] = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
        o = po.rtm(st, m, fx["wavelet"], s, fx["adj_vz"][i], fx["adj_vx"][i], 0, "f64")
        for k in range(3):
            tot64[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
    tol = 2e-3 if strips == "f16" else 2e-2
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        err = rel(out[strips][key], tot64[k])
        err32 = rel(out["f32"][key], tot64[k])
        assert err < tol, (key, err, f"FP32 strips: {err32:.3e}")


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
def test_live_reference_rtm_random(cuda_device):
    c, vp, vs, w, shots = small_case(nt=250)
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m0 = po.build_model(st, vp, vs, None, shots[0].win_left)
    obs = [po.forward(st, po.build_model(st, vp, vs, None, s.win_left), w, s) for s in shots]
    az = np.concatenate([o[0] for o in obs]).astype(np.float32)
    ax = np.concatenate([o[1] for o in obs]).astype(np.float32)
    vpm, vsm = synth.smooth(vp, 2.0), synth.smooth(vs, 2.0)
    pads = [po.build_model(st, vpm, vsm, None, s.win_left, rbc=1, seed=77, shot_id=i) for i, s in enumerate(shots)]
    ref_imgs, _ = po.ref_rtm(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                             vpm, vsm, w, shots, az, ax, rbc=1,
                             vp_pad=np.stack([p[0] for p in pads]), vs_pad=np.stack([p[1] for p in pads]))
    with _ctx(c, shots, boundary="random", seed=77) as e:
        e.set_models(vpm, vsm)
        e.set_wavelet(w)
        e.rtm(shots, az, ax)
        imgs = e.read_images()
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    tot32 = np.zeros((3, c["allnx"], c["allnz"]))
    ntr = shots[0].ntr
    for i, s in enumerate(shots):
        sl = slice(i * ntr, (i + 1) * ntr)
        for tot, prec in ((tot64, "f64"), (tot32, "f32")):
            o = po.rtm(st, pads[i], w, s, az[sl], ax[sl], 1, prec)
            for k in range(3):
                tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        floor = rel(tot32[k], tot64[k])
        err = rel(imgs[key], ref_imgs[k])
        assert err < gate(floor), f"{key}: vs reference {err:.3e}, FP32 floor {floor:.3e}"


@pytest.mark.parametrize("mode,pair_cta,pair_fcta,pair_split", [(1, 64, 64, 0), (1, 256, 256, 0),
                                                              (1, 160, 64, 0), (1, 0, 64, 1),
                                                              (2, 0, 256, 0)])
@pytest.mark.parametrize("pair_xr", [0, 24])
def test_pair_kernels_match_ring_and_oracle(cuda_device, mode, pair_cta, pair_fcta, pair_split,
                                            pair_xr):
    """Pair-blocked bulk-copy kernels of the random-boundary RTM step (forward with receiver
    records, backward with the residual injection and the imaging condition) against the
    one-column ring kernels and the FP64 oracle; fused, or split into a reconstruction launch and
    an adjoint + imaging launch.  On the 320-deep grid the 64-thread CTAs run four z-strips and
    the 160-thread ones two; xr 24 gives each shot four row blocks (x-halos between CTAs).  Mode
    2 runs the pair kernel for the forward step only and the one-column kernel backward."""
    c, _, _, w, _ = small_case(nt=200)
    c["allnz"] = 300
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=4)
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    with _ctx(c, shots, boundary="pml") as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward(shots)
    vpm, vsm = synth.smooth(vp, 3.0), synth.smooth(vs, 3.0)
    out = {}
    for pair in (0, 1):
        with _ctx(c, shots, boundary="random", seed=5) as e:
            e.set_option("pair", mode if pair else 0)
            e.set_option("tb", 0)  # one forward step per launch
            if pair:
                e.set_option("pair_cta", pair_cta)
                e.set_option("pair_fcta", pair_fcta)
                e.set_option("pair_split", pair_split)
                e.set_option("pair_xr", pair_xr)
            e.set_models(vpm, vsm)
            e.set_wavelet(w)
            rz, rx = e.forward(shots)
            e.rtm(shots, oz, ox)
            out[pair] = (rz, rx, e.read_images())
    assert np.abs(out[1][0]).max() > 0
    assert rel(out[1][0], out[0][0]) < GATE and rel(out[1][1], out[0][1]) < GATE
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    ntr = shots[0].ntr
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    tot32 = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        m = po.build_model(st, vpm, vsm, None, s.win_left, rbc=1, seed=5, shot_id=i)
        fz, fx = po.forward(st, m, w, s, "f64")
        sl = slice(i * ntr, (i + 1) * ntr)
        assert rel(out[1][0][sl], fz) < GATE and rel(out[1][1][sl], fx) < GATE
        for tot, prec in ((tot64, "f64"), (tot32, "f32")):
            o = po.rtm(st, m, w, s, oz[sl], ox[sl], 1, prec)
            for k in range(3):
                tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        floor = rel(tot32[k], tot64[k])
        err_ring = rel(out[1][2][key], out[0][2][key])
        err64 = rel(out[1][2][key], tot64[k])
        assert err_ring < gate(floor), (key, err_ring, f"FP32 floor {floor:.3e}")
        assert err64 < gate(floor), (key, err64, f"FP32 floor {floor:.3e}")


def test_pair_kernels_uneven_windows(cuda_device):
    """Shots of different aperture in one batch on the pair kernels (per-slot row counts, CTAs
    beyond a slot's window return at once) against the FP64 oracle."""
    c, vp, vs, w, _ = small_case(nt=200)
    shots = synth.uneven_shots(c["allnx"], c["pml"], 4, 20, c["allnx"], seed=9)
    wmax = max(s.nx for s in shots)
    with Elastic2D(c["allnx"], c["allnz"], wmax, c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="random", seed=8, max_shots=len(shots), max_ntr=wmax) as e:
        e.set_option("pair", 1)
        e.set_option("tb", 0)  # one forward step per launch
        e.set_option("pair_xr", 16)
        e.set_models(vp, vs)
        e.set_wavelet(w)
        rz, rx = e.forward(shots)
        e.rtm(shots, rz, rx)
        imgs = e.read_images()
    off = 0
    tot = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        st = po.Setup(c["allnx"], c["allnz"], s.nx, c["pml"], c["dx"], c["dz"], c["dt"])
        m = po.build_model(st, vp, vs, None, s.win_left, rbc=1, seed=8, shot_id=i)
        oz, ox = po.forward(st, m, w, s)
        assert rel(rz[off:off + s.ntr], oz) < GATE
        o = po.rtm(st, m, w, s, rz[off:off + s.ntr], rx[off:off + s.ntr], 1)
        for k in range(3):
            tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
        off += s.ntr
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        assert rel(imgs[key], tot[k]) < 1e-4, (key, rel(imgs[key], tot[k]))


def _headline_survey(nt):
    """The RTM benchmark's grid (1201x401 model, 40-cell band, dt 0.8 ms), its seeded model pair
    and two of its 60 surface shots."""
    c = dict(allnx=1201, allnz=401, nx=1201, pml=40, nt=nt, dx=10.0, dz=10.0, dt=0.0008)
    vp, vs = synth.dipping_lenses(c["allnx"], c["allnz"], seed=2024)
    vpm, vsm = synth.smooth(vp, 15.0), synth.smooth(vs, 15.0)
    w = synth.ricker(nt, 15.0, c["dt"])
    survey = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 60)
    return c, vp, vs, vpm, vsm, w, [survey[7], survey[41]]


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
def test_live_reference_rtm_headline(cuda_device):
    """Elastic RTM at the benchmark's full size (1201x401 + 40-cell random band, nt 4000, two
    shots) against the reference's own CUDA kernels on the same padded model, and one shot against
    the FP64 oracle.  In the undamped band every rounding difference stays in the grid for 4000
    steps: the reference's FP32 result itself lies about 1.5e-3 from the FP64 restatement of its
    scheme (its split-field update rounds differently), so the gate against it is the FP32 floor
    of the scheme (|oracle f32 - oracle f64|), which every assertion prints.  Against the FP64
    oracle this path must be at least as close as the reference is."""
    c, vp, vs, vpm, vsm, w, shots = _headline_survey(4000)
    g = tuple(c.values())
    with _ctx(c, shots, boundary="pml") as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        az, ax = e.forward(shots)
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    pads = [po.build_model(st, vpm, vsm, None, s.win_left, rbc=1, seed=77, shot_id=i)
            for i, s in enumerate(shots)]
    vpp, vsp = np.stack([p[0] for p in pads]), np.stack([p[1] for p in pads])
    ntr = shots[0].ntr
    ref2, _ = po.ref_rtm(*g, vpm, vsm, w, shots, az, ax, rbc=1, vp_pad=vpp, vs_pad=vsp)
    ref1, _ = po.ref_rtm(*g, vpm, vsm, w, shots[:1], az[:ntr], ax[:ntr], rbc=1, vp_pad=vpp[:1],
                         vs_pad=vsp[:1])
    with _ctx(c, shots, boundary="random", seed=77) as e:
        e.set_models(vpm, vsm)
        e.set_wavelet(w)
        e.rtm(shots, az, ax)
        ours2 = e.read_images()
        e.rtm(shots[:1], az[:ntr], ax[:ntr])
        ours1 = e.read_images()
    o64 = po.rtm(st, pads[0], w, shots[0], az[:ntr], ax[:ntr], 1, "f64")
    o32 = po.rtm(st, pads[0], w, shots[0], az[:ntr], ax[:ntr], 1, "f32")
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        f64 = po.place(o64[k], c["allnx"], c["allnz"], shots[0].win_left)
        f32 = po.place(o32[k], c["allnx"], c["allnz"], shots[0].win_left)
        floor = rel(f32, f64)
        e_ref = rel(ours2[key], ref2[k])
        e_64, r_64 = rel(ours1[key], f64), rel(ref1[k], f64)
        msg = (f"{key}: vs reference {e_ref:.3e}, vs FP64 {e_64:.3e} (reference vs FP64 "
               f"{r_64:.3e}), FP32 floor {floor:.3e}")
        assert e_ref < gate(floor), msg
        assert e_64 < gate(floor) and e_64 <= r_64 + GATE, msg


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
def test_live_reference_elsrtm_full_size(cuda_device):
    """Reference-mode ELSRTM (PML + FP32 strips, Born modelling, NCC adjoint source, seven
    gradients) at 1201x401, nt 2000, one shot, against the reference's own per-shot driver and
    the FP64 oracle.  Receivers within 300 columns of the source: the wavefield reaches all of
    them in 2000 steps (the reference's NCC divides by each trace's norm, FD2DGPU.cu:4567-4572,
    so an all-zero trace would give NaN in both).  Each output must be within the FP32 floor of
    the FP64 oracle, and within that floor plus the reference's own distance to the FP64 oracle of
    the reference."""
    from ds2d_b200.api import ShotGeom
    c, vp, vs, vpm, vsm, w, _ = _headline_survey(2000)
    g = tuple(c.values())
    s0 = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 16)[5]
    igx = np.arange(max(c["pml"], s0.isx - 300), min(c["pml"] + c["nx"], s0.isx + 301),
                    dtype=np.int32)
    s = ShotGeom(s0.win_left, s0.isx, s0.isz, s0.igz, igx)
    with _ctx(c, [s], boundary="pml") as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward([s])
    pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    r = po.ref_elsrtm(*g, vpm, vsm, w, pp, ps, s, oz, ox, 1)
    with _ctx(c, [s], boundary="pml", strips="f32") as e:
        e.set_models(vpm, vsm)
        e.set_wavelet(w)
        e.set_image(pp, ps)
        mis, (_, _, rz, rx) = e.elsrtm([s], oz, ox, 1, want_records=True)
        imgs = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m = po.build_model(st, vpm, vsm, None, s.win_left)
    args = (st, m, po.window_image(st, pp, s.win_left), po.window_image(st, ps, s.win_left), w, s,
            oz, ox, 1)
    r64 = po.elsrtm(*args, precision="f64")
    r32 = po.elsrtm(*args, precision="f32")
    outs = [(rz, r["res_vz"], r64["res_vz"], r32["res_vz"], "res_vz"),
            (rx, r["res_vx"], r64["res_vx"], r32["res_vx"], "res_vx")]
    for k, key in enumerate(Elastic2D.IMAGE_NAMES[:5]):
        outs.append((imgs[key], r["images"][k],
                     po.place(r64["images"][k], c["allnx"], c["allnz"], s.win_left),
                     po.place(r32["images"][k], c["allnx"], c["allnz"], s.win_left), key))
    for got, ref, f64, f32, key in outs:
        floor = rel(f32, f64)
        e_ref, e_64, r_64 = rel(got, ref), rel(got, f64), rel(ref, f64)
        msg = (f"{key}: vs reference {e_ref:.3e}, vs FP64 {e_64:.3e} (reference vs FP64 "
               f"{r_64:.3e}), FP32 floor {floor:.3e}")
        assert e_64 < gate(floor), msg
        assert e_ref < gate(floor) + r_64, msg
    assert mis == pytest.approx(r["misfit"], rel=1e-4) and mis == pytest.approx(r64["misfit"], rel=1e-4)


@pytest.mark.parametrize("opts,xr,allnz", [
    ({"bwd_ws": 96}, 128, 300), ({"bwd_ws": 128}, 24, 300), ({"bwd_ws": 192}, 24, 300),
    ({"bwd_ws": 192}, 128, 300), ({"bwd_1b": 1, "bwd_bulk": 0, "cta": 128}, 24, 300),
    ({"bwd_1b": 1, "bwd_bulk": 0, "cta": 192}, 128, 300),
    ({"bwd_bulk": 1, "bwd_cta": 128}, 24, 300), ({"bwd_bulk": 1, "bwd_cta": 192}, 128, 300),
    ({"bwd_bulk": 1, "bwd_cta": 256}, 24, 300), ({"bwd_bulk": 1, "bwd_cta": 256}, 128, 200),
    ({"bwd_bulk": 1, "bwd_1b": 1, "bwd_cta": 192}, 24, 300),
    ({"bwd_bulk": 1, "bwd_1b": 1, "bwd_cta": 256}, 128, 300)])
def test_backward_variants_match_ring_and_oracle(cuda_device, opts, xr, allnz):
    """Variants of the backward RTM step against the one-column ring kernel and the FP64 oracle,
    random boundary: the warp-specialised step (k_bwd_ws: the source field and the adjoint field
    on separate warps of one CTA, strains handed over in shared memory for the imaging
    condition), the ring kernel with one barrier per row step (bwd_1b) and the ring fed by bulk
    copies (k_bwd_bulk, with either barrier count, halo columns only at inner strip edges).  The
    320-deep grid gives every CTA width two or more z-strips, the 220-deep one a single
    256-thread strip; xr 24 gives each shot several row blocks."""
    c, _, _, w, _ = small_case(nt=200)
    c["allnz"] = allnz
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=4)
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    with _ctx(c, shots, boundary="pml") as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        oz, ox = e.forward(shots)
    vpm, vsm = synth.smooth(vp, 3.0), synth.smooth(vs, 3.0)
    out = {}
    for var in (0, 1):
        with _ctx(c, shots, boundary="random", seed=5) as e:
            e.set_option("pair", 0)
            e.set_option("xr", xr)  # rows per CTA of the one-column ring kernels
            e.set_option("pair_xr", xr)  # and of the bulk-copy ones
            e.set_option("bwd_1b", 0)  # the two-barrier per-thread ring kernel as the reference
            e.set_option("bwd_bulk", 0)
            for k, v in (opts if var else {}).items():
                e.set_option(k, v)
            e.set_models(vpm, vsm)
            e.set_wavelet(w)
            e.rtm(shots, oz, ox)
            out[var] = e.read_images()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    ntr = shots[0].ntr
    tot64 = np.zeros((3, c["allnx"], c["allnz"]))
    tot32 = np.zeros((3, c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        m = po.build_model(st, vpm, vsm, None, s.win_left, rbc=1, seed=5, shot_id=i)
        sl = slice(i * ntr, (i + 1) * ntr)
        for tot, prec in ((tot64, "f64"), (tot32, "f32")):
            o = po.rtm(st, m, w, s, oz[sl], ox[sl], 1, prec)
            for k in range(3):
                tot[k] += po.place(o[k], c["allnx"], c["allnz"], s.win_left)
    for k, key in enumerate(("pp_grad", "ps_grad", "illumination")):
        assert np.abs(out[1][key]).max() > 0
        floor = rel(tot32[k], tot64[k])
        err_ring = rel(out[1][key], out[0][key])
        err64 = rel(out[1][key], tot64[k])
        assert err_ring < gate(floor), (key, err_ring, f"FP32 floor {floor:.3e}")
        assert err64 < gate(floor), (key, err64, f"FP32 floor {floor:.3e}")

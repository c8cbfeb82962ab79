"""Acoustic Born operator pair and CG-LSRTM on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from ds2d_b200 import Elastic2D, synth
from oracle import pyoracle as po
from tests.helpers import gate, rel

pytestmark = pytest.mark.gpu

# The Born data of the scheme are reproducible only to ~3e-4 in FP32 (rounding-order floor of
# the scattered field, measured on the oracle), so the operator gates sit above that.
BORN_GATE = 2e-3


def acoustic_case(nt=300, nshots=3):
    c = dict(allnx=64, allnz=36, nx=64, pml=12, nt=nt, dx=10.0, dz=10.0, dt=0.0008, f0=15.0)
    vp = np.broadcast_to(np.linspace(1800, 4500, c["allnz"], dtype=np.float32),
                         (c["allnx"], c["allnz"])).copy()
    vs = np.zeros_like(vp)
    w = synth.ricker(nt, c["f0"], c["dt"])
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], nshots)
    m = synth.reflectivity(c["allnx"], c["allnz"], seed=4, density=0.05, std=0.05)
    m[:, :3] = 0
    return c, vp, vs, w, shots, m


def ctx(c, shots, seed=21):
    e = Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                  boundary="random", seed=seed, max_shots=len(shots), max_ntr=c["nx"])
    return e


def oracle_models(c, vp, vs, shots, seed=21):
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    return st, [po.build_model(st, vp, vs, None, s.win_left, rbc=1, seed=seed, shot_id=i)
                for i, s in enumerate(shots)]


def pad(st, m_full, s, c):
    out = np.zeros(st.shape)
    out[c["pml"]:c["pml"] + c["nx"], c["pml"]:-c["pml"]] = m_full[s.win_left:s.win_left + c["nx"]]
    return out


@pytest.mark.parametrize("n", [1, 1000, 3_000_001])
def test_dot_f64(cuda_device, n):
    import torch
    g = torch.Generator().manual_seed(n)
    a = torch.randn(n, generator=g, dtype=torch.float32)
    b = torch.randn(n, generator=g, dtype=torch.float32)
    ref = float((a.double() * b.double()).sum())
    da, db = a.cuda(), b.cuda()
    torch.cuda.synchronize()
    with Elastic2D(16, 16, 16, 8, 4, 10.0, 10.0, 0.001) as e:
        got = e.dot_f64(da.data_ptr(), db.data_ptr(), n)
        again = e.dot_f64(da.data_ptr(), db.data_ptr(), n)
    assert got == again  # deterministic order
    assert abs(got - ref) <= 1e-12 * max(1.0, float((a.double().abs() * b.double().abs()).sum()))


def test_ac_born_and_adjoint_vs_oracle(cuda_device):
    c, vp, vs, w, shots, m = acoustic_case()
    st, models = oracle_models(c, vp, vs, shots)
    with ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        dz, dx = e.ac_born(shots, m)
        rng = np.random.default_rng(3)
        rz = rng.normal(size=dz.shape).astype(np.float32)
        rx = rng.normal(size=dx.shape).astype(np.float32)
        g = e.ac_born_adj(shots, rz, rx)
    ntr = shots[0].ntr
    gref = np.zeros((c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        oz, ox = po.ac_born(st, models[i], w, s, pad(st, m, s, c))
        assert rel(dz[i * ntr:(i + 1) * ntr], oz) < BORN_GATE
        assert rel(dx[i * ntr:(i + 1) * ntr], ox) < BORN_GATE
        gp = po.ac_born_adj(st, models[i], w, s, rz[i * ntr:(i + 1) * ntr], rx[i * ntr:(i + 1) * ntr])
        gref[s.win_left:s.win_left + c["nx"]] += gp[c["pml"]:c["pml"] + c["nx"], c["pml"]:-c["pml"]]
    assert rel(g, gref) < BORN_GATE, rel(g, gref)


@pytest.mark.parametrize("cta,xr", [(0, 0), (128, 24), (192, 0), (256, 40)])
def test_ac_pair_kernels_match_ring_and_oracle(cuda_device, cta, xr):
    """Pair-blocked acoustic forward steps (k_ac_pair: background with the Born source written,
    scattered set with records, and the background replay of L^T) against the one-column ring
    kernels and the FP64 oracle.  The 300-deep grid gives the 128-thread CTAs two z-strips; xr
    24 / 40 gives every shot several row blocks (x-halos between CTAs)."""
    c, vp, vs, w, shots, m = acoustic_case(nt=300)
    c["allnz"] = 300
    vp = np.broadcast_to(np.linspace(1800, 4500, c["allnz"], dtype=np.float32),
                         (c["allnx"], c["allnz"])).copy()
    vs = np.zeros_like(vp)
    m = synth.reflectivity(c["allnx"], c["allnz"], seed=4, density=0.05, std=0.05)
    m[:, :3] = 0
    rng = np.random.default_rng(3)
    out = {}
    for pair in (0, 1):
        with ctx(c, shots) as e:
            e.set_option("ac_pair", pair)
            e.set_option("ac_pair_cta", cta)
            e.set_option("pair_xr", xr)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            dz, dx = e.ac_born(shots, m)
            if pair == 0:
                rz = rng.normal(size=dz.shape).astype(np.float32)
                rx = rng.normal(size=dx.shape).astype(np.float32)
            g = e.ac_born_adj(shots, rz, rx)
            out[pair] = (dz, dx, g)
    assert np.abs(out[1][0]).max() > 0
    # FP32 floor of the Born records: the oracle's elastic Born step at vs = 0 (the same operator)
    # in FP32 against FP64
    st, models = oracle_models(c, vp, vs, shots)
    ntr = shots[0].ntr
    floor = 0.0
    for i, s in enumerate(shots[:2]):
        dmp = po.window_image(st, m, s.win_left)
        dms = po.window_image(st, np.zeros_like(m), s.win_left)
        b64 = po.born(st, models[i], dmp, dms, w, s, "f64")
        b32 = po.born(st, models[i], dmp, dms, w, s, "f32")
        fl = max(rel(b32[0], b64[0]), rel(b32[1], b64[1]))
        floor = max(floor, fl)
        for j in range(2):
            err = rel(out[1][j][i * ntr:(i + 1) * ntr], b64[j])
            assert err < gate(fl), (i, j, err, f"FP32 floor {fl:.3e}")
    for k in range(3):
        err = rel(out[1][k], out[0][k])
        assert err < gate(floor), (k, err, f"FP32 floor {floor:.3e}")


@pytest.mark.parametrize("ac_pair", [0, 1])
def test_ac_dot_product_fp32(cuda_device, ac_pair):
    """<L m, d> = <m, L^T d> for the sm_100a pair (FP32 arithmetic, FP64 sums), on the
    one-column ring kernels and on the pair-blocked ones."""
    c, vp, vs, w, shots, m = acoustic_case(nt=400)
    with ctx(c, shots) as e:
        e.set_option("ac_pair", ac_pair)
        e.set_models(vp, vs)
        e.set_wavelet(w)
        dz, dx = e.ac_born(shots, m)
        rng = np.random.default_rng(8)
        rz = rng.normal(size=dz.shape).astype(np.float32)
        rx = rng.normal(size=dx.shape).astype(np.float32)
        g = e.ac_born_adj(shots, rz, rx)
    lhs = float((dz.astype(np.float64) * rz).sum() + (dx.astype(np.float64) * rx).sum())
    rhs = float((m.astype(np.float64) * g).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-4, (lhs, rhs)


def test_lsrtm_cg_matches_oracle_cgls(cuda_device):
    c, vp, vs, w, shots, m = acoustic_case(nt=300)
    st, models = oracle_models(c, vp, vs, shots)
    with ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        dz, dx = e.ac_born(shots, m)
        mg, hist = e.lsrtm(shots, dz, dx, niter=4)
    # CGLS in FP64 on the oracle operators with the same data
    ntr = shots[0].ntr
    d = [(dz[i * ntr:(i + 1) * ntr].astype(np.float64), dx[i * ntr:(i + 1) * ntr].astype(np.float64))
         for i in range(len(shots))]
    L = lambda mm: [po.ac_born(st, models[i], w, s, mm) for i, s in enumerate(shots)]
    LT = lambda dd: sum(po.ac_born_adj(st, models[i], w, s, *dd[i]) for i, s in enumerate(shots))
    dot = lambda a, b: sum((x * y).sum() + (u * v).sum() for (x, u), (y, v) in zip(a, b))
    mm = np.zeros(st.shape)
    r = [(a.copy(), b.copy()) for a, b in d]
    dn = np.sqrt(dot(d, d))
    s_ = LT(r)
    p = s_.copy()
    gam = (s_ * s_).sum()
    ref = []
    for _ in range(4):
        q = L(p)
        al = gam / dot(q, q)
        mm += al * p
        r = [(a - al * x, b - al * y) for (a, b), (x, y) in zip(r, q)]
        ref.append(np.sqrt(dot(r, r)) / dn)
        s_ = LT(r)
        gn = (s_ * s_).sum()
        p = s_ + (gn / gam) * p
        gam = gn
    assert len(hist) == 4
    np.testing.assert_allclose(hist, ref, rtol=5e-3)
    assert hist[-1] < hist[0] < 1.0


def test_lsrtm_pcg_plain_matches_cgls_and_net_descends(cuda_device):
    """ds2d_lsrtm_pcg with P = I follows CGLS (same residuals up to rounding); with a U-Net as P
    (untrained) the exact line search still makes every iteration decrease the residual."""
    import torch
    from ds2d_b200.unet import UNet, flatten
    from oracle import unet_oracle as uo
    c, vp, vs, w, shots, m = acoustic_case(nt=300, nshots=3)
    with ctx(c, shots) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        dz, dx = e.ac_born(shots, m)
        _, hist_cgls = e.lsrtm(shots, dz, dx, 4)
        tz, tx = torch.from_numpy(dz).cuda(), torch.from_numpy(dx).cuda()
        mo = torch.zeros((c["allnx"], c["allnz"]), dtype=torch.float32, device="cuda")
        hist, ms = e.lsrtm_pcg(shots, tz.data_ptr(), tx.data_ptr(), mo.data_ptr(), 4)
        assert len(hist) == 4 and np.all(np.diff(ms) > 0)
        np.testing.assert_allclose(hist, hist_cgls, rtol=2e-3)
        hp, wp = (c["allnx"] + 7) // 8 * 8, (c["allnz"] + 7) // 8 * 8
        with UNet(max_n=1, max_h=hp, max_w=wp) as net:
            net.set_params(flatten(uo.init_params(1)))
            mo.zero_()
            hist_n, _ = e.lsrtm_pcg(shots, tz.data_ptr(), tx.data_ptr(), mo.data_ptr(), 4, net=net)
    assert np.all(np.diff(np.concatenate([[1.0], hist_n])) < 0), hist_n


def test_acoustic_fused_steps_match_half_steps(cuda_device):
    """The fused one-column acoustic step (velocity + stress + Born source in one x-march,
    ping-pong state) against one launch per half step, for L and L^T.  The pair-blocked kernels
    (the default) round their z-taps differently and are gated against these at the FP32 floor in
    test_ac_pair_kernels_match_ring_and_oracle."""
    c, vp, vs, w, shots, m = acoustic_case(nt=300, nshots=3)
    out = {}
    for fused in (0, 1):
        with ctx(c, shots) as e:
            e.set_option("fused", fused)
            e.set_option("ac_pair", 0)
            e.set_models(vp, vs)
            e.set_wavelet(w)
            dz, dx = e.ac_born(shots, m)
            g = e.ac_born_adj(shots, dz, dx)
            out[fused] = (dz, dx, g)
    for a, b in zip(out[1], out[0]):
        assert rel(a, b) < 1e-6, rel(a, b)


def test_ac_born_vs_reference_golden(cuda_device):
    """The acoustic Born operator against the reference itself: first-order Born records of the
    reference's born_modeling (mode 1) with vs = 0 (mu = 0 removes every shear term), the random
    band injected and no damping, made by tests/golden/make_golden.py.  Born records are
    reproducible only to the FP32 floor of the scheme, measured per case on the oracle."""
    from tests.helpers import case_of, gate, load, shots_of
    fx = load("born_acoustic_random.npz")
    assert fx is not None, "golden fixture born_acoustic_random.npz missing"
    c = case_of(fx)
    shots = shots_of(fx)
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    seed = int(fx["seed"])
    with Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="random", seed=seed, max_shots=len(shots),
                   max_ntr=max(s.ntr for s in shots)) as e:
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        dz, dx = e.ac_born(shots, fx["img_pp"])
    ntr = shots[0].ntr
    zero = np.zeros_like(fx["img_pp"])
    for i, s in enumerate(shots):
        m = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left, rbc=1, seed=seed, shot_id=i)
        dmp = po.window_image(st, fx["img_pp"], s.win_left)
        dms = po.window_image(st, zero, s.win_left)
        b64 = po.born(st, m, dmp, dms, fx["wavelet"], s, "f64")
        b32 = po.born(st, m, dmp, dms, fx["wavelet"], s, "f32")
        for got, key, j in ((dz, "rec_vz", 0), (dx, "rec_vx", 1)):
            floor = rel(b32[j], b64[j])
            err = rel(got[i * ntr:(i + 1) * ntr], fx[key][i])
            assert err < gate(floor), (key, i, err, f"FP32 floor {floor:.3e}")


def _pml_case(nt=300):
    c = dict(allnx=64, allnz=36, nx=64, pml=12, nt=nt, dx=10.0, dz=10.0, dt=0.0008, f0=15.0)
    vp = np.broadcast_to(np.linspace(1800, 4500, c["allnz"], dtype=np.float32),
                         (c["allnx"], c["allnz"])).copy()
    w = synth.ricker(nt, c["f0"], c["dt"])
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    m = synth.reflectivity(c["allnx"], c["allnz"], seed=4, density=0.05, std=0.05)
    m[:, :3] = 0
    return c, vp, w, shots, m


def _pml_run(c, vp, w, shots, m, strips, rz=None, rx=None, opts=None):
    with Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="pml", strips=strips, max_shots=len(shots), max_ntr=c["nx"]) as e:
        for k, v in (opts or {}).items():
            e.set_option(k, v)
        e.set_models(vp, 0 * vp)
        e.set_wavelet(w)
        dz, dx = e.ac_born(shots, m)
        g = e.ac_born_adj(shots, dz if rz is None else rz, dx if rx is None else rx)
    return dz, dx, g


def test_ac_born_pml_vs_oracle_and_adjoint(cuda_device):
    """The acoustic Born pair with the reference's PML (split, damped update with mu = 0) and the
    background rebuilt on the interior from FP32 strips: L against the FP64 oracle, L^T against the
    oracle's exact transpose (which keeps the whole background history), and the dot-product test
    <L m, d> = <m, L^T d> in FP32."""
    c, vp, w, shots, m = _pml_case()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    rng = np.random.default_rng(3)
    ntr = shots[0].ntr
    rz = rng.normal(size=(len(shots) * ntr, c["nt"])).astype(np.float32)
    rx = rng.normal(size=rz.shape).astype(np.float32)
    dz, dx, g = _pml_run(c, vp, w, shots, m, "f32", rz, rx)
    gref = np.zeros((c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        model = po.build_model(st, vp, 0 * vp, None, s.win_left)
        assert model[5].max() > 0  # a damped PML
        oz, ox = po.ac_born(st, model, w, s, pad(st, m, s, c))
        assert rel(dz[i * ntr:(i + 1) * ntr], oz) < BORN_GATE
        assert rel(dx[i * ntr:(i + 1) * ntr], ox) < BORN_GATE
        gp = po.ac_born_adj(st, model, w, s, rz[i * ntr:(i + 1) * ntr], rx[i * ntr:(i + 1) * ntr])
        gref[s.win_left:s.win_left + c["nx"]] += gp[c["pml"]:c["pml"] + c["nx"], c["pml"]:-c["pml"]]
    assert rel(g, gref) < BORN_GATE, rel(g, gref)
    lhs = float(np.dot(dz.ravel().astype(np.float64), rz.ravel()) +
                np.dot(dx.ravel().astype(np.float64), rx.ravel()))
    rhs = float(np.dot(m.ravel().astype(np.float64), g.ravel()))
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("strips,gate", [("f16", 2e-3), ("bf16", 2e-2)])
def test_ac_born_adj_pml_half_precision_strips(cuda_device, strips, gate):
    """L^T with the background's boundary strips stored in FP16 / BF16 (one FP32 scale per
    32-cell segment) against the FP64 oracle's exact transpose: the error the storage format adds
    to the gradient (gates: FP16 2e-3, BF16 2e-2 relative L2)."""
    c, vp, w, shots, m = _pml_case()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    rng = np.random.default_rng(8)
    ntr = shots[0].ntr
    rz = rng.normal(size=(len(shots) * ntr, c["nt"])).astype(np.float32)
    rx = rng.normal(size=rz.shape).astype(np.float32)
    _, _, g16 = _pml_run(c, vp, w, shots, m, strips, rz, rx)
    gref = np.zeros((c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        model = po.build_model(st, vp, 0 * vp, None, s.win_left)
        gp = po.ac_born_adj(st, model, w, s, rz[i * ntr:(i + 1) * ntr], rx[i * ntr:(i + 1) * ntr])
        gref[s.win_left:s.win_left + c["nx"]] += gp[c["pml"]:c["pml"] + c["nx"], c["pml"]:-c["pml"]]
    err = rel(g16, gref)
    assert err < gate, f"{strips} strips: L^T vs FP64 oracle {err:.3e}"


@pytest.mark.parametrize("strips,gate_", [("f32", BORN_GATE), ("f16", 4e-3), ("bf16", 4e-2)])
def test_ac_born_adj_pml_checkpoints(cuda_device, strips, gate_):
    """L^T with the background checkpointed every 37 steps (option ac_ckpt: whole-state snapshots
    in the strip precision with one FP32 scale per field, shot and snapshot; each 37-step segment
    replayed from its snapshot with strips, then reversed; 300 steps give 8 full segments and a
    4-step one) against the FP64 oracle's exact transpose.  Each segment's reversal starts from
    the replayed forward state, where the all-strips path continues its own reversed background,
    so with FP32 snapshots the two gradients differ by rounding only (gate 1e-5).  With FP16 /
    BF16 both the snapshots and the strips are quantised: the gates are twice the strips-alone
    gates."""
    c, vp, w, shots, m = _pml_case()
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    rng = np.random.default_rng(8)
    ntr = shots[0].ntr
    rz = rng.normal(size=(len(shots) * ntr, c["nt"])).astype(np.float32)
    rx = rng.normal(size=rz.shape).astype(np.float32)
    _, _, g_ck = _pml_run(c, vp, w, shots, m, strips, rz, rx, opts={"ac_ckpt": 37})
    if strips == "f32":
        _, _, g_all = _pml_run(c, vp, w, shots, m, strips, rz, rx)
        assert rel(g_ck, g_all) < 1e-5, rel(g_ck, g_all)
    gref = np.zeros((c["allnx"], c["allnz"]))
    for i, s in enumerate(shots):
        model = po.build_model(st, vp, 0 * vp, None, s.win_left)
        gp = po.ac_born_adj(st, model, w, s, rz[i * ntr:(i + 1) * ntr], rx[i * ntr:(i + 1) * ntr])
        gref[s.win_left:s.win_left + c["nx"]] += gp[c["pml"]:c["pml"] + c["nx"], c["pml"]:-c["pml"]]
    err = rel(g_ck, gref)
    assert err < gate_, f"{strips} checkpoints + strips: L^T vs FP64 oracle {err:.3e}"


def test_ac_born_pml_vs_reference_golden(cuda_device):
    """The acoustic Born operator with the PML against the reference's own born_modeling (mode 1)
    with vs = 0 and its PML (tests/golden/born_acoustic_pml.npz), at the FP32 floor of the
    scheme."""
    from tests.helpers import case_of, gate, load, shots_of
    fx = load("born_acoustic_pml.npz")
    assert fx is not None, "golden fixture born_acoustic_pml.npz missing"
    c = case_of(fx)
    shots = shots_of(fx)
    st = po.Setup(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"], c["dt"])
    with Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="pml", max_shots=len(shots), max_ntr=max(s.ntr for s in shots)) as e:
        e.set_models(fx["vp"], fx["vs"])
        e.set_wavelet(fx["wavelet"])
        dz, dx = e.ac_born(shots, fx["img_pp"])
    ntr = shots[0].ntr
    zero = np.zeros_like(fx["img_pp"])
    for i, s in enumerate(shots):
        model = po.build_model(st, fx["vp"], fx["vs"], None, s.win_left)
        dmp = po.window_image(st, fx["img_pp"], s.win_left)
        b64 = po.born(st, model, dmp, po.window_image(st, zero, s.win_left), fx["wavelet"], s, "f64")
        b32 = po.born(st, model, dmp, po.window_image(st, zero, s.win_left), fx["wavelet"], s, "f32")
        for got, key, j in ((dz, "rec_vz", 0), (dx, "rec_vx", 1)):
            floor = rel(b32[j], b64[j])
            err = rel(got[i * ntr:(i + 1) * ntr], fx[key][i])
            assert err < gate(floor), (key, i, err, f"FP32 floor {floor:.3e}")

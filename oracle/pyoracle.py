"""Python binding of the CPU oracle (oracle/_build/libds2d_oracle.so) and of the reference
harness (oracle/_ref/libds2dref.so).  TEST INFRASTRUCTURE ONLY: used by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline and reference legs, always as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libds2d_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libds2dref.so")

fp = ctypes.POINTER(ctypes.c_float)
dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)


class OrcGrid(ctypes.Structure):
    _fields_ = [("nxpml", ctypes.c_int), ("nzpml", ctypes.c_int), ("pml", ctypes.c_int),
                ("nop", ctypes.c_int), ("dx", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float)]


class OrcShot(ctypes.Structure):
    _fields_ = [("isx", ctypes.c_int), ("isz", ctypes.c_int), ("igz", ctypes.c_int),
                ("ntr", ctypes.c_int), ("igx", ip)]


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_LIB


_orc = None


def lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build_oracle()
        L = ctypes.CDLL(ORACLE_LIB)
        G = ctypes.POINTER(OrcGrid)
        S = ctypes.POINTER(OrcShot)
        M = ctypes.POINTER(fp)
        L.orc_build_model.argtypes = [G, ctypes.c_int, ctypes.c_int, fp, fp, fp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_uint64, ctypes.c_int] + [fp] * 7
        L.orc_window_image.argtypes = [G, ctypes.c_int, ctypes.c_int, fp, ctypes.c_int, fp]
        L.orc_ricker.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, fp]
        L.orc_ricker.restype = None
        for p in ("f64", "f32"):
            getattr(L, f"orc_forward_{p}").argtypes = [G, M, fp, ctypes.c_int, S, dp, dp]
            getattr(L, f"orc_born_{p}").argtypes = [G, M, fp, fp, fp, ctypes.c_int, S, dp, dp]
            getattr(L, f"orc_elsrtm_{p}").argtypes = [G, M, fp, fp, fp, ctypes.c_int, S, fp, fp,
                                                       ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                       dp, dp, dp, dp, ctypes.POINTER(dp), dp]
            getattr(L, f"orc_rtm_{p}").argtypes = [G, M, fp, ctypes.c_int, S, fp, fp, ctypes.c_int,
                                                    ctypes.POINTER(dp)]
        L.orc_ac_born.argtypes = [G, M, fp, ctypes.c_int, S, dp, dp, dp]
        L.orc_ac_born_adj.argtypes = [G, M, fp, ctypes.c_int, S, dp, dp, dp]
        L.orc_ncc_residual.argtypes = [ctypes.c_int, ctypes.c_int, fp, fp, fp, fp, ctypes.c_int,
                                       dp, dp, dp]
        L.orc_ncc_residual.restype = None
        L.orc_adam_update.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(fp), fp, fp, dp,
                                      dp, dp, dp]
        L.orc_adam_update.restype = None
        L.orc_random_band_factor.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int]
        L.orc_random_band_factor.restype = ctypes.c_float
        _orc = L
    return _orc


def _f(a):
    return np.ascontiguousarray(a, np.float32)


def _p(a, t=fp):
    return None if a is None else a.ctypes.data_as(t)


class Setup:
    """Grid of a run in the oracle's terms."""

    def __init__(self, allnx, allnz, nx, pml, dx, dz, dt, nop=4):
        self.allnx, self.allnz, self.nx, self.pml = allnx, allnz, nx, pml
        self.g = OrcGrid(nx + 2 * pml, allnz + 2 * pml, pml, nop, dx, dz, dt)

    @property
    def shape(self):
        return (self.g.nxpml, self.g.nzpml)


def build_model(st, vp_all, vs_all, rho_all, win_left, rbc=0, seed=0, shot_id=0):
    """Padded per-shot model: vp, vs, rho, lam, mu, dampx, dampz ([nxpml][nzpml] each)."""
    out = [np.zeros(st.shape, np.float32) for _ in range(7)]
    rc = lib().orc_build_model(ctypes.byref(st.g), st.allnx, st.allnz, _p(_f(vp_all)),
                               _p(_f(vs_all)), _p(None if rho_all is None else _f(rho_all)),
                               win_left, rbc, seed, shot_id, *[_p(o) for o in out])
    if rc != 0:
        raise ValueError("orc_build_model: window outside the model")
    return out


def window_image(st, img_all, win_left):
    out = np.zeros(st.shape, np.float32)
    rc = lib().orc_window_image(ctypes.byref(st.g), st.allnx, st.allnz, _p(_f(img_all)), win_left,
                                _p(out))
    if rc != 0:
        raise ValueError("orc_window_image: window outside the model")
    return out


def _shot(s):
    gx = np.ascontiguousarray(s.igx, np.int32)
    return OrcShot(s.isx, s.isz, s.igz, len(gx), gx.ctypes.data_as(ip)), gx


def _model_ptrs(model):
    arrs = [_f(m) for m in model]
    ptrs = (fp * 7)(*[_p(a) for a in arrs])
    return ptrs, arrs


def forward(st, model, wavelet, shot, precision="f64"):
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    rz = np.zeros((shot.ntr, nt))
    rx = np.zeros((shot.ntr, nt))
    getattr(lib(), f"orc_forward_{precision}")(ctypes.byref(st.g), mp, _p(w), nt,
                                               ctypes.byref(sh), _p(rz, dp), _p(rx, dp))
    return rz, rx


def born(st, model, dm_p, dm_s, wavelet, shot, precision="f64"):
    """First-order elastic Born records (rec_vz, rec_vx) [ntr][nt] of one shot: the reference's
    born_modeling mode 1 (FD2DGPU.cu:1820-1831).  dm_p / dm_s are padded windows
    (window_image); with vs = 0 this is the acoustic Born operator of the elastic scheme."""
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    rz = np.zeros((shot.ntr, nt))
    rx = np.zeros((shot.ntr, nt))
    getattr(lib(), f"orc_born_{precision}")(ctypes.byref(st.g), mp, _p(_f(dm_p)), _p(_f(dm_s)),
                                            _p(w), nt, ctypes.byref(sh), _p(rz, dp), _p(rx, dp))
    return rz, rx


def elsrtm(st, model, dm_p, dm_s, wavelet, shot, obs_vz, obs_vx, iteration, rbc=0,
           precision="f64", adjoint_born=0):
    """Returns dict with lm_vz, lm_vx, res_vz, res_vx, images (7 window images), misfit.
    adjoint_born = 0 reproduces the reference's runs (scattered adjoint never excited)."""
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    recs = [np.zeros((shot.ntr, nt)) for _ in range(4)]
    imgs = [np.zeros((st.nx, st.allnz)) for _ in range(7)]
    iptr = (dp * 7)(*[_p(a, dp) for a in imgs])
    mis = ctypes.c_double(0.0)
    getattr(lib(), f"orc_elsrtm_{precision}")(
        ctypes.byref(st.g), mp, _p(_f(dm_p)), _p(_f(dm_s)), _p(w), nt, ctypes.byref(sh),
        _p(_f(obs_vz)), _p(_f(obs_vx)), iteration, rbc, adjoint_born, *[_p(r, dp) for r in recs], iptr,
        ctypes.byref(mis))
    return dict(lm_vz=recs[0], lm_vx=recs[1], res_vz=recs[2], res_vx=recs[3], images=imgs,
                misfit=mis.value)


def rtm(st, model, wavelet, shot, adj_vz, adj_vx, rbc=0, precision="f64"):
    """Returns the three window images (pp, ps, illumination), [nx][allnz] each."""
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    imgs = [np.zeros((st.nx, st.allnz)) for _ in range(3)]
    iptr = (dp * 3)(*[_p(a, dp) for a in imgs])
    getattr(lib(), f"orc_rtm_{precision}")(ctypes.byref(st.g), mp, _p(w), nt, ctypes.byref(sh),
                                           _p(_f(adj_vz)), _p(_f(adj_vx)), rbc, iptr)
    return imgs


def ac_born(st, model, wavelet, shot, m_pad):
    """Acoustic Born modelling L m of one shot (FP64): (rec_vz, rec_vx) [ntr][nt]."""
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    m = np.ascontiguousarray(m_pad, np.float64)
    rz, rx = np.zeros((shot.ntr, nt)), np.zeros((shot.ntr, nt))
    lib().orc_ac_born(ctypes.byref(st.g), mp, _p(w), nt, ctypes.byref(sh), _p(m, dp), _p(rz, dp),
                      _p(rx, dp))
    return rz, rx


def ac_born_adj(st, model, wavelet, shot, rz, rx):
    """Exact transpose L^T of ac_born for one shot: padded gradient [nxpml][nzpml] (FP64)."""
    sh, keep = _shot(shot)
    mp, keep2 = _model_ptrs(model)
    w = _f(wavelet)
    nt = len(w)
    g = np.zeros(st.shape)
    lib().orc_ac_born_adj(ctypes.byref(st.g), mp, _p(w), nt, ctypes.byref(sh),
                          _p(np.ascontiguousarray(rz, np.float64), dp),
                          _p(np.ascontiguousarray(rx, np.float64), dp), _p(g, dp))
    return g


def gaussian_bandpass(nx, nz, low, high):
    """construct_gaussian_bandpass_filter(filter, width = nz, height = nx, low, high) as the
    reference's bandpass_filter calls it (FD2DGPU.cu:4038-4077, :4135): FP32 distance with the
    width / height scale on the x offset, FP64 exponentials stored as FP32, clamped at 0,
    normalised to a maximum of 1; low == 0 is the low-pass form.  [nx][nz]."""
    cx, cy = nz // 2, nx // 2
    dz = (np.arange(nz) - cx)[None, :]
    dx = (np.arange(nx) - cy)[:, None]
    scale = np.float32(np.float32(nz) / np.float32(nx))
    t = (scale * dx.astype(np.float32)).astype(np.float32)
    dist = np.sqrt((dz * dz).astype(np.float32) + t * t).astype(np.float32)
    d2 = ((-dist) * dist).astype(np.float64)
    if low == 0:
        g = np.exp(d2 / (2.0 * high * high)).astype(np.float32)
    else:
        g = (np.exp(d2 / (2.0 * high * high)) - np.exp(d2 / (2.0 * low * low))).astype(np.float32)
    g = np.where(g < 0, np.float32(0), g).astype(np.float32)
    return (g / g.max()).astype(np.float32)


def quadrant_swap(a):
    """fft_shift / ifft_shift of FD2DGPU.cu:3922-3965 on [nx][nz]: quadrant (y, x) <-> (y + nx/2,
    x + nz/2) and (y, x + nz/2) <-> (y + nx/2, x) for y < nx/2, x < nz/2 (odd sizes keep the last
    row and column in place)."""
    nx, nz = a.shape
    hx, hz = nx // 2, nz // 2
    out = a.copy()
    out[:hx, :hz], out[hx:2 * hx, hz:2 * hz] = a[hx:2 * hx, hz:2 * hz], a[:hx, :hz]
    out[:hx, hz:2 * hz], out[hx:2 * hx, :hz] = a[hx:2 * hx, :hz], a[:hx, hz:2 * hz]
    return out


def bandpass(img, z1, z2):
    """The reference's bandpass_filter (FD2DGPU.cu:4125-4182) on one [nx][nz] image, step by
    step in FP64: FFT2 (cuFFT Z2Z forward, unnormalised), quadrant swap, multiply by the complex
    number (k, k) (GPU_lowpass), swap back, inverse FFT2, divide by nx*nz, real part as FP32."""
    nx, nz = img.shape
    k = gaussian_bandpass(nx, nz, z1, z2).astype(np.float64)
    f = np.fft.fft2(np.asarray(img, np.float64))
    f = quadrant_swap(f) * (k + 1j * k)
    g = np.fft.ifft2(quadrant_swap(f))  # numpy's inverse includes the 1 / (nx nz) of GPU_divide
    return g.real.astype(np.float32)


def ricker(nt, f0, dt):
    s = np.zeros(nt, np.float32)
    lib().orc_ricker(nt, f0, dt, _p(s))
    return s


def ncc_residual(syn_vz, syn_vx, obs_vz, obs_vx, iteration):
    ntr, nt = obs_vz.shape
    rz, rx = np.zeros((ntr, nt)), np.zeros((ntr, nt))
    mis = ctypes.c_double(0.0)
    lib().orc_ncc_residual(ntr, nt, _p(_f(syn_vz)), _p(_f(syn_vx)), _p(_f(obs_vz)),
                           _p(_f(obs_vx)), iteration, _p(rz, dp), _p(rx, dp), ctypes.byref(mis))
    return rz, rx, mis.value


def place(images_window, allnx, allnz, win_left):
    """Adds window images [nx][nz] into model-size images at column win_left."""
    out = np.zeros((allnx, allnz))
    nx = images_window.shape[0]
    out[win_left:win_left + nx] += images_window
    return out


# ---------------------------------------------------------------------------------------------
# Reference harness (the reference's own CUDA build; needs a GPU at call time).

_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} is missing (built by oracle/build_ref.sh)")
        L = ctypes.CDLL(REF_LIB)
        I, F = ctypes.c_int, ctypes.c_float
        L.ref_forward.argtypes = [I, I, I, I, I, F, F, F, fp, fp, fp, I, I, I, I, I, ip, fp, fp]
        L.ref_elsrtm.argtypes = [I, I, I, I, I, F, F, F, fp, fp, fp, fp, fp, I, I, I, I, I, ip, fp,
                                 fp, I, fp, fp, ctypes.POINTER(fp), dp, fp]
        L.ref_rtm.argtypes = [I, I, I, I, I, F, F, F, fp, fp, fp, I, ip, ip, I, I, I, ip, fp, fp, I,
                              fp, fp, ctypes.POINTER(fp), fp]
        L.ref_born.argtypes = [I, I, I, I, I, F, F, F, fp, fp, fp, fp, fp, I, I, I, I, I, ip, I,
                               fp, fp, fp, fp]
        L.ref_release.argtypes = []
        L.ref_bandpass.argtypes = [I, I, I, I, I, I, fp, fp]
        L.ref_cpu_acoustic.argtypes = [I, I, I, F, F, F, fp, fp, fp, I, I, fp, fp, dp]
        _ref = L
    return _ref


def ref_forward(allnx, allnz, nx, pml, nt, dx, dz, dt, vp, vs, wavelet, shot):
    gx = np.ascontiguousarray(shot.igx, np.int32)
    rz = np.zeros((len(gx), nt), np.float32)
    rx = np.zeros((len(gx), nt), np.float32)
    rc = ref_lib().ref_forward(allnx, allnz, nx, pml, nt, dx, dz, dt, _p(_f(vp)), _p(_f(vs)),
                               _p(_f(wavelet)), shot.win_left, shot.isx, shot.isz, shot.igz,
                               len(gx), _p(gx, ip), _p(rz), _p(rx))
    if rc != 0:
        raise RuntimeError(f"ref_forward: CUDA error {rc}")
    return rz, rx


def ref_born(allnx, allnz, nx, pml, nt, dx, dz, dt, vp, vs, wavelet, img_pp, img_ps, shot,
             rbc=0, vp_pad=None, vs_pad=None):
    """First-order Born records (rec_vz, rec_vx) of one shot by the reference's own kernels
    (born_modeling mode 1); rbc = 1 injects the padded model vp_pad / vs_pad with zero damping."""
    gx = np.ascontiguousarray(shot.igx, np.int32)
    rz = np.zeros((len(gx), nt), np.float32)
    rx = np.zeros((len(gx), nt), np.float32)
    rc = ref_lib().ref_born(allnx, allnz, nx, pml, nt, dx, dz, dt, _p(_f(vp)), _p(_f(vs)),
                            _p(_f(wavelet)), _p(_f(img_pp)), _p(_f(img_ps)), shot.win_left,
                            shot.isx, shot.isz, shot.igz, len(gx), _p(gx, ip), int(rbc),
                            _p(None if vp_pad is None else _f(vp_pad)),
                            _p(None if vs_pad is None else _f(vs_pad)), _p(rz), _p(rx))
    if rc != 0:
        raise RuntimeError(f"ref_born: CUDA error {rc}")
    return rz, rx


def ref_bandpass(img_pp, img_ps, z1, z2, x1=0, x2=0):
    """The reference's own bandpass_filter (cuFFT) on two [nx][nz] images; returns copies."""
    pp = np.array(img_pp, np.float32, order="C")
    ps = np.array(img_ps, np.float32, order="C")
    nx, nz = pp.shape
    rc = ref_lib().ref_bandpass(nx, nz, x1, x2, z1, z2, _p(pp), _p(ps))
    if rc != 0:
        raise RuntimeError(f"ref_bandpass: CUDA error {rc}")
    return pp, ps


def ref_cpu_acoustic(vp_pad, rho_pad, damp_pad, wavelet, isx, isz, dt, dx, dz):
    """The reference's own CPU acoustic stepper (main.cpp:602-727, OpenMP, all host threads)
    driven for len(wavelet) steps with the source split over px, pz at (isx, isz); padded
    [nxpml][nzpml] inputs.  Returns (final p, seconds)."""
    nxpml, nzpml = vp_pad.shape
    out = np.zeros((nxpml, nzpml), np.float32)
    sec = ctypes.c_double(0.0)
    w = _f(wavelet)
    rc = ref_lib().ref_cpu_acoustic(nxpml, nzpml, len(w), dt, dx, dz, _p(_f(vp_pad)),
                                    _p(_f(rho_pad)), _p(_f(damp_pad)), isx, isz, _p(w), _p(out),
                                    ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError(f"ref_cpu_acoustic: {rc}")
    return out, sec.value


def ref_release():
    """Frees the reference object the harness keeps between calls."""
    if _ref is not None:
        _ref.ref_release()


def ref_elsrtm(allnx, allnz, nx, pml, nt, dx, dz, dt, vp, vs, wavelet, img_pp, img_ps, shot,
               obs_vz, obs_vx, iteration):
    gx = np.ascontiguousarray(shot.igx, np.int32)
    res_z = np.zeros((len(gx), nt), np.float32)
    res_x = np.zeros((len(gx), nt), np.float32)
    imgs = [np.zeros((allnx, allnz), np.float32) for _ in range(7)]
    iptr = (fp * 7)(*[_p(a) for a in imgs])
    mis = ctypes.c_double(0.0)
    ms = ctypes.c_float(0)
    rc = ref_lib().ref_elsrtm(allnx, allnz, nx, pml, nt, dx, dz, dt, _p(_f(vp)), _p(_f(vs)),
                              _p(_f(wavelet)), _p(_f(img_pp)), _p(_f(img_ps)), shot.win_left,
                              shot.isx, shot.isz, shot.igz, len(gx), _p(gx, ip), _p(_f(obs_vz)),
                              _p(_f(obs_vx)), iteration, _p(res_z), _p(res_x), iptr,
                              ctypes.byref(mis), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_elsrtm: CUDA error {rc}")
    # elapsed_ms: CUDA-event time of the reference's per-shot driver call alone
    return dict(res_vz=res_z, res_vx=res_x, images=imgs, misfit=mis.value, elapsed_ms=ms.value)


def ref_rtm(allnx, allnz, nx, pml, nt, dx, dz, dt, vp, vs, wavelet, shots, adj_vz, adj_vx,
            rbc=0, vp_pad=None, vs_pad=None):
    """Shots share ntr, isz and igz (the reference's layout).  Returns (images, elapsed_ms)."""
    ntr = shots[0].ntr
    wl = np.array([s.win_left for s in shots], np.int32)
    isx = np.array([s.isx for s in shots], np.int32)
    gx = np.ascontiguousarray(np.concatenate([s.igx for s in shots]), np.int32)
    imgs = [np.zeros((allnx, allnz), np.float32) for _ in range(3)]
    iptr = (fp * 3)(*[_p(a) for a in imgs])
    ms = ctypes.c_float(0)
    rc = ref_lib().ref_rtm(allnx, allnz, nx, pml, nt, dx, dz, dt, _p(_f(vp)), _p(_f(vs)),
                           _p(_f(wavelet)), len(shots), _p(wl, ip), _p(isx, ip), shots[0].isz,
                           shots[0].igz, ntr, _p(gx, ip), _p(_f(adj_vz)), _p(_f(adj_vx)), rbc,
                           _p(None if vp_pad is None else _f(vp_pad)),
                           _p(None if vs_pad is None else _f(vs_pad)), iptr, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_rtm: CUDA error {rc}")
    return imgs, ms.value

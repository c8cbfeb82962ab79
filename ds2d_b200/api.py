"""Python host mirror of the DS2D elastic path over the C ABI (include/ds2d.h).

`Elastic2D` owns one device context (the reference's FD2DGPU_ELASTIC object,
FD2DGPU.cuh:124-422) and exposes the same operations: loading models and the reflectivity image,
forward modelling, reference-mode ELSRTM and elastic RTM of batches of shots, and read-out of the
accumulated gradient images.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class ShotGeom:
    """One shot in cells of the padded window (reference main.cpp:1019-1025).

    win_left: model column of the window's first interior column (delta_left + record_left_in_v)
    isx, isz: source cell; igz: receiver row; igx: receiver columns (distinct);
    nx: this shot's window width (0 = the context's nx).
    """
    win_left: int
    isx: int
    isz: int
    igz: int
    igx: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    nx: int = 0

    @property
    def ntr(self):
        return int(len(self.igx))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Elastic2D:
    """Device context for one grid (allnx x allnz model, nx-wide shot windows, pml cells)."""

    def __init__(self, allnx, allnz, nx, pml, nt, dx, dz, dt, boundary="pml", strips="f32",
                 max_shots=1, max_ntr=None, seed=0, device=0):
        self.lib = _lib.load()
        self.allnx, self.allnz, self.nx, self.pml, self.nt = allnx, allnz, nx, pml, nt
        self.nxpml, self.nzpml = nx + 2 * pml, allnz + 2 * pml
        self.dx, self.dz, self.dt = dx, dz, dt
        self.max_shots = max_shots
        self.max_ntr = nx if max_ntr is None else max_ntr
        g = _lib.Grid(allnx, allnz, nx, pml, nt, dx, dz, dt)
        o = _lib.Opts(_lib.BOUNDARY[boundary], _lib.STRIPS[strips], max_shots, self.max_ntr,
                      seed, device)
        h = ctypes.c_void_p()
        rc = self.lib.ds2d_create(ctypes.byref(g), ctypes.byref(o), ctypes.byref(h))
        if rc != 0:
            raise _lib.DS2DError(rc, self.lib.ds2d_last_error(None).decode())
        self.h = h
        self._keep = []

    # -- lifetime -------------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.ds2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise _lib.DS2DError(rc, self.lib.ds2d_last_error(self.h).decode())

    # -- inputs ---------------------------------------------------------------------------
    def set_stream(self, stream_handle):
        """Launch stream as an integer cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self.lib.ds2d_set_stream(self.h, ctypes.c_void_p(stream_handle or None)))

    def set_models(self, vp, vs, rho=None):
        vp, vs = _f32(vp), _f32(vs)
        assert vp.shape == (self.allnx, self.allnz) and vs.shape == vp.shape
        r = None if rho is None else _f32(rho)
        self._check(self.lib.ds2d_set_models(self.h, _fptr(vp), _fptr(vs),
                                             None if r is None else _fptr(r)))

    def set_wavelet(self, w):
        w = _f32(w)
        assert w.shape == (self.nt,)
        self._check(self.lib.ds2d_set_wavelet(self.h, _fptr(w)))

    def set_image(self, pp, ps):
        pp, ps = _f32(pp), _f32(ps)
        assert pp.shape == (self.allnx, self.allnz) and ps.shape == pp.shape
        self._check(self.lib.ds2d_set_image(self.h, _fptr(pp), _fptr(ps)))

    # -- shots ----------------------------------------------------------------------------
    def _shots(self, shots):
        arr = (_lib.Shot * len(shots))()
        keep = []
        for i, s in enumerate(shots):
            gx = np.ascontiguousarray(s.igx, dtype=np.int32)
            keep.append(gx)
            arr[i] = _lib.Shot(int(s.win_left), int(s.isx), int(s.isz), int(s.igz), len(gx),
                               gx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               int(getattr(s, "nx", 0)))
        return arr, keep

    def _rec(self, shots):
        ntr = sum(s.ntr for s in shots)
        return np.zeros((ntr, self.nt), np.float32)

    def forward(self, shots):
        """Background modelling; returns (rec_vz, rec_vx), each [sum ntr][nt]."""
        arr, keep = self._shots(shots)
        rz, rx = self._rec(shots), self._rec(shots)
        self._check(self.lib.ds2d_forward(self.h, arr, len(shots), _fptr(rz), _fptr(rx)))
        return rz, rx

    def elsrtm(self, shots, obs_vz, obs_vx, iteration, want_records=False):
        """Reference-mode ELSRTM; gradients accumulate on the device.  Returns the misfit
        increment (and Lm + Lm2 and the adjoint source when want_records)."""
        arr, keep = self._shots(shots)
        oz, ox = _f32(obs_vz), _f32(obs_vx)
        mis = ctypes.c_double(0.0)
        lz = lx = rz = rx = None
        if want_records:
            lz, lx, rz, rx = (self._rec(shots) for _ in range(4))
        p = lambda a: None if a is None else _fptr(a)
        self._check(self.lib.ds2d_elsrtm(self.h, arr, len(shots), _fptr(oz), _fptr(ox),
                                         int(iteration), ctypes.byref(mis), p(lz), p(lx), p(rz),
                                         p(rx)))
        if want_records:
            return mis.value, (lz, lx, rz, rx)
        return mis.value

    def elsrtm_device(self, shots, obs_vz_ptr, obs_vx_ptr, iteration):
        """Reference-mode ELSRTM with the observed records in device memory (integer device
        pointers, [sum ntr][nt] each); returns the misfit increment."""
        arr, keep = self._shots(shots)
        mis = ctypes.c_double(0.0)
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.ds2d_elsrtm(self.h, arr, len(shots), ctypes.cast(obs_vz_ptr, fp),
                                         ctypes.cast(obs_vx_ptr, fp), int(iteration),
                                         ctypes.byref(mis), None, None, None, None))
        return mis.value

    def rtm(self, shots, adj_vz, adj_vx):
        """Elastic RTM of the given shots with adj_* injected at the receivers."""
        arr, keep = self._shots(shots)
        az, ax = _f32(adj_vz), _f32(adj_vx)
        self._check(self.lib.ds2d_rtm(self.h, arr, len(shots), _fptr(az), _fptr(ax)))

    def rtm_device(self, shots, adj_vz_ptr, adj_vx_ptr):
        """RTM with the adjoint source already in device memory (integer device pointers)."""
        arr, keep = self._shots(shots)
        self._check(self.lib.ds2d_rtm_device(self.h, arr, len(shots), ctypes.c_void_p(adj_vz_ptr),
                                             ctypes.c_void_p(adj_vx_ptr)))

    def dot_f64(self, a_ptr, b_ptr, n):
        """FP64 <a, b> of two float device vectors (integer device pointers)."""
        out = ctypes.c_double(0.0)
        self._check(self.lib.ds2d_dot_f64(self.h, ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr),
                                          int(n), ctypes.byref(out)))
        return out.value

    # -- acoustic Born pair and CG-LSRTM (context built with boundary="random", vs = 0) ------
    def ac_born(self, shots, m):
        """d = L m: scattered vz, vx of the acoustic Born operator, each [sum ntr][nt]."""
        arr, keep = self._shots(shots)
        m = _f32(m)
        rz, rx = self._rec(shots), self._rec(shots)
        self._check(self.lib.ds2d_ac_born(self.h, arr, len(shots), _fptr(m), _fptr(rz), _fptr(rx)))
        return rz, rx

    def ac_born_adj(self, shots, rec_vz, rec_vx):
        """g = L^T d, the exact transpose of ac_born ([allnx][allnz])."""
        arr, keep = self._shots(shots)
        rz, rx = _f32(rec_vz), _f32(rec_vx)
        g = np.zeros((self.allnx, self.allnz), np.float32)
        self._check(self.lib.ds2d_ac_born_adj(self.h, arr, len(shots), _fptr(rz), _fptr(rx), _fptr(g)))
        return g

    def lsrtm(self, shots, obs_vz, obs_vx, niter, target=0.0):
        """CGLS on ||L m - d||^2 from m = 0: returns (m, relative residual after each iteration)."""
        arr, keep = self._shots(shots)
        oz, ox = _f32(obs_vz), _f32(obs_vx)
        m = np.zeros((self.allnx, self.allnz), np.float32)
        hist = np.zeros(max(niter, 1))
        done = ctypes.c_int(0)
        self._check(self.lib.ds2d_lsrtm(self.h, arr, len(shots), _fptr(oz), _fptr(ox), int(niter),
                                        float(target), _fptr(m),
                                        hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        ctypes.byref(done)))
        return m, hist[:done.value]

    def ac_normal_device(self, shots, m_ptr, img_ptr):
        """img = L^T L m on model-size device arrays (integer device pointers)."""
        arr, keep = self._shots(shots)
        self._check(self.lib.ds2d_ac_normal(self.h, arr, len(shots), ctypes.c_void_p(m_ptr),
                                            ctypes.c_void_p(img_ptr)))

    def ac_born_device(self, shots, m_ptr, rz_ptr, rx_ptr):
        """d = L m with m and the records [sum ntr][nt] in device memory."""
        arr, keep = self._shots(shots)
        fpp = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.ds2d_ac_born(self.h, arr, len(shots), ctypes.cast(m_ptr, fpp),
                                          ctypes.cast(rz_ptr, fpp), ctypes.cast(rx_ptr, fpp)))

    def ac_born_adj_device(self, shots, rz_ptr, rx_ptr, g_ptr):
        """g = L^T d with the records [sum ntr][nt] and g in device memory."""
        arr, keep = self._shots(shots)
        fpp = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.ds2d_ac_born_adj(self.h, arr, len(shots), ctypes.cast(rz_ptr, fpp),
                                              ctypes.cast(rx_ptr, fpp), ctypes.cast(g_ptr, fpp)))

    def lsrtm_pcg(self, shots, obs_vz_ptr, obs_vx_ptr, m_ptr, niter, target=0.0, net=None):
        """Flexible preconditioned CG-LSRTM on device arrays; net = ds2d_b200.unet.UNet or None
        (plain CG).  Returns (relative residual per iteration, wall ms per iteration)."""
        arr, keep = self._shots(shots)
        hist = np.zeros(max(niter, 1))
        ms = np.zeros(max(niter, 1))
        done = ctypes.c_int(0)
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.ds2d_lsrtm_pcg(
            self.h, net.h if net is not None else None, arr, len(shots), ctypes.c_void_p(obs_vz_ptr),
            ctypes.c_void_p(obs_vx_ptr), int(niter), float(target), ctypes.c_void_p(m_ptr),
            hist.ctypes.data_as(dp), ms.ctypes.data_as(dp), ctypes.byref(done)))
        return hist[:done.value], ms[:done.value]

    IMAGE_NAMES =("pp_grad", "ps_grad", "illumination", "b_pp", "b_ps", "b_pp2", "b_ps2")

    def read_images(self, reset=True, which=None):
        """imagebuffer_resettozero: the accumulated images as [allnx][allnz] arrays."""
        which = self.IMAGE_NAMES if which is None else which
        out = {k: np.zeros((self.allnx, self.allnz), np.float32) for k in which}
        ptrs = (ctypes.POINTER(ctypes.c_float) * 7)()
        for i, k in enumerate(self.IMAGE_NAMES):
            ptrs[i] = _fptr(out[k]) if k in out else ctypes.POINTER(ctypes.c_float)()
        self._check(self.lib.ds2d_read_images(self.h, ptrs, int(bool(reset))))
        return out

    def read_images_device(self, out, reset=True, which=None):
        """Device read-out: copies the named images into `out` (a CUDA tensor [len(which)][allnx]
        [allnz], FP32) on the context stream, then zeroes them when reset."""
        which = self.IMAGE_NAMES if which is None else which
        if tuple(out.shape) != (len(which), self.allnx, self.allnz) or not out.is_contiguous():
            raise ValueError("out must be a contiguous [len(which)][allnx][allnz] tensor")
        ptrs = (ctypes.c_void_p * 7)()
        plane = self.allnx * self.allnz * 4
        for i, k in enumerate(which):
            ptrs[self.IMAGE_NAMES.index(k)] = out.data_ptr() + i * plane
        self._check(self.lib.ds2d_read_images_device(self.h, ptrs, int(bool(reset))))
        return out

    def set_option(self, key, value):
        """Tuning knob by name ("fused", "xr", "ring", "occ", "cta", "graph", "pair", "pair_xr",
        "ac_pair", ...; the list and ranges are documented at ds2d_set_option in ds2d.h)."""
        self._check(self.lib.ds2d_set_option(self.h, key.encode(), int(value)))

    def profile(self, enable=True):
        """Per-launch CUDA-event timing of every kernel from now on (adds small overhead)."""
        self._check(self.lib.ds2d_profile(self.h, int(bool(enable))))

    def profile_report(self):
        """{kernel: (launches, total_ms, algorithmic_bytes)} since the last report."""
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self.lib.ds2d_profile_report(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms, by = line.split()
            out[name] = (int(n), float(ms), float(by))
        return out

    @property
    def last_cell_updates(self):
        return self.lib.ds2d_last_cell_updates(self.h)

    @property
    def last_launches(self):
        return self.lib.ds2d_last_launches(self.h)


def bandpass_filter(grad_pp, grad_ps, z1, z2, x1=0, x2=0):
    """Band-pass filter of two [nx][nz] gradient images (reference bandpass_filter,
    FD2DGPU.cu:4125-4182) on the GPU; returns the filtered copies.  z1 = low cut-off (0: low-pass),
    z2 = high cut-off; x1, x2 are unused, as in the reference's live filter."""
    lib = _lib.load()
    pp = _f32(grad_pp).copy()
    ps = _f32(grad_ps).copy()
    nx, nz = pp.shape
    rc = lib.ds2d_bandpass_filter(nx, nz, int(x1), int(x2), int(z1), int(z2), _fptr(pp), _fptr(ps))
    if rc != 0:
        raise _lib.DS2DError(rc, lib.ds2d_last_error(None).decode())
    return pp, ps


def bandpass_filter_device(pp_ptr, ps_ptr, nx, nz, z1, z2, stream=0, x1=0, x2=0):
    """In-place band-pass of two device images (either pointer may be 0) on `stream`."""
    lib = _lib.load()
    rc = lib.ds2d_bandpass_filter_device(nx, nz, int(x1), int(x2), int(z1), int(z2),
                                         ctypes.c_void_p(pp_ptr or None),
                                         ctypes.c_void_p(ps_ptr or None), ctypes.c_void_p(stream))
    if rc != 0:
        raise _lib.DS2DError(rc, lib.ds2d_last_error(None).decode())

"""Gradient band-pass filter (reference bandpass_filter, FD2DGPU.cu:4125-4182) on the GPU against
the FP64 restatement of the reference's steps and against the reference's own cuFFT results."""
import numpy as np
import pytest

from ds2d_b200.api import bandpass_filter, bandpass_filter_device
from oracle import pyoracle as po
from tests.helpers import load, rel

pytestmark = pytest.mark.gpu

# FP64 transforms stored as FP32: the GPU's DFT products, numpy's FFT and cuFFT round the FP64
# intermediates differently, which reaches the FP32 results at the last-bit level only.
TOL = 1e-6


@pytest.mark.parametrize("nx,nz,z1,z2", [(1201, 401, 0, 80), (1201, 401, 20, 80), (81, 41, 3, 12),
                                         (64, 32, 0, 6)])
def test_bandpass_vs_oracle(cuda_device, nx, nz, z1, z2):
    rng = np.random.default_rng(nx + z1)
    pp = rng.standard_normal((nx, nz)).astype(np.float32)
    ps = rng.standard_normal((nx, nz)).astype(np.float32)
    fpp, fps = bandpass_filter(pp, ps, z1, z2)
    assert rel(fpp, po.bandpass(pp, z1, z2)) < TOL
    assert rel(fps, po.bandpass(ps, z1, z2)) < TOL
    assert np.array_equal(pp, pp)  # inputs untouched (copies are filtered)


def test_bandpass_device_in_place(cuda_device):
    import torch
    rng = np.random.default_rng(5)
    img = rng.standard_normal((121, 41)).astype(np.float32)
    d = torch.from_numpy(img).cuda()
    torch.cuda.synchronize()
    bandpass_filter_device(d.data_ptr(), 0, 121, 41, 0, 10)
    assert rel(d.cpu().numpy(), po.bandpass(img, 0, 10)) < TOL


def test_bandpass_vs_reference_golden(cuda_device):
    fx = load("bandpass.npz")
    assert fx is not None, "golden fixture bandpass.npz missing"
    for i, (nx, nz, z1, z2) in enumerate(fx["cases"]):
        fpp, fps = bandpass_filter(fx[f"in_pp{i}"], fx[f"in_ps{i}"], int(z1), int(z2))
        assert rel(fpp, fx[f"out_pp{i}"]) < TOL, (i, rel(fpp, fx[f"out_pp{i}"]))
        assert rel(fps, fx[f"out_ps{i}"]) < TOL, (i, rel(fps, fx[f"out_ps{i}"]))


def test_bandpass_rejects_bad_arguments(cuda_device):
    from ds2d_b200._lib import DS2DError
    with pytest.raises(DS2DError):
        bandpass_filter(np.zeros((8, 8), np.float32), np.zeros((8, 8), np.float32), 0, 0)

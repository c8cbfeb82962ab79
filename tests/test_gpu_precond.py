"""What the trained network gains: on a small acoustic survey, a U-Net trained on the GPU (by the
package's own BF16 kernels, on CG-trajectory pairs this code generates) makes preconditioned
LSRTM reach a lower Born-data residual than plain CG after the same number of iterations, on a
reflectivity it was not trained on."""
import numpy as np
import pytest

from ds2d_b200 import Elastic2D, precond, synth

pytestmark = pytest.mark.gpu


def test_trained_network_beats_plain_cg(cuda_device):
    import torch
    from ds2d_b200.unet import UNet, he_normal
    nx, nz, band, nt, dx, dt = 96, 48, 12, 500, 10.0, 0.0008
    shots = synth.surface_shots(nx, nx, band, 8)
    with Elastic2D(nx, nz, nx, band, nt, dx, dx, dt, boundary="random", max_shots=len(shots),
                   max_ntr=nx, seed=3) as e:
        vp = precond.background(nx, nz, seed=1)
        e.set_models(vp, np.zeros_like(vp))
        e.set_wavelet(synth.ricker(nt, 15.0, dt))
        X, Y = precond.make_trajectory_pairs(e, shots, nmodels=8, iters=8, seed=5)
        with UNet(max_n=8, max_h=nx, max_w=nz) as net:
            net.set_params(he_normal(2))
            hist = precond.train(net, X, Y, steps=800, batch=8, crop=(48, None), lr=1e-3)
            assert hist[-1] < 0.8 * hist[0]
            # held-out reflectivity (the configs' sparse kind), Born data by the same operator
            rng = np.random.default_rng(99)
            m_true = torch.from_numpy(precond.random_reflectivity(nx, nz, rng, reflectors=0)).cuda()
            ntr = sum(s.ntr for s in shots)
            dz = torch.zeros((ntr, nt), device="cuda")
            dxr = torch.zeros_like(dz)
            e.ac_born_device(shots, m_true.data_ptr(), dz.data_ptr(), dxr.data_ptr())
            m = torch.zeros_like(m_true)
            plain, _ = e.lsrtm_pcg(shots, dz.data_ptr(), dxr.data_ptr(), m.data_ptr(), 4)
            m.zero_()
            learned, _ = e.lsrtm_pcg(shots, dz.data_ptr(), dxr.data_ptr(), m.data_ptr(), 4, net=net)
    assert np.all(np.diff(learned) < 0)
    # the gain: a clearly lower residual after the first iterations
    assert learned[0] < 0.95 * plain[0], (learned, plain)
    assert learned[-1] < plain[-1], (learned, plain)

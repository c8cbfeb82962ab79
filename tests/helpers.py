"""Shared helpers of the parity tests: fixtures, geometry and the parity gates."""
import os

import numpy as np

from ds2d_b200.api import ShotGeom

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Gate of the path: 1e-5 relative L2 in FP32.  Outputs built from the Born (scattered) fields
# are reproducible only to the FP32 rounding floor of the scheme itself (the same FP32 code with
# a different FMA contraction moves them by ~3e-4 on records, ~6e-5 on gradients), so their
# gate is a multiple of that floor, measured per case as |oracle_f32 - oracle_f64|.
GATE = 1e-5
FLOOR_FACTOR = 4.0


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def gate(floor=0.0):
    return max(GATE, FLOOR_FACTOR * floor)


def load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        return None
    return dict(np.load(path))


def case_of(fx):
    allnx, allnz, nx, pml, nt = (int(v) for v in fx["case"])
    dx, dz, dt, f0 = (float(v) for v in fx["steps"])
    return dict(allnx=allnx, allnz=allnz, nx=nx, pml=pml, nt=nt, dx=dx, dz=dz, dt=dt, f0=f0)


def shots_of(fx):
    return [ShotGeom(int(fx["win_left"][i]), int(fx["isx"][i]), int(fx["isz"][i]),
                     int(fx["igz"][i]), fx["igx"][i].astype(np.int32))
            for i in range(len(fx["win_left"]))]


def small_case(nt=300):
    """A small elastic case the oracle replays in well under a second."""
    from ds2d_b200 import synth
    c = dict(allnx=72, allnz=36, nx=56, pml=10, nt=nt, dx=10.0, dz=10.0, dt=0.0008, f0=15.0)
    vp, vs = synth.layered(c["allnx"], c["allnz"], seed=3)
    w = synth.ricker(nt, c["f0"], c["dt"])
    shots = synth.surface_shots(c["allnx"], c["nx"], c["pml"], 3)
    return c, vp, vs, w, shots

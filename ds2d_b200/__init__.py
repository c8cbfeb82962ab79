"""B200-native DS2D time-stepping path: elastic staggered-grid modelling, Born modelling, RTM and
reference-mode ELSRTM on hand-written sm_100a CUDA kernels behind a C ABI (include/ds2d.h)."""
from .api import Elastic2D, ShotGeom  # noqa: F401
from ._lib import DS2DError  # noqa: F401

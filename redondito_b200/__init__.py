"""redondito_b200: B200-native (sm_100a) pseudospectral transform core for
spherical shells -- scalar/vector spherical-harmonic transforms on a
Gauss-Legendre grid, the FC-Gram Fourier-continuation radial transform and
its operators, no-slip boundary imposition and the nonlinear-term/RK3 step.

The compute lives in redondito_b200/_lib/libsph_b200.so behind the C ABI of
include/sph_b200.h; redondito_b200.sphp mirrors the reference's Fortran
routine names over it.
"""
from . import build  # noqa: F401

__all__ = ["build", "sphp"]

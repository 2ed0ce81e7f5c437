"""B200-native finite-volume step of ExoCubed's cubed-sphere dynamical core.

The compute path is hand-written CUDA for sm_100a in libexo_b200.so, reached
through the C ABI of include/exo_b200.h.  This package is the host-side
mirror of the reference's operator interface (see atmosphere.py) plus the
seeded synthetic workloads used by the tests and the benchmark.
"""
from . import _native  # noqa: F401
from .atmosphere import CubedSphereAtmosphere, cell_geometry, make_config, riemann_rows  # noqa: F401

__all__ = ["CubedSphereAtmosphere", "cell_geometry", "make_config", "riemann_rows"]

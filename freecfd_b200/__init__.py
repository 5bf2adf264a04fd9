"""freecfd_b200 — B200-native (sm_100a) residual path of Free CFD.

The unstructured finite-volume residual of Free CFD's navier_stokes module
(LSQ / Green-Gauss gradients, limiters, Roe / AUSM+up / Van Leer / SD-SLAU /
Steger-Warming fluxes, viscous fluxes,
boundary conditions, local time step) as hand-written CUDA kernels behind the
C ABI in include/fcfd.h.  Importing this package loads libfcfd_b200.so; there
is no CPU fallback.
"""
from ._lib import FcfdError, LIB_PATH, build, lib  # noqa: F401
from .solver import Case, Mesh, NavierStokes, point_flux, read_restart, write_restart  # noqa: F401
from . import cases  # noqa: F401

FLUX = {"Roe": 1, "vanLeer": 2, "AUSM+up": 3, "SD-SLAU": 4, "SW": 5}

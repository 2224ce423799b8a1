"""B200-native TWoS (Topological Walk on Spheres) estimator.

A drop-in for the compiled Embree/OpenMP backend of hertjo/walking-into-holes:
geometry and query sites in; per-site primal/adjoint values, the cross-index
topological derivative, its jackknife standard error and step statistics out.
The work runs in hand-written sm_100a kernels of libtwos.so (C ABI in
include/twos.h); this package is the host side.
"""
from ._abi import (MODE_COMPLIANCE, MODE_HOT, MODE_PAIRED, PREC_FP64, PREC_MIXED, SITE_DTYPE, TwosError, load)
from .mesh import Config, Mesh, ball_green_integral, estimate_batch, l2_read_gbs, sobol_directions
from . import sources, geometry, shard

__all__ = ["Config", "Mesh", "estimate_batch", "ball_green_integral", "l2_read_gbs", "sobol_directions", "TwosError",
           "load", "sources", "geometry", "shard", "SITE_DTYPE", "MODE_COMPLIANCE", "MODE_PAIRED", "MODE_HOT", "PREC_FP64", "PREC_MIXED"]

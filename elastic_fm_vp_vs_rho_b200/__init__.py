"""B200-native elastic FDTD / FWI with moment tensors.

A from-scratch sm_100a implementation of the hot path of jheyston/Elastic_FM_Vp_Vs_Rho:
3-D isotropic-elastic velocity-stress staggered-grid FDTD with CPML and a moment-tensor
source, adjoint gradients for lambda/mu/rho (Vp/Vs/rho) and the six moment-tensor
components, and the L-BFGS update -- behind the reference's driver surface
(``Elastic3D``, ``lbfgs.compute_sk_yk`` / ``lbfgs.L_BFGS``).

Compute runs in ``libefm.so`` (hand-written CUDA, C ABI in ``include/efm.h``); there is
no CPU fallback.
"""
from .elastic3d import (CPML, Alpha, Earthquake, Elastic3D, Gather, Geometry, Gradients,  # noqa: F401
                        Model, Station, StressTensor, Wavelet, multifrequency_fwi,
                        observed_data)
from .engine import ShotBatch, chain_rule, dot, smooth_mask  # noqa: F401
from .lbfgs import L_BFGS, compute_sk_yk  # noqa: F401
from ._lib import EfmError  # noqa: F401

__version__ = "0.1.0"

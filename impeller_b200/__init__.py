"""B200-native (sm_100a) BN254 G1 multi-scalar multiplication.

A drop-in for the MSM operator of SJTU-Liquid/Impeller's core crate
(core/src/msm.rs over core/src/msm/src/msm.h), plus a resident-SRS context,
batched CUDA-graph MSMs and a continuous-batching serving loop.  All
arithmetic runs in libimpeller_msm.so; importing this package does not load
it (see impeller_b200.lib.load).
"""
from .lib import ImpellerError, load  # noqa: F401

__all__ = ["ImpellerError", "load"]

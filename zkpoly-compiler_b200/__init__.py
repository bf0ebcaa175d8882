"""zkpoly_b200: a B200-native (sm_100a) drop-in for zkpoly's BN254 hot path.

The CUDA libraries in lib/ export the reference's C ABI (NTT, MSM, poly, fused kernels);
these modules are the host-side mirror of the reference's Rust operator wrappers.  torch
provides device memory and streams only.
"""
from . import field, native, scalar  # noqa: F401
from . import artifact, batched, fused, gen, msm, ntt, pipeline, poly, program, serving, tuner  # noqa: F401
from .scalar import ScalarArray  # noqa: F401

"""B200-native (sm_100a) implementation of TOP3D_XL's matrix-free voxel FEA optimisation loop.

``TOP3D_XL`` mirrors the reference entry point; ``Context`` exposes the C ABI of
libtopx.so (include/topx.h) one call at a time.
"""
from .top3d_xl import TOP3D_XL, Context, TopxError  # noqa: F401

__all__ = ["TOP3D_XL", "Context", "TopxError"]

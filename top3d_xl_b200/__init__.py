"""B200-native (sm_100a) implementation of TOP3D_XL's matrix-free voxel FEA optimisation loop.

``TOP3D_XL`` mirrors the reference entry point; ``Context`` exposes the C ABI of
libtopx.so (include/topx.h) one call at a time; ``Server`` runs many design jobs
at once on one GPU (continuous batching).
"""
from .top3d_xl import TOP3D_XL, Context, Server, TopxError  # noqa: F401

__all__ = ["TOP3D_XL", "Context", "Server", "TopxError"]

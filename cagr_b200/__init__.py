"""B200-native treecode for CAGR (convection-augmented Gauss reconstruction).

The hot path -- octree build, node moments and the treecode evaluation of the
convection-augmented Gauss operator A.mu and its transpose form A^T.w -- runs
as hand-written sm_100a CUDA behind the C ABI in include/cagr.h
(``cagr_b200/lib/libcagr_b200.so``).  ``WindingNumberTreecode`` is the
drop-in for the reference's Python operator object.
"""
from .wn_treecode import WindingNumberTreecode  # noqa: F401

__all__ = ["WindingNumberTreecode"]

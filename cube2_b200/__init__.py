"""cube2_b200 -- B200-native fine-scale kick (PM3 + PP) of the CUBE2 N-body code.

The compute path is the C-ABI shared library ``libcube2_b200.so`` built from
``csrc/`` for sm_100a; this package holds the host-side mirror of the
reference interface (:mod:`cube2_b200.kick`), the particle layout utilities
(:mod:`cube2_b200.layout`) and seeded synthetic inputs (:mod:`cube2_b200.ic`).
"""
from .layout import RATIO_SF, Image, Layout, apm3_table, build_image, classify_subtiles, ixyz3_table  # noqa: F401

__all__ = ["Layout", "Image", "build_image", "classify_subtiles", "ixyz3_table", "apm3_table", "RATIO_SF"]

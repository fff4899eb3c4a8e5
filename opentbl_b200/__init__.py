"""OpenTBL-B200: the RK3 substep of OpenTBL's boundary-layer DNS on one B200.

The compute path is the in-tree CUDA library ``libotbl.so`` (hand-written
sm_100a kernels behind a C ABI, include/otbl.h); this package is the host-side
mirror of the reference's subroutine interface plus box setup.
"""
from .config import BoxConfig, C1, C2, SMALL, TINY, replace  # noqa: F401
from .box import Box, make_box  # noqa: F401
from . import native, synth  # noqa: F401

__all__ = ["BoxConfig", "C1", "C2", "SMALL", "TINY", "replace", "Box", "make_box",
           "native", "synth"]

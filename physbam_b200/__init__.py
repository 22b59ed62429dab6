"""B200-native explicit MPM substep (PhysBAM Hybrid_Methods MPM_DRIVER drop-in).

The compute lives in ``libphysbam_mpm.so`` (hand-written sm_100a CUDA behind
the C ABI in ``include/mpm_capi.h``); this package only loads it and mirrors
the reference driver's API.  See ``driver.MPM_DRIVER``.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "driver"]

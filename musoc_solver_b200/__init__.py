"""B200-native (sm_100a) SEVP barotropic elliptic solver.

Drop-in for the TIMCOM (huyong1109/MUSOC_SOLVER) SEVP solver calls through
the C ABI in ``include/sevp_b200.h``; ``libsevp_b200.so`` holds every kernel.
"""
from . import problems  # noqa: F401

__all__ = ["problems", "native", "solver", "build"]

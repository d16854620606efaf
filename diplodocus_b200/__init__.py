"""B200-native BVH build-and-trace engine (PLOC build, closest-hit trace) behind the acceleration-structure
interface of MasterVotr/Diplodocus. The compute path is libdipl_bvh.so (sm_100a CUDA, C ABI in
include/dipl_bvh.h); this package holds its ctypes binding, the host-side mirror of the reference
interface (accel.py) and the seeded workload generators (scenes.py).
"""
from ._lib import DiplError, load  # noqa: F401

__all__ = ["DiplError", "load"]

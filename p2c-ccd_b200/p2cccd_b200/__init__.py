"""B200-native (sm_100a) certification hot path of P2C-CCD.

Layers:
  * ``libp2c_b200.so`` (csrc/, C ABI in include/p2c_b200.h): the CUDA kernels.
  * ``p2cccd_b200``: host runtime over the C ABI - device-buffer and host-buffer
    batch certification, scene candidate generation, group any-hit with
    fallback replay, batching and serving.
  * ``p2cccd_cpp`` (sibling module): the reference's pybind surface for this
    path, so reference callers switch by import.
"""
from .records import (EDGE_EDGE_DTYPE, FAMILY_EDGE_EDGE, FAMILY_POINT_TRIANGLE, INTERVAL_RESULT_DTYPE,
                      POINT_TRIANGLE_DTYPE, STATUS_COLLISION, STATUS_SEPARATION, STATUS_UNDECIDED)

__all__ = [
    "EDGE_EDGE_DTYPE", "FAMILY_EDGE_EDGE", "FAMILY_POINT_TRIANGLE", "INTERVAL_RESULT_DTYPE",
    "POINT_TRIANGLE_DTYPE", "STATUS_COLLISION", "STATUS_SEPARATION", "STATUS_UNDECIDED",
]

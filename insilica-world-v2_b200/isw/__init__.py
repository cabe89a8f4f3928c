"""isw: a B200-native (sm_100a) dynamical core for the stacked-layer TRiSK shallow-water step and FCT tracer transport,
with the reference's Layers / Transport / DeviceGrid / dsum interface. Device work runs in the in-tree CUDA library
libisw.so through its C ABI (include/isw.h); importing the device modules fails if that library is missing."""
from . import cases, grid  # noqa: F401  (host-only modules)

__all__ = ['cases', 'grid']

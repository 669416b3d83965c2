"""gm1_b200: B200-native (sm_100a) CM1 large-step dynamical-core hot path.

The CUDA kernels live in libgm1b.so (gm1_b200/lib), reached through the C ABI
declared in include/gm1b.h; this package holds the host-side mirror of the
reference operator API.
"""

__version__ = "0.1.0"

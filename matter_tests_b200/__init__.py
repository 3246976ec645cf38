"""B200-native explicit MPM time step of Matter (twmeehan/matter-tests).

The product is libmatter_gpu.so (hand-written sm_100a CUDA behind the C ABI
of include/matter_gpu.h) and the C++ drop-in Simulation in host/.  This Python
package holds the ctypes binding (gpu.py), the ABI struct mirror (abi.py),
the seeded workloads (scenes.py) and the build script (build.py).
"""
from . import abi  # noqa: F401

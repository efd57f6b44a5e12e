"""charming-b200: a single-GPU, B200-native (sm_100a) message-driven runtime
with the chare / entry-method / message API of CharminG.

Python is the host-side front end over the C ABI of libcharming_b200.so;
the runtime itself (persistent scheduler, inbox rings, Jacobi chares,
serving) is CUDA C++.
"""
from ._lib import CharmingError, F32, F64, LIB_PATH, load  # noqa: F401
from .runtime import Runtime, runtime  # noqa: F401

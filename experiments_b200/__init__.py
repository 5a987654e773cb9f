"""B200-native rigid-body step (grid broadphase -> SAT narrowphase -> Jacobi
solver -> integrate) behind a C ABI; see include/b3gpu.h."""
from . import b3, scenes  # noqa: F401
from .b3 import (B3Error, BoundSearch, Context, Fill, PhysicsWorld, PrefixScan,  # noqa: F401
                 RadixSort32, default_config)

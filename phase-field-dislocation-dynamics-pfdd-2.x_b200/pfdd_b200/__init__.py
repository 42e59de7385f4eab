"""pfdd_b200: B200-native PFDD Ginzburg-Landau stepper.

capi     ctypes binding of libpfdd_b200.so (the C ABI in include/pfdd_b200.h)
configs  seeded synthetic workloads and the reference decks describing them
"""
from . import configs  # noqa: F401

__all__ = ["configs", "capi"]

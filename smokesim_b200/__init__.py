"""smokesim_b200 - SmokeSim's per-frame smoke step on B200 (sm_100a).

The product is libsmokesim.so (C ABI in include/smokesim.h); this package is
its thin Python host binding (`Sim`), the ctypes mirror of the ABI types
(`abi`), the seeded benchmark scenes (`scene`) and the in-tree build
(`build`).
"""
from . import abi  # noqa: F401
from .sim import Sim, SmokeSimError  # noqa: F401

__all__ = ["abi", "Sim", "SmokeSimError"]

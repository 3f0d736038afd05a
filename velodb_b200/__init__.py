"""velodb_b200 -- B200-native (sm_100a) oblivious operator hot path of VelODB.

The compute lives in ``libvelo_obl.so`` (hand-written CUDA behind the C ABI of
``include/velo_obl.h``); this package loads it and offers thin Python calls
(``capi``) and the seeded synthetic workloads (``workloads``).
"""
from ._lib import LIB_PATH, VeloError, check, lib  # noqa: F401

__all__ = ["LIB_PATH", "VeloError", "check", "lib"]

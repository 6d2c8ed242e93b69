"""GP5-B200: pseudo-spectral Gross-Pitaevskii time stepping on one NVIDIA B200 (sm_100a).

The compute path is libgp5cu.so (hand-written CUDA behind the C ABI of include/gp5cu.h).
``gp5_b200._abi`` binds it with ctypes; ``gp5_b200.gp`` mirrors the reference's Python
``gp`` package (python/gp/gp.py) over the pybind11 ``gpCpp`` module.  There is no CPU
fallback: without the built library every entry point raises.
"""
from . import _abi  # noqa: F401

__all__ = ["_abi"]

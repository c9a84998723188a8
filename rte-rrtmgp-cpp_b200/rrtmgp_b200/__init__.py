"""rrtmgp_b200: B200-native RTE+RRTMGP column-radiation hot path (C ABI + Python binding).

The compute path is the CUDA library rrtmgp_b200/_lib/librrtmgp_b200.so (built by
rte-rrtmgp-cpp_b200/build.py); importing `rrtmgp_b200.api` fails loudly if it is missing.
"""
from . import synthetic  # noqa: F401

__all__ = ["synthetic"]

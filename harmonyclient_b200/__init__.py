"""B200-native engine for Harmony's IVF query hot path.

The package holds the CUDA engine (``csrc/`` -> ``libhy.so``, C-ABI in
``include/hy.h``), its Python mirror of the reference ``harmony::Index``
(``index.py``) and the seeded synthetic workloads (``datasets.py``).
"""
from .index import (EDGEDEVIVE_DISABLED, EDGEDEVIVE_ENABLED, METRIC_IP, METRIC_L2, OPT_ALL, OPT_NONE,
                    OPT_SUBNN_IP, OPT_SUBNN_L2, OPT_TRIANGLE, HyError, Index, file_inspect)

__all__ = ["Index", "HyError", "file_inspect", "METRIC_IP", "METRIC_L2", "OPT_NONE", "OPT_TRIANGLE", "OPT_SUBNN_L2",
           "OPT_SUBNN_IP", "OPT_ALL", "EDGEDEVIVE_ENABLED", "EDGEDEVIVE_DISABLED"]

"""tdscha_b200: B200 (sm_100a) engine for the TD-SCHA Lanczos linear response.

The compute path lives in the CUDA library ``_lib/libtdscha_b200.so`` (C ABI in
include/tdscha_b200.h); ``DynamicalLanczos.Lanczos`` is the reference-compatible host API
(``MODE_B200``), ``rocksalt`` the seeded synthetic ensemble generator.
"""
from . import build  # noqa: F401

__version__ = "0.1.0"

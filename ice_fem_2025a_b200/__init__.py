"""B200 element assembly for IceFEM's phase-field / viscoplastic / thermal models.

The product is the native library built from ``csrc/`` (C-ABI in ``include/icefem_b200.h``);
this package holds its Python-side helpers: ctypes marshalling (``abi``), reference-style
configuration (``config``) and the synthetic mesh generator (``meshgen``).
"""
from . import abi, meshgen, config  # noqa: F401

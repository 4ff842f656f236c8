"""B200-native (sm_100a) implementation of DUCC's type-1 / type-2 NUFFT.

``ducc_b200.nufft`` is a drop-in for ``ducc0.nufft``; the compute path is the
CUDA library built by ``python -m ducc_b200.build`` behind the C-ABI of
``include/ducc_b200.h``.
"""
from . import nufft  # noqa: F401

__version__ = "0.1.0"

"""Global flags (btorch/config.py:17-20): BTORCH_SPARSE_BACKEND selects the
default sparse backend name; ``sparse`` is the config registry."""

import os

from ._sparse_config import B200SparseConfig, SparseConfigRegistry, TritonSparseConfig

SPARSE_BACKEND = os.environ.get("BTORCH_SPARSE_BACKEND")
SPARSE_BACKEND = SPARSE_BACKEND.lower() if SPARSE_BACKEND else None
sparse = SparseConfigRegistry(SPARSE_BACKEND)

__all__ = ["SPARSE_BACKEND", "B200SparseConfig", "TritonSparseConfig", "sparse"]

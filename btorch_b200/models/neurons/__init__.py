from .alif import ALIF
from .lif import LIF

__all__ = ["LIF", "ALIF"]

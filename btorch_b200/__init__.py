"""B200-native recurrent spiking step with btorch's module API.

    import btorch_b200 as btorch
    from btorch_b200.models import LIF, ExponentialPSC, SparseConn, RecurrentNN

Compute runs in hand-written sm_100a kernels behind the C ABI declared in
include/btorch_b200.h (library: btorch_b200/_lib/libbtorch_b200.so).
"""

__version__ = "0.1.0"

from . import config, connectome, models  # noqa: E402

__all__ = ["config", "connectome", "models", "__version__"]

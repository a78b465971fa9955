"""Delay expansion of a connection matrix (API of
btorch/connectome/connection.py:973-1027): row pre * n_delay_bins + bin,
bin = clip(delay, 0, n_delay_bins - 1).  The fused engine decodes the bin of
each stored edge from this row index."""

from __future__ import annotations

import numpy as np
import scipy.sparse


def expand_conn_for_delays(conn, delays: np.ndarray, n_delay_bins: int = 5):
    delays = np.asarray(delays)
    if np.any(delays < 0):
        raise ValueError("delays must be non-negative")
    c = conn.tocoo()
    n_pre, n_post = c.shape
    bins = np.clip(delays, 0, n_delay_bins - 1).astype(int)
    return scipy.sparse.coo_array((c.data, (c.row * n_delay_bins + bins, c.col)),
                                  shape=(n_pre * n_delay_bins, n_post))


__all__ = ["expand_conn_for_delays"]

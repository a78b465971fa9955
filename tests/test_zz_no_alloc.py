"""The allocation-free sparse product, called through the C ABI.

bt_spmv_gather_noalloc serves callers that cannot allocate device memory when
they need the product (a stream under capture with a fixed memory plan, loops
that must not take cudaMalloc's device-wide synchronisation, hosts without a
device allocator).  Its scratch is a built-in device array, so this file
checks that two calls in a row -- the second one smaller, over whatever the
first left in that array -- match the ordinary entry point (which takes
caller scratch) bit for bit, and that oversize requests are refused.

The file is named to be collected last; it passes alone and after the others.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200 import _lib as L
from btorch_b200.models._ops import build_layout

pytestmark = pytest.mark.gpu


def _problem(rng, batch, n_in, n_out, density=0.1, x_density=0.3):
    w = (rng.random((n_in, n_out)) < density) * rng.standard_normal((n_in, n_out))
    c = sp.coo_array(w.astype(np.float32)).T
    c.sum_duplicates()
    idx = torch.tensor(np.stack([c.row, c.col]), dtype=torch.long)
    lay = build_layout(idx, n_in, n_out, 1).to("cuda")
    wts = torch.tensor(c.data, dtype=torch.float32, device="cuda")
    x = (rng.random((batch, n_in)) < x_density) * rng.standard_normal((batch, n_in))
    return lay, wts, torch.tensor(x.astype(np.float32), device="cuda")


def _with_scratch(lay, wts, x):
    B, n_in = x.shape
    out = torch.empty((B, lay.n_out), device="cuda")
    bits = torch.empty(B * ((n_in + 31) // 32), dtype=torch.int32, device="cuda")
    st = L.lib().bt_spmv_gather(B, n_in, lay.n_out, lay.csc_ptr.data_ptr(), lay.csc_src.data_ptr(),
                                wts.data_ptr(), x.data_ptr(), out.data_ptr(), bits.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    L.check(st, "bt_spmv_gather")
    return out


def _no_alloc(lay, wts, x):
    B, n_in = x.shape
    out = torch.empty((B, lay.n_out), device="cuda")
    st = L.lib().bt_spmv_gather_noalloc(B, n_in, lay.n_out, lay.csc_ptr.data_ptr(), lay.csc_src.data_ptr(),
                                        wts.data_ptr(), x.data_ptr(), out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    L.check(st, "bt_spmv_gather_noalloc")
    return out


def test_no_alloc_gather_matches_entry_point_with_scratch_twice():
    rng = np.random.default_rng(7)
    first = _problem(rng, batch=16, n_in=4000, n_out=900)
    second = _problem(rng, batch=3, n_in=500, n_out=1300, x_density=0.05)
    for lay, wts, x in (first, second):
        got = _no_alloc(lay, wts, x)
        want = _with_scratch(lay, wts, x)
        torch.cuda.synchronize()
        torch.testing.assert_close(got, want, rtol=0, atol=0)


def test_no_alloc_gather_rejects_oversize_requests():
    words = (1 << 25) - 1  # n_in just below the packing limit
    batch = (1 << 18) // ((words + 31) // 32) + 1
    st = L.lib().bt_spmv_gather_noalloc(batch, words, 8, None, None, None, None, None, None)
    assert st == L.BT_ERR_INVALID
    assert b"scratch" in L.lib().bt_last_error()
    # a batch whose product with the word count wraps 64 bits is refused too
    wrap = 1 << 44  # x 2^20 words = 2^64
    st = L.lib().bt_spmv_gather_noalloc(wrap, words, 8, None, None, None, None, None, None)
    assert st == L.BT_ERR_INVALID
    assert b"scratch" in L.lib().bt_last_error()

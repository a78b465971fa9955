"""The reciprocal division of the kernels is enabled per divisor only after an
exhaustive device check against IEEE division (bt_fast_div_check over all 2^32
fp32 inputs)."""

import numpy as np
import pytest
import torch

from btorch_b200 import _lib as L
from btorch_b200.models import _ops

pytestmark = pytest.mark.gpu


def mismatches(c, r):
    m = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.check(L.lib().bt_fast_div_check(float(c), float(r), m.data_ptr(), L.stream_of(torch.device("cuda"))))
    return int(m.item())


@pytest.mark.parametrize("c", [5.0, 20.0, 200.0, 3.0, 7.0, 10.0, 0.1, 1.5])
def test_common_time_constants(c):
    c32 = np.float32(c)
    n_bad = mismatches(c32, np.float32(1.0) / c32)
    ok, r = _ops.fast_division(c, torch.device("cuda"))
    assert ok == (n_bad == 0)
    print(f"\ndivisor {c}: fast path {'on' if ok else 'off'} (exhaustive check over 2^32 inputs)")


def test_wrong_reciprocal_is_caught():
    """The correction step absorbs a reciprocal a few ulp off, not a wrong one."""
    c32 = np.float32(20.0)
    assert mismatches(c32, np.float32(1.0) / c32 * np.float32(1.001)) > 0


@pytest.mark.parametrize("c", [5.0, 20.0, 200.0])
def test_benchmark_time_constants_take_the_fast_path(c):
    """The synaptic (5), membrane (20) and adaptation (200) time constants of
    the benchmark networks divide exactly through the reciprocal path for
    every fp32 input, zeros and tiny quotients included."""
    c32 = np.float32(c)
    assert mismatches(c32, np.float32(1.0) / c32) == 0

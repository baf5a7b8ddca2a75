"""The give-up path of the bounded device-side waits, on the GPU and without a
fault: a CTA waits with a short limit on an mbarrier that nothing arrives on
(lbm_selftest_wait_timeout), the wait returns after the limit, the kernel sets
the device error word and exits, and lbm_device_error_flags reports the bit and
clears it.  The same wait with an arrival succeeds and leaves the word clear;
the context stays usable throughout."""
import ctypes as C

import pytest
import torch

import lbm_b200 as L
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu


def _wait(limit, arrive, cycles):
    return L.lib().lbm_selftest_wait_timeout(int(limit), int(arrive), L._ptr(cycles), L._stream(None))


def test_bounded_wait_gives_up_and_reports():
    SV.device_error_flags(clear=True)
    cycles = torch.zeros(1, dtype=torch.int64, device="cuda")
    limit = 100_000  # about 50 us at the B200's clock
    assert _wait(limit, 0, cycles) == 0
    flags = SV.device_error_flags(clear=True)
    assert flags & 1
    took = int(cycles.item())
    assert limit < took < 100 * limit, took
    assert SV.device_error_flags(clear=False) == 0  # cleared by the read above
    # the context is still usable: a plain torch kernel and a second timeout
    x = torch.arange(1000, device="cuda", dtype=torch.float32)
    assert float(x.sum().item()) == 499500.0
    assert _wait(2 * limit, 0, cycles) == 0
    assert SV.device_error_flags(clear=True) & 1
    assert int(cycles.item()) > 2 * limit


def test_bounded_wait_that_completes_leaves_the_word_clear():
    SV.device_error_flags(clear=True)
    cycles = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert _wait(100_000, 1, cycles) == 0
    assert SV.device_error_flags(clear=True) == 0
    assert int(cycles.item()) < 100_000


def test_selftest_refuses_bad_limits():
    lib = L.lib()
    assert lib.lbm_selftest_wait_timeout(0, 0, None, None) == 1001
    assert lib.lbm_selftest_wait_timeout((1 << 31) + 1, 0, None, None) == 1001
    assert lib.lbm_selftest_wait_timeout(1000, 2, None, None) == 1001

"""Failure detection without a GPU fault: the device waits of this library are bounded, and a wait
that runs out sets the context's status word, returns, and is reported by the call that made it.
The wait here polls a tile flag that nothing ever publishes."""
import os

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu
AXC_EINTERNAL = 10
DEV_SPIN_LIMIT = 3


@pytest.mark.parametrize("spin_limit", [1, 1000, 100000])
def test_bounded_wait_gives_up_and_the_context_recovers(ctx, spin_limit):
    rc = ax.lib().axc_selftest_bounded_wait(ctx._h, spin_limit)
    assert rc == AXC_EINTERNAL
    assert f"status word = {DEV_SPIN_LIMIT}" in ax.lib().axc_last_error(ctx._h).decode()
    # the status word was cleared and the context still partitions correctly
    g = ax.read(os.path.join(GOLDEN, "snn_4x64.snn"))
    p = ax.params_incc(16, 64, 1 << 20, cnc=4, rfr=8)
    part, st = ctx.partition(g, p)
    ref, K, _, _ = O.partition(g.n, g.off, g.pins, g.nsrc, g.w, 0, omega=16, delta=64, max_parts=1 << 20,
                               cnc=4, rfr=8, ipm=1)
    np.testing.assert_array_equal(part, ref)
    assert st.valid == 1


def test_bounded_wait_rejects_a_zero_limit(ctx):
    assert ax.lib().axc_selftest_bounded_wait(ctx._h, 0) == 1  # AXC_EINVAL

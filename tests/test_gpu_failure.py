"""Failure handling on the GPU without a fault: every wait in the
tensor-core kernel is bounded.  Here one warp waits, with that same bounded
wait, on an mbarrier nothing arrives at; the wait must give up after its
limit and report it, and the context must stay usable for a normal step."""
import ctypes

import numpy as np
import pytest

from nrg_b200 import fields
from tests.gpu_util import run_device

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_context_stays_usable(decks, W):
    from nrg_b200.chemistry import ChemicalKineticsSolver, lib
    flag, ms = ctypes.c_int(-1), ctypes.c_double(-1.0)
    assert lib().nrg_selftest_bounded_wait(2_000_000, ctypes.byref(flag), ctypes.byref(ms)) == 0
    assert flag.value == 1
    assert 2.0 <= ms.value < 200.0, ms.value
    assert lib().nrg_selftest_bounded_wait(0, ctypes.byref(flag), None) != 0  # limit must be positive
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        f = fields.slice_field(fields.random_field(W), 256)
        g, st = run_device(s, f, "fast")
    finally:
        s.close()
    assert st["cells_bad"] == 0 and np.all(g["status"] == 1)

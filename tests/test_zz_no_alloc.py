"""The no-allocation step, for callers that cannot allocate device memory
while they step (their device memory is owned by another allocator, or they
step from a context where cudaMalloc is not allowed).

nrg_chem_step_device_noalloc keeps its scratch in a fixed array inside the
library.  It must give the same results as nrg_chem_step_device, on two calls
in a row (the second call finds the first call's scratch contents and must
not depend on them).  This file is collected last so that a run stopping at
its first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from nrg_b200 import fields

pytestmark = pytest.mark.gpu

TOL_Y = 1e-9
TOL_T = 1e-6


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    yield s
    s.close()


def _buffers(f, bc):
    import torch
    dev = torch.device("cuda:0")
    T, rho, Y = (torch.tensor(a, device=dev) for a in (f.T, f.rho, f.Y))
    out = dict(Y_prod=torch.zeros_like(Y), Y_prod2=torch.full_like(Y, 3.25), E_f_prod=torch.zeros_like(T),
               T_after=torch.zeros_like(T), status=torch.zeros(f.n, dtype=torch.uint8, device=dev))
    return T, rho, Y, torch.tensor(bc, dtype=torch.int8, device=dev), out


def _run(step, f, bc):
    import torch
    T, rho, Y, bct, o = _buffers(f, bc)
    st = step(f.dt, T, rho, Y, o["Y_prod"], o["Y_prod2"], o["E_f_prod"], bc=bct, T_after=o["T_after"],
              status=o["status"])
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in o.items()}, st


def test_noalloc_matches_step_device_on_two_calls(solver, W):
    f = fields.slice_field(fields.random_field(W), 3000)
    f.T[:40] = 300.0  # below the reference's 305 K threshold
    bc = np.zeros(f.n, np.int8)
    bc[40:80] = 1
    ref, st_ref = _run(solver.step_device, f, bc)
    skipped = np.arange(f.n) < 80
    for call in range(2):
        got, st = _run(solver.step_device_noalloc, f, bc)
        np.testing.assert_array_equal(got["status"], ref["status"])
        assert np.all(got["Y_prod"][:, skipped] == 0.0) and np.all(got["E_f_prod"][skipped] == 0.0)
        assert np.all(got["Y_prod2"][:, skipped] == 3.25)  # untouched, as in the reference
        act = ~skipped
        dy = np.abs(got["Y_prod"] - ref["Y_prod"])[:, act] * f.dt / f.rho[None, act]
        assert dy.max() <= TOL_Y, (call, dy.max())
        dT = np.abs(got["T_after"] - ref["T_after"])[act] / f.T[act]
        assert dT.max() <= TOL_T, (call, dT.max())
        assert st["cells"] == f.n and st["cells_active"] == st_ref["cells_active"] == f.n - 80
        assert st["cells_bad"] == 0


def test_noalloc_rejects_fields_above_its_limit(solver):
    from nrg_b200.chemistry import lib
    n = (1 << 20) + 1
    rc = lib().nrg_chem_step_device_noalloc(solver.handle, 1e-6, n, n, None, None, None, None, None, None, None,
                                            None, None, None, None)
    assert rc == -1
    assert b"1048576" in lib().nrg_chem_last_error(solver.handle)

"""The no-allocation step, for callers that cannot allocate device memory
while they step (their device memory is owned by another allocator, or they
step from a context where cudaMalloc is not allowed).

nrg_chem_step_device_noalloc keeps its scratch in a fixed array inside the
library.  It runs the same integrator kernels on the same cells as
nrg_chem_step_device, so its outputs must equal that entry point's bit for
bit, on two calls in a row (the second call finds the first call's scratch
contents and must not depend on them), for every launch shape; and one call
is checked directly against the CPU oracle.  This file is collected last so
that a run stopping at its first failure has already run every other test.
"""
import numpy as np
import pytest

from nrg_b200 import fields

pytestmark = pytest.mark.gpu

TOL_Y = 1e-9
TOL_T = 1e-6
OUTPUTS = ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status")
SHAPES = [dict(kernel="thread", block=32), dict(kernel="thread_queue", block=64),
          dict(kernel="warp_queue", block=256)]


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


def _field_with_skips(W, n=3000):
    f = fields.slice_field(fields.random_field(W), n)
    f.T[:40] = 300.0  # below the reference's 305 K threshold
    bc = np.zeros(f.n, np.int8)
    bc[40:80] = 1
    return f, bc, np.arange(f.n) < 80


@pytest.mark.parametrize("shape", SHAPES, ids=[s["kernel"] for s in SHAPES])
def test_noalloc_equals_step_device_on_two_calls(solver, W, shape):
    f, bc, skipped = _field_with_skips(W)
    solver.set_launch(**shape)
    try:
        ref, st_ref = _run(solver.step_device, f, bc)
        for call in range(2):
            got, st = _run(solver.step_device_noalloc, f, bc)
            for k in OUTPUTS:
                np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}, {k}")
            assert np.all(got["Y_prod"][:, skipped] == 0.0) and np.all(got["E_f_prod"][skipped] == 0.0)
            assert np.all(got["Y_prod2"][:, skipped] == 3.25)  # untouched, as in the reference
            assert np.all(got["T_after"][skipped] == f.T[skipped])
            for k in ("cells_active", "steps", "rhs_evals", "jacobians", "solves", "cells_bad"):
                assert st[k] == st_ref[k], (call, k, st[k], st_ref[k])
            assert st["cells"] == f.n and st["cells_active"] == f.n - 80
    finally:
        solver.set_launch(kernel="thread", block=32)


def test_noalloc_matches_the_oracle(solver, oracle_mech, W):
    f, bc, skipped = _field_with_skips(W, n=1024)
    got, st = _run(solver.step_device_noalloc, f, bc)
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y, bc=bc)
    T_o = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
    act = ~skipped
    dy = np.abs(got["Y_prod"] - o["Y_prod"])[:, act] * f.dt / f.rho[None, act]
    assert dy.max() <= TOL_Y, dy.max()
    dT = np.abs(got["T_after"] - T_o)[act] / f.T[act]
    assert dT.max() <= TOL_T, dT.max()
    assert np.all(got["status"][act] == 1) and np.all(got["status"][skipped] == 0)


def test_noalloc_at_its_cell_limit_with_sparse_active_cells(solver, W):
    """1,048,576 cells (1,024 compaction blocks, the documented limit), all
    but 300 of them below 305 K: status and counters equal step_device's, and
    the active cells' results equal it bit for bit."""
    n = 1 << 20
    base = fields.random_field(W)
    rng = np.random.default_rng(11)
    act_idx = np.sort(rng.choice(n, size=300, replace=False))
    src = rng.integers(0, base.n, size=n)
    f = fields.Field("sparse", base.T[src].copy(), base.rho[src].copy(), base.p[src].copy(),
                     np.ascontiguousarray(base.Y[:, src]), base.dt, (n,))
    cold = np.ones(n, bool)
    cold[act_idx] = False
    f.T[cold] = 300.0
    bc = np.zeros(n, np.int8)
    ref, st_ref = _run(solver.step_device, f, bc)
    for call in range(2):
        got, st = _run(solver.step_device_noalloc, f, bc)
        np.testing.assert_array_equal(got["status"], ref["status"])
        assert st["cells_active"] == st_ref["cells_active"] == 300
        for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}, {k}")


def test_noalloc_rejects_fields_above_its_limit(solver):
    from nrg_b200.chemistry import lib
    n = (1 << 20) + 1
    rc = lib().nrg_chem_step_device_noalloc(solver.handle, 1e-6, n, n, None, None, None, None, None, None, None,
                                            None, None, None, None)
    assert rc == -1
    assert b"1048576" in lib().nrg_chem_last_error(solver.handle)

"""Gated inference on held-out states of the wide-range distribution: the
training distribution of the networks (T ~ U[800, 2600] K, p ~ U[0.5, 5]
atm, reactants blended to products, radicals log-U[1e-8, 1e-3]) with
dt ~ log-U[1e-7, 1e-5] s, drawn with a seed used neither for training nor
for calibrating the gate (seed 11).

The networks run with the gate bands calibrated on held-out wide-range
states (`load_default(..., gates="wide-range")`, seed 12).  A step of the
library takes one dt, so the sample is split into ten logarithmic dt bins,
each stepped with its bin's geometric-mean dt; every bin is compared with the
CPU oracle.  Reported: the answered fraction per dt decade and the maxima of
|dY_k| and |dT| of the answered cells per species.  Every active cell, the
answered ones and those integrated in FP64, must stay within the surrogate
mode's bounds (1 K, 1e-4); steps above 1e-6 s are never answered."""
import numpy as np
import pytest

from nrg_b200 import fields
from tests.gpu_util import dY, run_device

pytestmark = pytest.mark.gpu

TOL_T_K = 1.0
TOL_Y = 1e-4
N_CELLS = 16384
SEED = 11


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    from nrg_b200.surrogate import load_default
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    s.set_launch(kernel="thread", block=64)
    load_default(s, gates="wide-range")
    yield s
    s.close()


def test_held_out_wide_range_states_against_oracle(solver, oracle_mech, W, capsys):
    states = fields.training_states(W, N_CELLS, seed=SEED, coupled=0.0)
    edges = np.logspace(-7.0, -5.0, 11)
    answered = {-7: [0, 0], -6: [0, 0]}
    err_y = np.zeros(9)
    err_t = 0.0
    for lo, hi in zip(edges[:-1], edges[1:]):
        idx = np.flatnonzero((states.dt_cells >= lo) & (states.dt_cells < hi))
        dt = float(np.sqrt(lo * hi))
        f = fields.Field("held_out", states.T[idx].copy(), states.rho[idx].copy(), states.p[idx].copy(),
                         np.ascontiguousarray(states.Y[:, idx]), dt, (idx.size,))
        g, _ = run_device(solver, f, "surrogate")
        o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y)
        To = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
        act = f.T >= 305.0
        acc = (g["status"] == 5) & act
        dec = int(np.floor(np.log10(lo) + 1e-9))
        answered[dec][0] += int(acc.sum())
        answered[dec][1] += int(act.sum())
        e = np.abs(dY(g, f) - o["Y_prod"] * f.dt / f.rho[None, :])
        et = np.abs(g["T_after"] - To)
        if dt > 1e-6:
            assert acc.sum() == 0, (dt, int(acc.sum()))
        if acc.any():
            err_y = np.maximum(err_y, e[:, acc].max(axis=1))
            err_t = max(err_t, float(et[acc].max()))
        assert e[:, act].max() <= TOL_Y, (dt, float(e[:, act].max()))
        assert et[act].max() <= TOL_T_K, (dt, float(et[act].max()))
    total = sum(a for a, _ in answered.values())
    with capsys.disabled():
        print(f"\nheld-out wide-range sample, {N_CELLS} cells: answered by the networks "
              + ", ".join(f"dt in [1e{d}, 1e{d + 1}) s: {a} of {n}" for d, (a, n) in sorted(answered.items()))
              + f"; answered cells' max |dT| {err_t:.3f} K, max |dY_k| "
              + " ".join(f"{s}={v:.1e}" for s, v in zip(fields.SPECIES, err_y)))
    assert total > 0
    assert err_y.max() <= TOL_Y and err_t <= TOL_T_K

"""Chemistry sources applied to the state and the state equation on the GPU
(nrg_chem_apply_state_device) against the oracle's restatement of the
reference (cpm_solver.f90:513-560 reactive terms, apply_state_equation in
table_approximated_real_gas.f90:368-470)."""
import numpy as np
import pytest

from nrg_b200 import fields
from tests.gpu_util import run_device
from tests.test_oracle import _energy_per_mass

pytestmark = pytest.mark.gpu

KEYS = ("T", "p", "gamma", "cp", "h_s", "h_full", "v_s", "mix_mol_mass")


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    yield s
    s.close()


def _device_state(solver, f, E, v, T0, bc=None, Y_prod=None, E_f_prod=None):
    import torch
    dev = torch.device("cuda")
    t = lambda a, dt=torch.float64: None if a is None else torch.tensor(a, dtype=dt, device=dev)
    rho, Y, Ef, T = t(f.rho), t(f.Y), t(E), t(T0)
    outs = {k: torch.zeros(f.n, dtype=torch.float64, device=dev) for k in KEYS if k != "T"}
    st = torch.zeros(f.n, dtype=torch.uint8, device=dev)
    solver.apply_state_device(rho, Y, Ef, T, outs["p"], outs["gamma"], v=t(v), time_step=f.dt,
                              Y_prod=t(Y_prod), E_f_prod=t(E_f_prod), bc=t(bc, torch.int8),
                              cp_mass=outs["cp"], h_s=outs["h_s"], h_full=outs["h_full"], v_s=outs["v_s"],
                              mix_mol_mass=outs["mix_mol_mass"], status=st)
    torch.cuda.synchronize()
    r = {k: x.cpu().numpy() for k, x in outs.items()}
    r.update(T=T.cpu().numpy(), Y=Y.cpu().numpy(), E_f=Ef.cpu().numpy(), status=st.cpu().numpy())
    return r


def test_state_equation_matches_oracle(solver, oracle_mech, W):
    f = fields.slice_field(fields.wide_range_field(W, n_side=64), 3000)
    rng = np.random.default_rng(8)
    v = rng.uniform(-500.0, 500.0, (3, f.n))
    E = _energy_per_mass(oracle_mech, f.T, f.Y, W, v)
    T0 = f.T * rng.uniform(0.8, 1.2, f.n)
    g = _device_state(solver, f, E, v, T0)
    o = oracle_mech.apply_state(f.rho, f.Y, E, T0, v=v)
    np.testing.assert_array_equal(g["status"], o["status"])
    for k in KEYS:
        np.testing.assert_allclose(g[k], o[k], rtol=1e-13, atol=0, err_msg=k)
    assert np.max(np.abs(g["T"] - f.T)) < 1e-6


def test_chemistry_step_then_state_update_on_device(solver, oracle_mech, W):
    """Step, then sources + state equation, all on the device, against the
    oracle chain; bc cells untouched."""
    f = fields.slice_field(fields.random_field(W), 2048)
    bc = np.zeros(f.n, np.int8)
    bc[100:140] = 1
    g_step, _ = run_device(solver, f, "fast", bc=bc)
    o_step = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y, bc=bc)
    E = _energy_per_mass(oracle_mech, f.T, f.Y, W, np.zeros((0, f.n)))
    g = _device_state(solver, f, E, None, f.T, bc=bc, Y_prod=g_step["Y_prod"], E_f_prod=g_step["E_f_prod"])
    o = oracle_mech.apply_state(f.rho, f.Y, E, f.T, dt=f.dt, Y_prod=o_step["Y_prod"], E_f_prod=o_step["E_f_prod"],
                                bc=bc)
    act = bc == 0
    assert np.all(g["status"][act] == 1) and np.all(g["status"][~act] == 0)
    np.testing.assert_array_equal(g["Y"][:, ~act], f.Y[:, ~act])
    assert np.max(np.abs(g["Y"] - o["Y"])) <= 1e-9
    assert np.max(np.abs(g["T"] - o["T"])[act] / f.T[act]) <= 1e-6
    assert np.max(np.abs(g["p"] - o["p"])[act] / o["p"][act]) <= 1e-6
    # the state equation's T equals the chemistry step's own closure
    assert np.max(np.abs(g["T"][act] - g_step["T_after"][act])) < 1e-6


def test_acetylene_state_equation_matches_oracle():
    """The 17-species C2H2/O2 deck with the FFCM-1 thermo data."""
    from nrg_b200 import eact_units, mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver, mechanism_tables
    from oracle import oracle_py as op
    paths = mechanism_paths("ACETYLENE")
    units = eact_units("ACETYLENE")
    om = op.Mechanism(*paths, 1.0, units)
    W17 = mechanism_tables(*paths, 1.0, units)["molar_mass"]
    f = fields.acetylene_state(om.species()[:om.n_species], W17, 2000, seed=4)
    rng = np.random.default_rng(9)
    v = rng.uniform(-300.0, 300.0, (2, f.n))
    E = _energy_per_mass(om, f.T, f.Y, W17, v)
    T0 = f.T * rng.uniform(0.9, 1.1, f.n)
    s = ChemicalKineticsSolver(None, *paths, E_act_units=units, mode="fast")
    try:
        g = _device_state(s, f, E, v, T0)
    finally:
        s.close()
    o = om.apply_state(f.rho, f.Y, E, T0, v=v)
    np.testing.assert_array_equal(g["status"], o["status"])
    for k in KEYS:
        np.testing.assert_allclose(g[k], o[k], rtol=1e-13, atol=0, err_msg=k)

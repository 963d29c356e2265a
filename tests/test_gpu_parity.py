"""Parity of the CUDA integrator with the CPU oracle, through the C ABI.

Tolerances (from the task statement for the plain FP64 form):
|dY| <= 1e-9 (mass fraction after the step) and |dT|/T <= 1e-6, where T is
the temperature after the reference energy closure."""
import numpy as np
import pytest

from nrg_b200 import fields
from tests.gpu_util import dY, run_device

pytestmark = pytest.mark.gpu

TOL_Y = 1e-9
TOL_T = 1e-6


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="reference")
    yield s
    s.close()


def oracle_run(oracle_mech, f, bc=None):
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y, bc=bc)
    o["T_after"] = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
    return o


def check_parity(g, o, f, active):
    err_y = np.max(np.abs(dY(g, f)[:, active] - dY(o, f)[:, active]))
    err_t = np.max(np.abs(g["T_after"][active] - o["T_after"][active]) / f.T[active])
    assert err_y <= TOL_Y, f"max |dY| = {err_y:.3e}"
    assert err_t <= TOL_T, f"max |dT|/T = {err_t:.3e}"
    return err_y, err_t


@pytest.mark.parametrize("mode", ["reference", "fast"])
def test_random_field_parity(solver, oracle_mech, W, mode):
    f = fields.random_field(W)
    o = oracle_run(oracle_mech, f)
    g, st = run_device(solver, f, mode)
    assert np.all(g["status"] == 1)
    check_parity(g, o, f, np.ones(f.n, bool))
    assert st["cells_active"] == f.n
    if mode == "reference":
        # same algorithm, same decisions: the work counters agree closely
        assert abs(st["steps"] - o["nstep"].sum()) <= 0.01 * o["nstep"].sum()
        assert abs(st["rhs_evals"] - o["nfe"].sum()) <= 0.01 * o["nfe"].sum()


def test_ignition_field_sample_parity(solver, oracle_mech, W):
    f = fields.slice_field(fields.ignition_field(W, n_side=128), 2048, stride=7)
    o = oracle_run(oracle_mech, f)
    for mode in ("reference", "fast"):
        g, _ = run_device(solver, f, mode)
        check_parity(g, o, f, np.ones(f.n, bool))


def test_launch_shapes_and_graph_agree(solver, W):
    f = fields.random_field(W)
    base, _ = run_device(solver, f, "fast", launch=dict(kernel="warp_queue", block=256))
    for launch in (dict(kernel="warp_queue", block=128, grid=0, chunk=1),
                   dict(kernel="warp_queue", block=256, grid=296, chunk=4),
                   dict(kernel="warp_queue", block=128, grid=148, chunk=7)):
        for graph in (True, False):
            g, _ = run_device(solver, f, "fast", launch=launch, graph=graph)
            for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after"):
                np.testing.assert_array_equal(g[k], base[k])
    solver.set_launch(kernel="warp_queue", block=256, grid=0, chunk=1)


@pytest.mark.parametrize("kernel,block", [("thread", 64), ("thread", 32), ("thread_queue", 64),
                                          ("thread_queue", 32)])
def test_thread_per_cell_kernels_parity(solver, oracle_mech, W, kernel, block):
    f = fields.slice_field(fields.random_field(W), 1024)
    o = oracle_run(oracle_mech, f)
    for mode in ("reference", "fast"):
        g, _ = run_device(solver, f, mode, launch=dict(kernel=kernel, block=block, grid=0, chunk=1))
        check_parity(g, o, f, np.ones(f.n, bool))
    solver.set_launch(kernel="warp_queue", block=256, grid=0, chunk=1)


def test_thread_block_sizes_give_identical_results(solver, W):
    """Per-cell arithmetic does not depend on the block shape."""
    f = fields.slice_field(fields.ignition_field(W, n_side=128), 4000, stride=3)
    outs = [run_device(solver, f, "fast", launch=dict(kernel=k, block=b, grid=0, chunk=1))[0]
            for k, b in (("thread", 64), ("thread", 32), ("thread_queue", 32))]
    for g in outs[1:]:
        for key in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
            np.testing.assert_array_equal(g[key], outs[0][key])
    solver.set_launch(kernel="warp_queue", block=256, grid=0, chunk=1)


@pytest.mark.parametrize("mode", ["reference", "fast", "mixed"])
def test_temperature_order_changes_no_result(solver, W, mode):
    """The integrator takes a step's cells grouped by temperature (default) or
    in cell order: same bits, same statuses and same event counts, with
    skipped, boundary-marked and hot cells mixed into a flame sample, for
    every launch shape."""
    f = fields.slice_field(fields.flame_field(W, n_side=256), 5000, stride=13)
    f.T[:40] = 300.0
    f.T[40:48] = 3500.0
    bc = np.zeros(f.n, np.int8)
    bc[60:90] = 1
    init2 = np.full((9, f.n), 3.25)
    keys = ("cells_active", "steps", "rhs_evals", "jacobians", "solves", "cells_bad")
    try:
        for launch in (dict(kernel="thread", block=32, grid=0, chunk=1),
                       dict(kernel="thread_queue", block=64, grid=0, chunk=2),
                       dict(kernel="warp_queue", block=128, grid=0, chunk=1)):
            solver.set_cell_order(False)
            a, sa = run_device(solver, f, mode, bc=bc, launch=launch, y_prod2_init=init2)
            solver.set_cell_order(True)
            b, sb = run_device(solver, f, mode, bc=bc, launch=launch, y_prod2_init=init2)
            for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
                np.testing.assert_array_equal(b[k], a[k], err_msg=f"{k} {launch}")
            assert all(sb[k] == sa[k] for k in keys), (sa, sb)
            assert sb["cells_active"] == int(np.sum((f.T >= 305.0) & (bc == 0))) and sb["cells_bad"] == 0
    finally:
        solver.set_cell_order(True)
        solver.set_launch(kernel="warp_queue", block=256, grid=0, chunk=1)


def test_skip_rule_bc_and_untouched_y_prod2(solver, oracle_mech, W):
    f = fields.slice_field(fields.random_field(W), 1024)
    f.T[:32] = 300.0
    bc = np.zeros(f.n, np.int8)
    bc[32:64] = 1
    init2 = np.full((9, f.n), 3.25)
    g, st = run_device(solver, f, "reference", bc=bc, y_prod2_init=init2)
    o = oracle_run(oracle_mech, f, bc=bc)
    assert np.all(g["status"][:64] == 0) and np.all(g["status"][64:] == 1)
    assert np.all(g["Y_prod"][:, :64] == 0.0) and np.all(g["E_f_prod"][:64] == 0.0)
    assert np.all(g["Y_prod2"][:, :64] == 3.25)
    assert st["cells_active"] == f.n - 64
    act = np.arange(f.n) >= 64
    check_parity(g, o, f, act)


def test_empty_and_nonfinite_inputs(solver, W):
    import torch
    f = fields.slice_field(fields.random_field(W), 256)
    z = torch.zeros((9, 0), dtype=torch.float64, device="cuda")
    e = torch.zeros(0, dtype=torch.float64, device="cuda")
    st = solver.step_device(1e-6, e, e, z, z, z, e)
    assert st["cells"] == 0
    f.Y[4, :16] = np.nan
    g, st = run_device(solver, f, "fast")
    assert np.all(g["status"][:16] == 4) and np.all(g["status"][16:] == 1)
    assert st["cells_bad"] >= 16


def test_host_layout_drop_in(decks, oracle_mech, W):
    """solve_chemical_kinetics on Fortran-layout host arrays with ghost cells."""
    from nrg_b200.chemistry import DataManager, chemical_kinetics_solver_c
    f = fields.random_field(W)
    nx, ny = f.shape
    m = DataManager.block(nx, ny)
    T = m.create_scalar_field("temperature")
    m.create_scalar_field("pressure")
    rho = m.create_scalar_field("density")
    Y = m.create_vector_field("specie_mass_fraction", 9)
    bc = np.zeros(m.shape, np.int8, order="F")
    m.fields["bc_markers"] = bc
    m.interior(T)[...] = f.T.reshape(ny, nx).T[:, :, None]
    m.interior(rho)[...] = f.rho.reshape(ny, nx).T[:, :, None]
    for k in range(9):
        m.interior(Y[k])[...] = f.Y[k].reshape(ny, nx).T[:, :, None]
    T[0, :, :] = 2000.0  # ghost cells hold data that must not be touched or read
    s = chemical_kinetics_solver_c(m, *decks, mode="reference")
    for k in range(9):
        m.fields["specie_production_chemistry2"][k][...] = -1.0
    st = s.solve_chemical_kinetics(f.dt)
    assert st["cells"] == f.n
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y)
    yp = np.stack([m.interior(a)[:, :, 0].T.reshape(-1) for a in m.fields["specie_production_chemistry"]])
    np.testing.assert_allclose(yp * f.dt / f.rho, o["Y_prod"] * f.dt / f.rho, rtol=0, atol=TOL_Y)
    # ghost layer untouched
    assert np.all(m.fields["specie_production_chemistry2"][0][0, :, :] == -1.0)
    s.close()


def test_host_step_runs_on_the_handles_device_and_keeps_the_callers(decks, oracle_mech, W):
    """A handle created on device 0 steps host arrays while another device is
    current: the work runs on device 0 and the caller's current device is
    still current afterwards."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    from nrg_b200.chemistry import DataManager, chemical_kinetics_solver_c
    f = fields.slice_field(fields.random_field(W), 1024)
    nx, ny = 32, 32
    m = DataManager.block(nx, ny)
    T = m.create_scalar_field("temperature")
    m.create_scalar_field("pressure")
    rho = m.create_scalar_field("density")
    Y = m.create_vector_field("specie_mass_fraction", 9)
    m.interior(T)[...] = f.T.reshape(ny, nx).T[:, :, None]
    m.interior(rho)[...] = f.rho.reshape(ny, nx).T[:, :, None]
    for k in range(9):
        m.interior(Y[k])[...] = f.Y[k].reshape(ny, nx).T[:, :, None]
    torch.cuda.set_device(0)
    s = chemical_kinetics_solver_c(m, *decks, mode="fast")
    try:
        torch.cuda.set_device(1)
        s.solve_chemical_kinetics(f.dt)
        assert torch.cuda.current_device() == 1
    finally:
        s.close()
        torch.cuda.set_device(0)
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y)
    yp = np.stack([m.interior(a)[:, :, 0].T.reshape(-1) for a in m.fields["specie_production_chemistry"]])
    np.testing.assert_allclose(yp * f.dt / f.rho, o["Y_prod"] * f.dt / f.rho, rtol=0, atol=TOL_Y)


def test_mixed_precision_wide_range_error_per_species(solver, oracle_mech, W):
    """Config 2 (T ~ U[800, 2600] K, p ~ U[0.5, 5] atm, dt = 1e-5 s): the FP32
    LU with FP64 residual and one refinement sweep against the FP64 oracle,
    reported per species.  The Newton matrix only steers the chord
    iteration, so the converged step keeps the FP64 path's accuracy."""
    f = fields.slice_field(fields.wide_range_field(W, n_side=128), 4096, stride=3)
    o = oracle_run(oracle_mech, f)
    rows = []
    for mode in ("fast", "mixed"):
        g, st = run_device(solver, f, mode)
        assert st["cells_bad"] == 0
        e = np.abs(dY(g, f) - dY(o, f)).max(axis=1)
        et = np.max(np.abs(g["T_after"] - o["T_after"]) / f.T)
        rows.append((mode, e, et))
        assert e.max() <= TOL_Y, (mode, e)
        assert et <= TOL_T, (mode, et)
    names = fields.SPECIES
    for mode, e, et in rows:
        print(f"{mode:6s} max|dY_k - oracle|: " + " ".join(f"{n}={v:.1e}" for n, v in zip(names, e))
              + f"  max|dT|/T={et:.1e}")


@pytest.mark.parametrize("mode", ["fast", "mixed"])
def test_specialised_code_gives_the_table_driven_bits(decks, W, mode):
    """The generated straight-line RHS / iteration matrix and the table walk
    perform the same operations in the same order."""
    from nrg_b200.chemistry import ChemicalKineticsSolver
    f = fields.slice_field(fields.ignition_field(W, n_side=128), 4000, stride=3)
    s = ChemicalKineticsSolver(None, *decks, mode=mode)
    try:
        outs = []
        for spec in (True, False):
            s.set_specialised(spec)
            outs.append(run_device(s, f, mode, launch=dict(kernel="thread", block=32, grid=0, chunk=1))[0])
    finally:
        s.close()
    for key in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(outs[0][key], outs[1][key])


@pytest.mark.parametrize("name", ["ZHANG", "TEREZA", "KONNOV"])
def test_other_mechanisms_specialised_code_gives_the_table_driven_bits(name):
    """Each reference mechanism's generated code against its own table walk
    (analytic-Jacobian mode, thread-per-cell grid kernel)."""
    from nrg_b200 import mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver, mechanism_tables
    paths = mechanism_paths(name)
    s = ChemicalKineticsSolver(None, *paths, mode="fast")
    try:
        base = fields.slice_field(fields.ignition_field(fields_W(), n_side=128), 2000, stride=5)
        f = fields.state_for_species(base, s.species_names, mechanism_tables(*paths)["molar_mass"])
        outs = []
        for spec in (True, False):
            s.set_specialised(spec)
            g, st = run_device(s, f, "fast", launch=dict(kernel="thread", block=32, grid=0, chunk=1))
            assert st["cells_bad"] == 0
            outs.append(g)
    finally:
        s.close()
    for key in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(outs[0][key], outs[1][key])


@pytest.mark.parametrize("name", ["ZHANG", "TEREZA", "KONNOV"])
def test_other_reference_mechanisms_parity(name):
    """The reference's other H2/air mechanisms (9/28, 10/24 and 13/71
    species/reactions, compiled for the thread-per-cell grid kernel) against
    the oracle in both FP64 modes."""
    from nrg_b200 import mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver
    from oracle import oracle_py as op
    paths = mechanism_paths(name)
    om = op.Mechanism(*paths, 1.0, "cal.mol")
    W = om.tables()["molar_mass"]
    names = om.species()[:om.n_species]
    base = fields.slice_field(fields.random_field(fields_W()), 1024)
    f = fields.state_for_species(base, names, W)
    o = oracle_run(om, f)
    s = ChemicalKineticsSolver(None, *paths, mode="reference")
    try:
        s.autotune(f.dt, *[x for x in _dev(f)], *_dev_out(f))
        for mode in ("reference", "fast"):
            g, st = run_device(s, f, mode)
            assert st["cells_bad"] == 0, (mode, st)
            check_parity(g, o, f, np.ones(f.n, bool))
    finally:
        s.close()


def test_acetylene_mechanism_parity():
    """The reference's C2H2/O2 deck (17 species, 25 irreversible reactions,
    FFCM-1 thermo data, E_act in J/mol) on random C2H2/O2/Ar cells against
    the oracle in both FP64 modes, and its generated code against its table
    walk."""
    from nrg_b200 import eact_units, mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver, mechanism_tables
    from oracle import oracle_py as op
    paths = mechanism_paths("ACETYLENE")
    units = eact_units("ACETYLENE")
    om = op.Mechanism(*paths, 1.0, units)
    W = mechanism_tables(*paths, 1.0, units)["molar_mass"]
    f = fields.acetylene_state(om.species()[:om.n_species], W, 1024, seed=3)
    o = oracle_run(om, f)
    s = ChemicalKineticsSolver(None, *paths, E_act_units=units, mode="reference")
    try:
        outs = {}
        for mode in ("reference", "fast"):
            g, st = run_device(s, f, mode, launch=dict(kernel="thread", block=32, grid=0, chunk=1))
            assert st["cells_bad"] == 0, (mode, st)
            check_parity(g, o, f, np.ones(f.n, bool))
            outs[mode] = g
        s.set_specialised(False)
        g, _ = run_device(s, f, "fast", launch=dict(kernel="thread", block=32, grid=0, chunk=1))
        for key in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
            np.testing.assert_array_equal(g[key], outs["fast"][key])
    finally:
        s.close()


def fields_W():
    from nrg_b200 import keromnes_paths
    from nrg_b200.chemistry import mechanism_tables
    return mechanism_tables(*keromnes_paths())["molar_mass"]


def _dev(f):
    import torch
    d = torch.device("cuda")
    return torch.tensor(f.T, device=d), torch.tensor(f.rho, device=d), torch.tensor(f.Y, device=d)


def _dev_out(f):
    import torch
    d = torch.device("cuda")
    Y = torch.zeros((f.Y.shape[0], f.n), dtype=torch.float64, device=d)
    return Y, torch.zeros_like(Y), torch.zeros(f.n, dtype=torch.float64, device=d)


@pytest.mark.parametrize("shape", [(37, 5, 3), (3, 1, 1), (11, 13, 1)])
def test_host_layout_shapes_match_the_device_step(decks, W, shape):
    """The host path (row chunks gathered, copied, stepped and scattered in
    overlap) on 3-D, single-row and few-row blocks with bc cells gives the
    device path's bits, leaves ghost cells alone and keeps Y_prod2 in
    skipped cells."""
    from nrg_b200.chemistry import ChemicalKineticsSolver, DataManager, chemical_kinetics_solver_c
    nx, ny, nz = shape
    n = nx * ny * nz
    f = fields.slice_field(fields.ignition_field(W, n_side=64), n, stride=3)
    bc_flat = (np.arange(n) % 7 == 3).astype(np.int8)
    m = DataManager.block(nx, ny, nz)
    T = m.create_scalar_field("temperature")
    m.create_scalar_field("pressure")
    rho = m.create_scalar_field("density")
    Y = m.create_vector_field("specie_mass_fraction", 9)
    bc = np.full(m.shape, 5, np.int8, order="F")
    m.fields["bc_markers"] = bc
    cube = lambda a: a.reshape(nz, ny, nx).transpose(2, 1, 0)  # cell order: i fastest, then j, then k
    m.interior(T)[...] = cube(f.T)
    m.interior(rho)[...] = cube(f.rho)
    m.interior(bc)[...] = cube(bc_flat)
    for k in range(9):
        m.interior(Y[k])[...] = cube(f.Y[k])
    s = chemical_kinetics_solver_c(m, *decks, mode="fast")
    for k in range(9):
        m.fields["specie_production_chemistry2"][k][...] = -1.0
    s.set_launch(kernel="thread", block=32, grid=0, chunk=1)
    st = s.solve_chemical_kinetics(f.dt)
    s.close()
    assert st["cells"] == n
    d = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        g, _ = run_device(d, f, "fast", bc=bc_flat, launch=dict(kernel="thread", block=32, grid=0, chunk=1),
                          y_prod2_init=np.full((9, n), -1.0))
    finally:
        d.close()
    flat = lambda a: m.interior(a).transpose(2, 1, 0).reshape(-1)
    yp = np.stack([flat(a) for a in m.fields["specie_production_chemistry"]])
    yp2 = np.stack([flat(a) for a in m.fields["specie_production_chemistry2"]])
    np.testing.assert_array_equal(yp, g["Y_prod"])
    np.testing.assert_array_equal(yp2, g["Y_prod2"])
    np.testing.assert_array_equal(flat(m.fields["energy_production_chemistry"]), g["E_f_prod"])
    assert np.all(yp2[:, bc_flat != 0] == -1.0)
    ghost = np.ones(m.shape, bool)
    ghost[tuple(slice(lo - l, hi - l + 1) for lo, hi, l in zip(m.lo, m.hi, m.lb))] = False
    assert np.all(m.fields["specie_production_chemistry2"][0][ghost] == -1.0)


def test_integrator_eps_override_and_restore(solver, oracle_mech, W):
    """nrg_chem_set_eps, in the warp-per-cell and the thread-per-cell
    kernels: a looser EPS takes fewer BDF steps and stays within its own
    bound of the oracle; 0 restores the reference's 1e-9 bits."""
    f = fields.slice_field(fields.random_field(W), 2048)
    for launch in (dict(kernel="warp_queue", block=256, grid=0, chunk=1), dict(kernel="thread", block=32)):
        _check_eps(solver, oracle_mech, f, launch)


def _check_eps(solver, oracle_mech, f, launch):
    from nrg_b200.chemistry import NrgError
    solver.set_launch(**launch)
    base, st0 = run_device(solver, f, "fast")
    try:
        solver.set_eps(1e-5)
        loose, st1 = run_device(solver, f, "fast")
        with pytest.raises(NrgError):
            solver.set_eps(-1.0)
        with pytest.raises(NrgError):
            solver.set_eps(1.5)
    finally:
        solver.set_eps(0.0)
    again, _ = run_device(solver, f, "fast")
    assert st1["steps"] < st0["steps"]
    o = oracle_run(oracle_mech, f)
    act = f.T >= 305.0
    # the random field's states are harsher than the flame's: 1.3e-6 measured
    assert np.abs(dY(loose, f) - dY(o, f))[:, act].max() <= 1e-5
    for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(again[k], base[k])


@pytest.mark.parametrize("mode", ["reference", "fast", "mixed"])
def test_lu_forms_give_identical_results(solver, W, mode):
    """nrg_chem_set_lu_form: the unrolled and the looped LU factorisation of
    the thread-per-cell kernels take the same operations in the same order."""
    f = fields.slice_field(fields.ignition_field(W, n_side=128), 4000, stride=3)
    try:
        outs = [run_device(solver, f, mode, launch=dict(kernel="thread", block=32, grid=0, chunk=1, lu_rolled=r))
                for r in (False, True)]
    finally:
        solver.set_launch(kernel="warp_queue", block=256, grid=0, chunk=1, lu_rolled=False)
    (a, sa), (b, sb) = outs
    for key in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    for key in ("steps", "rhs_evals", "jacobians", "solves"):
        assert sa[key] == sb[key], key
    assert solver.get_launch()["lu_rolled"] is False

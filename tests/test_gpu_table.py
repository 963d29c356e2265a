"""The table_approximated mode on the GPU against the oracle, through the C
ABI (chemical_kinetics_solver.f90:542-685 and the mode's branches of
:228-346).

The table is made the way the reference makes one: one row of the flame
field (a 1-D flame from 300 K to 2400 K) is stepped by the plain FP64
integrator, and its T and Y_prod2 are written with the table writer; the
library and the oracle each read the file back.  The interpolated sources
(Y_prod, Y_prod2, E_f_prod) must equal the oracle's bit for bit -- the
device kernel is compiled without FMA contraction and keeps the
reference's operation order -- and the temperature after the step must
agree to 1e-6 relative."""
import numpy as np
import pytest

from nrg_b200 import fields
from nrg_b200.chemistry import DataManager
from tests.gpu_util import run_device

pytestmark = pytest.mark.gpu

TOL_T = 1e-6


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    yield s
    s.close()


@pytest.fixture(scope="module")
def flame(W):
    return fields.flame_field(W)


@pytest.fixture(scope="module")
def table_file(solver, flame, tmp_path_factory):
    """The flame's first row stepped by the plain integrator, tabulated."""
    from nrg_b200 import chemistry
    n = flame.shape[0]
    row = fields.slice_field(flame, n)
    out, _ = run_device(solver, row, "fast")
    m = DataManager((0, 1, 1), (n + 1, 1, 1), (1, 1, 1), (n, 1, 1))
    T = m.create_scalar_field("temperature")
    y2 = m.create_vector_field("specie_production_chemistry2", 9)
    m.interior(T)[:, 0, 0] = row.T
    for k in range(9):
        m.interior(y2[k])[:, 0, 0] = out["Y_prod2"][k]
    path = tmp_path_factory.mktemp("table") / "H2-Air_table(T).dat"
    chemistry.write_table(path, solver.species_names, m)
    return path


def _oracle_table(oracle_mech, T_t, Y_t, f, bc=None, init=None):
    o = oracle_mech.table_step(T_t, Y_t, f.dt, f.T, f.Y, bc=bc, Y_prod2_init=init)
    o["T_after"] = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
    return o


def _compare(g, o, f, skipped):
    act = ~skipped
    for k in ("Y_prod", "Y_prod2", "E_f_prod"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    dT = np.abs(g["T_after"] - o["T_after"])[act] / f.T[act]
    assert np.nanmax(dT) <= TOL_T if dT.size else True
    np.testing.assert_array_equal(g["T_after"][skipped], f.T[skipped])


def test_flame_table_step_equals_the_oracle(solver, oracle_mech, flame, table_file):
    from oracle import oracle_py as op
    T_t, Y_t = op.table_read(table_file, 9)
    assert 200 < T_t.size < 2048 and T_t[0] > 300.5 and T_t[-1] == 2400.0
    solver.read_chemical_kinetics_table(table_file)
    f = fields.slice_field(flame, 64 * 2048, offset=900 * 2048)
    bc = np.zeros(f.n, np.int8)
    bc[::97] = 1
    init = np.full((9, f.n), -5.0)
    g, st = run_device(solver, f, "table", bc=bc, y_prod2_init=init)
    o = _oracle_table(oracle_mech, T_t, Y_t, f, bc=bc, init=init)
    skipped = (f.T < 305.0) | (bc != 0)
    _compare(g, o, f, skipped)
    # Rounded to seven digits, the last rows of the table all read 2400 K, so
    # a cell at exactly 2400 K falls in the last interval [2400, 2400] and the
    # reference's interpolation divides 0 by 0: its sources are NaN there, in
    # the oracle and on the device alike, and the device flags those cells.
    nan_cells = ~np.isfinite(o["E_f_prod"])
    assert T_t[-2] == T_t[-1] == 2400.0
    assert np.array_equal(nan_cells, ~skipped & (f.T == 2400.0))
    assert np.all(g["status"][skipped] == 0)
    assert np.all(g["status"][~skipped & ~nan_cells] == 1) and np.all(g["status"][nan_cells] == 4)
    assert st["cells_active"] == int((~skipped).sum()) and st["cells_bad"] == int(nan_cells.sum())
    assert np.all(g["Y_prod2"][:, skipped] == -5.0)


@pytest.mark.parametrize("nodes", [
    [400.0, 800.0, 800.0, 1600.0, 2400.0],            # sorted, a repeated node (bisection)
    [400.0, 800.0, 1600.0, 1200.0, 2000.0, 2400.0],   # not sorted (the reference's scan)
    [900.0],                                          # one row, no interval
])
def test_interpolation_edge_cases_equal_the_oracle(solver, oracle_mech, W, nodes):
    rng = np.random.default_rng(5)
    T_t = np.array(nodes)
    Y_t = rng.standard_normal((9, T_t.size)) * 1e-4
    base = fields.random_field(W)
    probes = np.concatenate([T_t, [300.0, 305.0, 350.0, 1000.0, 1300.0, 1400.0, 2399.0, 2600.0, 3000.0]])
    f = fields.slice_field(base, probes.size)
    f.T[:] = probes
    solver.set_table(T_t, Y_t)
    g, st = run_device(solver, f, "table")
    o = _oracle_table(oracle_mech, T_t, Y_t, f)
    skipped = f.T < 305.0
    for k in ("Y_prod", "Y_prod2", "E_f_prod"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=f"{nodes}: {k}")
    fin = np.isfinite(o["E_f_prod"])
    assert np.array_equal(g["status"] == 4, ~fin & ~skipped)


def test_bucket_search_and_sources_on_hard_operands_equal_the_oracle(solver, oracle_mech, W):
    """The kernel finds a cell's interval by bisection inside one bucket of a
    4,096-bucket index over the sorted nodes; the interval and the sources
    must be the reference's bit for bit.  Operands that stress them: a
    cluster of 500 nodes inside one bucket, node gaps of one ulp (~2e-13 K),
    repeated nodes (0 / 0), cell temperatures exactly at nodes, at the host's
    bucket edges and one ulp either side, table values over the whole double
    range (zeros, subnormals, values near the overflow threshold), and an odd
    step length."""
    rng = np.random.default_rng(23)
    nodes = np.concatenate([
        rng.uniform(400.0, 2600.0, 300),
        1200.0 + rng.uniform(0.0, 1e-3, 500),                      # one bucket
        1800.0 + np.arange(40) * 2.2737367544323206e-13,            # 1 ulp of 1800 K apart
        np.repeat(rng.uniform(500.0, 2500.0, 5), 2),                # repeated nodes
        [400.0, 2600.0]])
    T_t = np.sort(nodes)
    M = T_t.size
    mag = 10.0 ** rng.uniform(-320.0, 305.0, (9, M))
    Y_t = np.where(rng.random((9, M)) < 0.5, -1.0, 1.0) * mag
    Y_t[:, ::17] = 0.0
    Y_t[:, 5::41] = 5e-324
    w = (T_t[-1] - T_t[0]) / 4096
    edges = T_t[0] + np.arange(4097) * w
    probes = np.concatenate([
        T_t, np.nextafter(T_t, np.inf), np.nextafter(T_t, -np.inf),
        edges, np.nextafter(edges, np.inf), np.nextafter(edges, -np.inf),
        rng.uniform(305.0, 3000.0, 20000),
        1200.0 + rng.uniform(-1e-4, 1.1e-3, 8000),
        1800.0 + rng.uniform(-1e-12, 1e-11, 2000)])
    base = fields.random_field(W, n_side=256)
    f = fields.slice_field(base, probes.size)
    f.T[:] = probes
    f.dt = 3.7e-7
    solver.set_table(T_t, Y_t)
    g, st = run_device(solver, f, "table")
    o = _oracle_table(oracle_mech, T_t, Y_t, f)
    for k in ("Y_prod", "Y_prod2", "E_f_prod"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    skipped = f.T < 305.0
    fin = np.isfinite(o["E_f_prod"]) & np.all(np.isfinite(o["Y_prod"]) & np.isfinite(o["Y_prod2"]), axis=0)
    assert np.array_equal(g["status"] == 4, ~fin & ~skipped)
    # finite sources and overflows both occur
    ok = np.isfinite(o["Y_prod"]) & (o["Y_prod"] != 0.0)
    assert ok.sum() > 100000 and (~np.isfinite(o["Y_prod"])).sum() > 0


def test_host_layout_table_mode_through_the_reference_constructor(decks, oracle_mech, flame, table_file):
    """chemical_kinetics_solver_c(..., ODE_solver='table_approximated') on
    Fortran-layout host arrays with a ghost layer."""
    from oracle import oracle_py as op
    from nrg_b200.chemistry import chemical_kinetics_solver_c
    f = fields.slice_field(flame, 16 * 2048, offset=1000 * 2048)
    nx, ny = 2048, 16
    m = DataManager.block(nx, ny)
    for name in ("temperature", "pressure", "density"):
        m.create_scalar_field(name)
    Y = m.create_vector_field("specie_mass_fraction", 9)
    m.interior(m.fields["temperature"])[...] = f.T.reshape(ny, nx).T[:, :, None]
    m.interior(m.fields["density"])[...] = f.rho.reshape(ny, nx).T[:, :, None]
    for k in range(9):
        m.interior(Y[k])[...] = f.Y[k].reshape(ny, nx).T[:, :, None]
    s = chemical_kinetics_solver_c(m, *decks, ODE_solver="table_approximated", table_file=table_file)
    try:
        st = s.solve_chemical_kinetics(f.dt)
    finally:
        s.close()
    T_t, Y_t = op.table_read(table_file, 9)
    o = oracle_mech.table_step(T_t, Y_t, f.dt, f.T, f.Y)
    yp = np.stack([m.interior(a)[:, :, 0].T.reshape(-1) for a in m.fields["specie_production_chemistry"]])
    ef = m.interior(m.fields["energy_production_chemistry"])[:, :, 0].T.reshape(-1)
    np.testing.assert_array_equal(yp, o["Y_prod"])
    np.testing.assert_array_equal(ef, o["E_f_prod"])
    assert st["cells"] == f.n


def test_table_mode_without_a_table_is_refused(decks, W):
    from nrg_b200.chemistry import ChemicalKineticsSolver, NrgError
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        with pytest.raises(NrgError, match="no table"):
            run_device(s, fields.slice_field(fields.random_field(W), 64), "table")
    finally:
        s.close()

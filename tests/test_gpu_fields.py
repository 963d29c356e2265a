"""Parity with the CPU oracle on the configured benchmark fields, through the
C ABI.

* the 2048 x 2048 flame field: a seeded sample of 34,816 cells drawn from
  every temperature band (cold pass-through, preheat, front, trailing edge,
  burnt), in plain FP64 (|dY| <= 1e-9, |dT|/T <= 1e-6) and through the
  surrogate with its FP64 fallback (|dT| <= 1 K, |dY_k| <= 1e-4);
* the 512 x 512 ignition field (20 % of the cells within 50 K of the 1e-5 s
  ignition temperature, dt = 1e-5 s): all 262,144 cells, reference and
  analytic-Jacobian modes;
* the 1024 x 1024 wide-range field (T ~ U[800, 2600] K, p ~ U[0.5, 5] atm,
  dt = 1e-5 s): a 65,536-cell sample in mixed precision (FP32 LU, FP64
  residual), error reported per species.

Each test prints its per-species maxima."""
import numpy as np
import pytest

from nrg_b200 import fields
from nrg_b200.surrogate import FALLBACK_EPS
from tests.gpu_util import dY, run_device

pytestmark = pytest.mark.gpu

TOL_Y = 1e-9
TOL_T = 1e-6
SUR_TOL_T_K = 1.0
SUR_TOL_Y = 1e-4
# cells the gate rejects, integrated in FP64 at EPS 1e-5
FALLBACK_TOL_Y = 1e-6
FALLBACK_TOL_T_K = 0.01

# (T_lo, T_hi, cells drawn) per band of the flame field
FLAME_BANDS = [(0.0, 305.0, 2048), (305.0, 800.0, 8192), (800.0, 2380.0, 14336), (2380.0, 2399.9, 4096),
               (2399.9, 1e9, 6144)]


def _oracle(oracle_mech, f):
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y)
    o["T_after"] = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
    return o


def _report(capsys, title, e_species, extra=""):
    with capsys.disabled():
        print(f"\n{title}: max|dY_k - oracle| " + " ".join(f"{n}={v:.1e}" for n, v in zip(fields.SPECIES, e_species))
              + (f"  {extra}" if extra else ""))


def flame_sample(W, seed=21):
    """Cells of the 2048 x 2048 flame field drawn per temperature band."""
    full = fields.flame_field(W)
    rng = np.random.default_rng(seed)
    idx = []
    for lo, hi, k in FLAME_BANDS:
        band = np.flatnonzero((full.T >= lo) & (full.T < hi))
        idx.append(rng.choice(band, size=min(k, band.size), replace=False))
    idx = np.sort(np.concatenate(idx))
    return fields.Field("flame_sample", full.T[idx].copy(), full.rho[idx].copy(), full.p[idx].copy(),
                        np.ascontiguousarray(full.Y[:, idx]), full.dt, (idx.size,))


@pytest.fixture(scope="module")
def flame(W, oracle_mech):
    f = flame_sample(W)
    return f, _oracle(oracle_mech, f)


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    s.set_launch(kernel="thread", block=64)
    yield s
    s.close()


def test_flame_field_sample_plain_fp64_parity(solver, flame, capsys):
    f, o = flame
    g, st = run_device(solver, f, "fast")
    act = f.T >= 305.0
    assert act.sum() >= 32768
    assert np.array_equal(g["status"] != 0, act) and np.all(g["status"][act] == 1)
    e = np.abs(dY(g, f) - dY(o, f))[:, act].max(axis=1)
    et = np.max(np.abs(g["T_after"] - o["T_after"])[act] / f.T[act])
    _report(capsys, f"flame sample, plain FP64, {act.sum()} active cells", e, f"max|dT|/T={et:.1e}")
    assert e.max() <= TOL_Y, e
    assert et <= TOL_T, et
    assert np.all(g["Y_prod"][:, ~act] == 0.0)


def test_flame_field_sample_surrogate_against_oracle(solver, flame, capsys):
    """The committed networks (the main one and the band networks), each
    with its calibrated gate, against the oracle; every network answers
    some of the cells routed to it."""
    from nrg_b200.surrogate import COMMITTED, load_default, routed_to
    f, o = flame
    nets = load_default(solver)
    assert len(nets) == len(COMMITTED)
    g, st = run_device(solver, f, "surrogate")
    route = routed_to(nets, f.T)
    for s in nets:
        assert ((g["status"] == 5) & (route == s.net) & (f.T >= 305.0)).sum() > 0, s.net
    act = f.T >= 305.0
    acc = g["status"] == 5
    assert acc.sum() > 0 and np.array_equal(g["status"] != 0, act)
    dT = np.abs(g["T_after"] - o["T_after"])[act]
    e = np.abs(dY(g, f) - dY(o, f))[:, act].max(axis=1)
    _report(capsys, f"flame sample, surrogate + fallback, {acc.sum()} of {act.sum()} answered by the network",
            e, f"max|dT|={dT.max():.3f} K")
    for lo, hi, _ in FLAME_BANDS[1:]:
        b = act & (f.T >= lo) & (f.T < hi)
        with capsys.disabled():
            print(f"  band {lo:.0f}-{min(hi, 2400):.0f} K: {int((acc & b).sum())} of {int(b.sum())} accepted")
    assert dT.max() <= SUR_TOL_T_K, dT.max()
    assert e.max() <= SUR_TOL_Y, e
    # the rejected cells, integrated at the fallback tolerance (1e-5)
    fb = act & ~acc
    assert fb.sum() > 0
    assert np.abs(dY(g, f) - dY(o, f))[:, fb].max() <= FALLBACK_TOL_Y
    assert np.abs(g["T_after"] - o["T_after"])[fb].max() <= FALLBACK_TOL_T_K


def test_surrogate_fallback_at_the_reference_eps_gives_the_plain_bits(solver, flame):
    """With the fallback at the reference's EPS (1e-9) the rejected cells are
    the plain integrator's cells bit for bit; the accepted ones are the
    network's either way."""
    from nrg_b200.surrogate import load_default
    f, _ = flame
    plain, _ = run_device(solver, f, "fast")
    nets = load_default(solver, fallback_eps=0.0)
    try:
        g, st = run_device(solver, f, "surrogate")
    finally:
        nets[0].set_fallback_eps(FALLBACK_EPS)
    g5, _ = run_device(solver, f, "surrogate")
    fb = (g["status"] != 5) & (g["status"] != 0)
    assert fb.sum() > 0
    for k in ("Y_prod", "Y_prod2"):
        np.testing.assert_array_equal(g[k][:, fb], plain[k][:, fb])
    for k in ("E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(g[k][fb], plain[k][fb])
    acc = g["status"] == 5
    np.testing.assert_array_equal(g5["status"] == 5, acc)
    np.testing.assert_array_equal(g5["Y_prod"][:, acc], g["Y_prod"][:, acc])


def test_surrogate_host_layout_equals_the_device_step(decks, W):
    """solve_chemical_kinetics in surrogate mode on Fortran-layout host arrays
    (only Y_prod2 crosses PCIe; the host rebuilds Y_prod = Y_prod2 W / dt)
    gives the device entry point's bits, skipped cells included."""
    from nrg_b200.chemistry import ChemicalKineticsSolver, DataManager, chemical_kinetics_solver_c
    from nrg_b200.surrogate import load_default
    full = fields.flame_field(W)
    nx, ny = 2048, 6
    f = fields.slice_field(full, nx * ny, offset=1021 * 2048)
    assert (f.T < 305.0).any() and (f.T > 2000.0).any()
    m = DataManager.block(nx, ny)
    for name in ("temperature", "pressure", "density"):
        m.create_scalar_field(name)
    Y = m.create_vector_field("specie_mass_fraction", 9)
    m.interior(m.fields["temperature"])[...] = f.T.reshape(ny, nx).T[:, :, None]
    m.interior(m.fields["density"])[...] = f.rho.reshape(ny, nx).T[:, :, None]
    for k in range(9):
        m.interior(Y[k])[...] = f.Y[k].reshape(ny, nx).T[:, :, None]
    host = chemical_kinetics_solver_c(m, *decks)
    for k in range(9):
        m.fields["specie_production_chemistry2"][k][...] = -1.0
    try:
        load_default(host)
        host.set_mode("surrogate")
        st = host.solve_chemical_kinetics(f.dt)
    finally:
        host.close()
    d = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        load_default(d)
        g, _ = run_device(d, f, "surrogate", y_prod2_init=np.full((9, f.n), -1.0))
    finally:
        d.close()
    flat = lambda a: m.interior(a)[:, :, 0].T.reshape(-1)
    yp = np.stack([flat(a) for a in m.fields["specie_production_chemistry"]])
    yp2 = np.stack([flat(a) for a in m.fields["specie_production_chemistry2"]])
    assert (g["status"] == 5).sum() > 0 and (g["status"] == 0).sum() > 0
    np.testing.assert_array_equal(yp, g["Y_prod"])
    np.testing.assert_array_equal(yp2, g["Y_prod2"])
    np.testing.assert_array_equal(flat(m.fields["energy_production_chemistry"]), g["E_f_prod"])
    assert st["cells"] == f.n


@pytest.mark.parametrize("mode", ["reference", "fast"])
def test_ignition_field_all_cells_parity(solver, oracle_mech, W, mode, capsys):
    f = fields.ignition_field(W)
    assert f.n == 262144
    o = _ignition_oracle(oracle_mech, f)
    g, st = run_device(solver, f, mode)
    assert np.all(g["status"] == 1) and st["cells_bad"] == 0
    e = np.abs(dY(g, f) - dY(o, f)).max(axis=1)
    et = np.max(np.abs(g["T_after"] - o["T_after"]) / f.T)
    steps = o["nstep"]
    _report(capsys, f"ignition field, all {f.n} cells, {mode}", e,
            f"max|dT|/T={et:.1e}  oracle steps/cell {steps.min()}..{steps.max()}")
    assert e.max() <= TOL_Y, e
    assert et <= TOL_T, et


_IGN = {}


def _ignition_oracle(oracle_mech, f):
    if "o" not in _IGN:
        _IGN["o"] = _oracle(oracle_mech, f)
    return _IGN["o"]


def test_wide_range_field_sample_mixed_precision_per_species(solver, oracle_mech, W, capsys):
    f = fields.slice_field(fields.wide_range_field(W), 65536, stride=16, offset=5)
    o = _oracle(oracle_mech, f)
    for mode in ("fast", "mixed"):
        g, st = run_device(solver, f, mode)
        assert st["cells_bad"] == 0
        e = np.abs(dY(g, f) - dY(o, f)).max(axis=1)
        et = np.max(np.abs(g["T_after"] - o["T_after"]) / f.T)
        _report(capsys, f"wide-range sample, {f.n} cells, {mode}", e, f"max|dT|/T={et:.1e}")
        assert e.max() <= TOL_Y, (mode, e)
        assert et <= TOL_T, (mode, et)

"""Transport decks and the oracle's mixture-averaged diffusion coefficients
(thermophysical_properties_class.f90:560-577, 737-814, 1343-1414): the
library's reader against the oracle's, bit for bit, and the oracle against
published kinetic-theory values and the binary limit."""
import os

import numpy as np
import pytest

from nrg_b200 import MECHANISMS, eact_units, mechanism_paths, transport_path
from oracle import oracle_py as op

P_ATM = 101325.0


@pytest.fixture(scope="module")
def om():
    m = op.Mechanism(*mechanism_paths("KEROMNES"), 1.0, "cal.mol")
    m.load_transport(transport_path("KEROMNES"))
    return m


@pytest.mark.parametrize("name", MECHANISMS + ("ACETYLENE",))
def test_transport_tables_product_equals_oracle(name):
    from nrg_b200.chemistry import transport_tables
    t = transport_tables(*mechanism_paths(name), transport_path(name))
    m = op.Mechanism(*mechanism_paths(name), 1.0, eact_units(name))
    m.load_transport(transport_path(name))
    o = m.transport_tables()
    for k in t:
        np.testing.assert_array_equal(t[k], o[k], err_msg=k)
    assert np.all(t["well_depth"] > 0) and np.all(t["collision_diameter"] > 0)


def test_hand_read_transport_values():
    """KEROMNES_TRANSDATA.txt: H2 38.000 K, 2.920 A; H2O 572.400 K, 2.605 A."""
    from nrg_b200.chemistry import transport_tables
    t = transport_tables(*mechanism_paths("KEROMNES"), transport_path("KEROMNES"))
    assert t["well_depth"][0] == 38.0 and t["collision_diameter"][0] == 2.920 * 0.1
    assert t["well_depth"][6] == 572.4 and t["collision_diameter"][6] == 2.605 * 0.1


def test_collision_integral_matches_tabulated_values(om):
    """Neufeld fit against the Hirschfelder-Curtiss-Bird table of the (1,1)
    integral: 1.439 at T* = 1, 0.9490 at T* = 3, 0.7424 at T* = 10."""
    for T_red, ref in ((1.0, 1.439), (3.0, 0.9490), (10.0, 0.7424)):
        assert abs(op.lib().orc_omega(T_red, 1, 1) / ref - 1.0) < 2e-3


def test_binary_coefficients_match_published_values(om):
    """H2-N2 0.78 cm2/s and O2-N2 0.20 cm2/s at 298 K, 1 atm (within 5 %)."""
    sp = om.species()
    d = om.binary_diffusion(298.0, P_ATM, sp.index("H2"), sp.index("N2"))
    assert abs(d / 0.78e-4 - 1.0) < 0.05
    d = om.binary_diffusion(298.0, P_ATM, sp.index("O2"), sp.index("N2"))
    assert abs(d / 0.202e-4 - 1.0) < 0.05
    # D ~ T^1.5 / (p Omega): halving p doubles it exactly
    a = om.binary_diffusion(1500.0, P_ATM, 0, 1)
    assert om.binary_diffusion(1500.0, 0.5 * P_ATM, 0, 1) == pytest.approx(2.0 * a, rel=1e-15)


def test_trace_species_in_a_pure_gas_gets_the_binary_coefficient(om):
    sp = om.species()[:9]
    W = om.tables()["molar_mass"]
    n2 = sp.index("N2")
    T = np.array([300.0, 1200.0, 2400.0])
    p = np.full(3, P_ATM)
    Y = np.zeros((9, 3))
    Y[n2] = 1.0
    for k in range(9):
        if k == n2:
            continue
        Yk = Y.copy()
        Yk[k] = 1e-14
        D = om.mixture_diffusivity(T, p, Yk, np.full(3, W[n2]))
        for c in range(3):
            assert D[k, c] == pytest.approx(om.binary_diffusion(T[c], p[c], k, n2), rel=1e-10)


def test_bc_cells_and_invalid_states_get_zero(om):
    W = om.tables()["molar_mass"]
    n = 4
    Y = np.full((9, n), 1.0 / 9)
    mm = np.full(n, 1.0 / np.sum(Y[:, 0] / W))
    T = np.array([1000.0, 1000.0, -1.0, 1000.0])
    p = np.array([P_ATM, P_ATM, P_ATM, 0.0])
    D = om.mixture_diffusivity(T, p, Y, mm, bc=np.array([0, 1, 0, 0], np.int8))
    assert np.all(D[:, 0] > 0) and np.all(D[:, 1:] == 0)


def test_missing_species_is_an_error(tmp_path):
    from nrg_b200.chemistry import NrgError, transport_tables
    lines = open(transport_path("KEROMNES")).read().splitlines()
    bad = tmp_path / "no_h2o2.txt"
    bad.write_text("\n".join(l for l in lines if not l.startswith("H2O2 ")) + "\n")
    with pytest.raises(NrgError):
        transport_tables(*mechanism_paths("KEROMNES"), str(bad))
    m = op.Mechanism(*mechanism_paths("KEROMNES"), 1.0, "cal.mol")
    with pytest.raises(RuntimeError):
        m.load_transport(str(bad))

"""The product's deck reader (libnrg_chem, host only) against the oracle's
restatement of the reference readers: tables must agree bit for bit."""
import numpy as np
import pytest

from nrg_b200 import chemistry


def test_product_parser_matches_oracle(decks, oracle_mech):
    p = chemistry.mechanism_tables(*decks, 1.0, "cal.mol")
    o = oracle_mech.tables()
    assert p["n_species"] == 9 and p["n_reactions"] == 24
    np.testing.assert_array_equal(p["reaction_type"], o["reaction_type"])
    np.testing.assert_array_equal(p["coeffs"], o["coeffs"])
    arr = np.stack([o["A"], o["beta"], o["E_act"], o["A_low"], o["beta_low"], o["E_act_low"],
                    o["troe"][:, 0], o["troe"][:, 1], o["troe"][:, 2]], axis=1)
    np.testing.assert_array_equal(p["arrhenius"], arr)
    np.testing.assert_array_equal(p["troe3"], o["troe"][:, 3])
    np.testing.assert_array_equal(p["eff"], o["eff"])
    np.testing.assert_array_equal(p["a_coeffs"], o["a_coeffs"])
    np.testing.assert_array_equal(p["molar_mass"], o["molar_mass"])


def test_units_and_default_efficiency(decks, oracle_mech):
    p = chemistry.mechanism_tables(*decks, 0.5, "kcal.mol")
    o = chemistry.mechanism_tables(*decks, 1.0, "cal.mol")
    np.testing.assert_allclose(p["arrhenius"][:, 2], o["arrhenius"][:, 2] * 1000.0, rtol=1e-15)
    # unlisted species take the default; listed ones keep the deck value
    assert p["eff"][0, 0] == 0.5 and p["eff"][4, 0] == 2.5


def test_missing_deck_is_an_error(decks, tmp_path):
    import pytest
    with pytest.raises(chemistry.NrgError):
        chemistry.mechanism_tables(str(tmp_path / "none.txt"), decks[1], decks[2])


def test_bad_units_rejected(decks):
    import pytest
    with pytest.raises(KeyError):
        chemistry.mechanism_tables(*decks, 1.0, "erg.mol")


@pytest.mark.parametrize("name", ["KEROMNES", "ZHANG", "TEREZA", "KONNOV", "ACETYLENE"])
def test_other_reference_mechanisms_parse_alike(name):
    """The reference's other decks (H2/air, and C2H2/O2 with the FFCM-1
    thermo data): the product reader and the oracle's restatement give the
    same tables bit for bit."""
    from nrg_b200 import eact_units, mechanism_paths
    from oracle import oracle_py as op
    paths = mechanism_paths(name)
    p = chemistry.mechanism_tables(*paths, 1.0, eact_units(name))
    o = op.Mechanism(*paths, 1.0, eact_units(name)).tables()
    assert p["n_species"] == len(o["species"]) - 1
    np.testing.assert_array_equal(p["reaction_type"], o["reaction_type"])
    np.testing.assert_array_equal(p["coeffs"], o["coeffs"])
    arr = np.stack([o["A"], o["beta"], o["E_act"], o["A_low"], o["beta_low"], o["E_act_low"],
                    o["troe"][:, 0], o["troe"][:, 1], o["troe"][:, 2]], axis=1)
    np.testing.assert_array_equal(p["arrhenius"], arr)
    np.testing.assert_array_equal(p["troe3"], o["troe"][:, 3])
    np.testing.assert_array_equal(p["eff"], o["eff"])
    np.testing.assert_array_equal(p["a_coeffs"], o["a_coeffs"])
    np.testing.assert_array_equal(p["molar_mass"], o["molar_mass"])


def test_acetylene_deck_structure():
    """ACETYLENE_Varatharajan.txt: 17 species, 25 irreversible reactions
    (types 5, and 6 for the five third-body ones), E_act in J/mol."""
    from nrg_b200 import eact_units, mechanism_paths
    t = chemistry.mechanism_tables(*mechanism_paths("ACETYLENE"), 1.0, eact_units("ACETYLENE"))
    assert t["n_species"] == 17 and t["n_reactions"] == 25
    assert set(t["reaction_type"].tolist()) == {5, 6} and int(np.sum(t["reaction_type"] == 6)) == 5
    # H+O2=>OH+O  3.52E+16 -0.70 71400.0: A in m^3/(mol s) (2 reactants: x 1e-6), E unchanged
    assert t["arrhenius"][0, 0] == 3.52e16 * 1e-6 and t["arrhenius"][0, 2] == 71400.0

"""The table_approximated mode without a GPU: the table file format (the
writer and reader of chemical_kinetics_solver.f90:542-650) in the library
against the oracle, known answers of the Fortran E14.7 edit descriptor, and
the oracle's interpolation rules (:651-685)."""
import numpy as np
import pytest

from nrg_b200 import chemistry
from nrg_b200.chemistry import DataManager
from oracle import oracle_py as op

NAMES = ["H2", "O2", "N2", "O", "H", "OH", "H2O", "HO2", "H2O2"]


@pytest.mark.parametrize("x,text", [
    (300.5, " 0.3005000E+03"), (-1.234567e-4, "-0.1234567E-03"), (0.0, " 0.0000000E+00"),
    (2400.0, " 0.2400000E+04"), (9999999.5, " 0.1000000E+08"), (1e-120, " 0.1000000-119"),
    (-2.5e150, "-0.2500000+151"), (0.5, " 0.5000000E+00"), (float("nan"), "           NaN"),
])
def test_e14_7_known_answers(x, text):
    assert op.format_e14_7(x) == text
    if x == x:
        assert op.parse_e14_7(text) == float(text.replace("E", "e") if "E" in text else
                                             text[:-4] + "e" + text[-4:])


@pytest.mark.parametrize("field,value", [
    ("  1234567     ", 0.1234567), ("    1.5D3     ", 1500.0), ("   -25-3      ", -2.5e-9),
    ("              ", 0.0), (" 0.3005000E+03", 300.5), ("   .5E1       ", 5.0), ("  +7.25e-2    ", 0.0725),
])
def test_e14_7_input_rules(field, value):
    assert op.parse_e14_7(field) == pytest.approx(value, rel=1e-15)


def _flame_row(n=64, lb=0, seed=3):
    """A 1-D row with a ghost layer: T rising from 300 K through 305 K to a
    peak, then a plateau; Y_prod2 values over many decades."""
    rng = np.random.default_rng(seed)
    m = DataManager((0, 1, 1), (n + 1, 1, 1), (1, 1, 1), (n, 1, 1))  # cells(0:n+1, 1:1, 1:1), a 1-D block
    T = m.create_scalar_field("temperature")
    y2 = m.create_vector_field("specie_production_chemistry2", 9)
    prof = 300.0 + 2100.0 / (1.0 + np.exp(-(np.arange(n) - n / 2) / 4.0))
    prof[n // 2:] = np.maximum.accumulate(prof[n // 2:])
    m.interior(T)[:, 0, 0] = prof
    T[0, 0, 0] = 250.0
    for k in range(9):
        y2[k][:, 0, 0] = rng.standard_normal(m.shape[0]) * 10.0 ** rng.uniform(-12, -1, m.shape[0])
    return m


def _oracle_write(mech, m, path):
    T = m.fields["temperature"][:, 0, 0]
    y2 = np.stack([a[:, 0, 0] for a in m.fields["specie_production_chemistry2"]])
    mech.table_write(path, m.lb[0], m.ub[0], m.lo[0], m.hi[0], T, y2)


def test_library_and_oracle_write_the_same_file(oracle_mech, tmp_path):
    m = _flame_row()
    chemistry.write_table(tmp_path / "lib.dat", NAMES, m)
    _oracle_write(oracle_mech, m, tmp_path / "orc.dat")
    a, b = (tmp_path / "lib.dat").read_bytes(), (tmp_path / "orc.dat").read_bytes()
    assert a == b
    lines = a.decode().splitlines()
    assert lines[0] == "T  r(H2)  r(O2)  r(N2)  r(O)  r(H)  r(OH)  r(H2O)  r(HO2)  r(H2O2)"
    assert all(len(x) == 140 for x in lines[1:])
    T = m.interior(m.fields["temperature"])[:, 0, 0]
    first = int(np.flatnonzero((T > 300.5) & (T < 310.0))[0])
    last = int(np.argmax(T))
    assert len(lines) - 1 == last - first + 1


def test_row_without_a_cell_near_300_k_starts_at_index_0(oracle_mech, tmp_path):
    """No interior cell between 300.5 and 310 K: the reference's min_index
    stays 0 and the table starts at cell 0, the ghost cell of the row."""
    m = _flame_row()
    T = m.fields["temperature"]
    T[1:, 0, 0] = np.maximum(T[1:, 0, 0], 320.0)
    chemistry.write_table(tmp_path / "lib.dat", NAMES, m)
    _oracle_write(oracle_mech, m, tmp_path / "orc.dat")
    assert (tmp_path / "lib.dat").read_bytes() == (tmp_path / "orc.dat").read_bytes()
    assert (tmp_path / "lib.dat").read_text().splitlines()[1].startswith(" 0.2500000E+03")


def test_library_and_oracle_read_the_same_rows(oracle_mech, tmp_path):
    m = _flame_row()
    chemistry.write_table(tmp_path / "t.dat", NAMES, m)
    T1, Y1 = chemistry.table_read(tmp_path / "t.dat", 9)
    T2, Y2 = op.table_read(tmp_path / "t.dat", 9)
    np.testing.assert_array_equal(T1, T2)
    np.testing.assert_array_equal(Y1, Y2)
    # rows are the written values rounded to seven significant digits
    T = m.interior(m.fields["temperature"])[:, 0, 0]
    first = int(np.flatnonzero((T > 300.5) & (T < 310.0))[0])
    np.testing.assert_allclose(T1, T[first:first + T1.size], rtol=5e-7)


def test_hand_written_table_with_blank_short_and_unusual_records(oracle_mech, tmp_path):
    rec = lambda vals: "".join(f"{v:>14s}" for v in vals)
    text = "\n".join([
        "", "  T  r(H2) ...",                                     # a blank record before the header
        rec(["0.3000000E+03"] + ["1234567"] * 9),                 # implied decimal point
        rec(["0.4000000E+03"] + ["1.5D-3"] * 9),
        "",                                                       # blank record: a row of zeros
        rec(["0.6000000E+03", "-0.2500000-101"]),                 # short record, 3-digit exponent
        rec(["0.7000000E+03"] + ["-0.1000000E+01"] * 9) + "\r",
    ]) + "\n"
    (tmp_path / "h.dat").write_text(text)
    T1, Y1 = chemistry.table_read(tmp_path / "h.dat", 9)
    T2, Y2 = op.table_read(tmp_path / "h.dat", 9)
    np.testing.assert_array_equal(T1, T2)
    np.testing.assert_array_equal(Y1, Y2)
    # 5 non-blank records: header + 4 rows; the 4 records after the header
    # include the blank one
    np.testing.assert_array_equal(T1, [300.0, 400.0, 0.0, 600.0])
    assert Y1[0, 0] == 0.1234567 and Y1[0, 1] == 1.5e-3 and Y1[0, 3] == -2.5e-102 and Y1[1, 3] == 0.0


def test_malformed_table_is_an_error(tmp_path):
    (tmp_path / "bad.dat").write_text("T\n" + " 0.3000000E+03" + "   abc        " * 9 + "\n")
    with pytest.raises(chemistry.NrgError):
        chemistry.table_read(tmp_path / "bad.dat", 9)
    (tmp_path / "empty.dat").write_text("T header only\n")
    with pytest.raises(chemistry.NrgError):
        chemistry.table_read(tmp_path / "empty.dat", 9)


def test_oracle_interpolation_rules(oracle_mech):
    T_t = np.array([400.0, 800.0, 800.0, 1600.0, 2400.0])
    Y_t = np.outer(np.arange(1, 10), [1.0, 2.0, 3.0, 4.0, 5.0]) * 1e-3
    T = np.array([300.0, 350.0, 400.0, 600.0, 800.0, 1200.0, 2400.0, 2500.0])
    n = T.size
    Y = np.full((9, n), 0.1)
    bc = np.zeros(n, np.int8)
    o = oracle_mech.table_step(T_t, Y_t, 1e-6, T, Y, bc=bc, Y_prod2_init=np.full((9, n), 7.0))
    W = oracle_mech.tables()["molar_mass"]
    val = o["Y_prod"] * 1e-6 / W[:, None]
    np.testing.assert_array_equal(o["Y_prod"][:, 0], 0.0)           # skipped (< 305 K)
    np.testing.assert_array_equal(o["Y_prod2"][:, 0], 7.0)          # untouched
    np.testing.assert_allclose(val[:, 1], 0.0, atol=0)             # below the first node
    np.testing.assert_allclose(val[:, 2], Y_t[:, 0], rtol=1e-14)    # on the first node
    np.testing.assert_allclose(val[:, 3], 0.5 * (Y_t[:, 0] + Y_t[:, 1]), rtol=1e-14)
    np.testing.assert_allclose(val[:, 4], Y_t[:, 2], rtol=1e-14)    # last interval holding 800 K: [800, 1600]
    np.testing.assert_allclose(val[:, 5], 0.5 * (Y_t[:, 2] + Y_t[:, 3]), rtol=1e-14)
    np.testing.assert_allclose(val[:, 6], Y_t[:, 4], rtol=1e-14)    # on the last node
    np.testing.assert_allclose(val[:, 7], Y_t[:, 4], rtol=1e-14)    # above: the last row
    np.testing.assert_allclose(o["Y_prod2"][:, 1:], val[:, 1:] - 0.1, rtol=1e-12)

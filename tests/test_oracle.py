"""The CPU oracle against hand-read deck values, an independent numpy
restatement of the rates, and scipy's BDF at tight tolerance.  The reference
ships no golden vectors for this path, so these checks pin the restatement."""
import numpy as np
import pytest

from oracle import oracle_py as op
from nrg_b200 import fields

R = 8.31446261815324


def test_species_and_reaction_count(oracle_mech):
    assert oracle_mech.species() == ["H2", "O2", "N2", "O", "H", "OH", "H2O", "HO2", "H2O2", "M"]
    assert oracle_mech.n_reactions == 24


def test_hand_read_deck_values(oracle_mech):
    t = oracle_mech.tables()
    cal = R / 1.98720425864083
    # KEROMNES.txt:29  H+O2<=>O+OH  1.04E+14 0.00 15286.0 (bimolecular: A*1e-6)
    assert t["reaction_type"][0] == 0
    assert list(t["coeffs"][0][0]) == [2, 5, 2, 0] and list(t["coeffs"][1][0]) == [2, 4, 6, 0]
    assert t["A"][0] == 1.04e14 * 1e-6 and t["E_act"][0] == 15286.0 * cal
    # :33 H2+M<=>H+H+M with H2/2.5/ H2O/12/ (CO, CO2, HE not in the mechanism)
    assert t["reaction_type"][4] == 1
    assert list(t["coeffs"][1][4]) == [3, 5, 5, 10]
    assert t["eff"][4][0] == 2.5 and t["eff"][4][6] == 12.0 and t["eff"][4][1] == 1.0
    # :41-44 H+O2(+M)<=>HO2(+M) Troe: A*1e-6, A_low*1e-12
    assert t["reaction_type"][8] == 3
    assert t["A"][8] == 4.650e12 * 1e-6 and t["A_low"][8] == 1.737e19 * 1e-12
    assert list(t["troe"][8]) == [0.67, 1.0e-30, 1.0e30, 1.0e30]
    # :45-52 bath-gas duplicates: every mechanism species has efficiency 0
    assert np.all(t["eff"][9] == 0.0) and np.all(t["eff"][10] == 0.0)
    # :62-63 exponent without a letter: 4.8749+04
    assert t["E_act"][17] == 48749.0 * cal and t["E_act_low"][17] == 48749.0 * cal
    assert t["A"][17] == 2.0e12 and t["A_low"][17] == 2.49e24 * 1e-6
    # :65 H2O/0.0/ CO2/1.6/ N2/1.5/ O2/1.2/ HE/0.65/ H2O2/7.7/ H2/3.7/ CO/2.8/
    assert list(t["eff"][17]) == [3.7, 1.2, 1.5, 1.0, 1.0, 1.0, 0.0, 1.0, 7.7]
    # molar_masses.dat
    assert t["molar_mass"][0] == 2.0159e-3 and t["molar_mass"][8] == 3.4015e-2
    # KEROMNES_THERMO.txt H2 block: high range first, low range second, times R
    assert t["a_coeffs"][0][1][0] == pytest.approx(0.02991423e2 * R, rel=0, abs=0)
    assert t["a_coeffs"][0][0][0] == 0.03298124e2 * R
    assert t["a_coeffs"][0][0][6] == -0.03294094e2 * R
    # OH block carries a trailing 15th number on its last record: ignored
    assert t["a_coeffs"][5][0][6] == -1.03998477e-01 * R


def test_gear_coefficients():
    el, tq = op.ddcst(5)
    # BDF order 1 (backward Euler) and order 2 l-vectors
    assert el[0, 0] == 1.0 and el[1, 0] == 1.0
    assert el[0, 1] == pytest.approx(2.0 / 3.0) and el[2, 1] == pytest.approx(1.0 / 3.0)
    assert tq[1, 0] == pytest.approx(2.0)


def test_dnrm2_matches_two_norm():
    rng = np.random.default_rng(1)
    for scale in (1e-30, 1e-12, 1.0, 1e12, 1e25):
        x = rng.standard_normal(9) * scale
        assert op.dnrm2(x) == pytest.approx(np.linalg.norm(x), rel=1e-14)
    assert op.dnrm2(np.zeros(9)) == 0.0


def _numpy_rates(t, Tc, mc):
    a = t["a_coeffs"][:, 1 if Tc >= 1000 else 0, :]
    h = (((((a[:, 4] / 5 * Tc + a[:, 3] / 4) * Tc + a[:, 2] / 3) * Tc + a[:, 1] / 2) * Tc + a[:, 0]) + a[:, 5] / Tc) * Tc
    s = ((((a[:, 4] / 4 * Tc + a[:, 3] / 3) * Tc + a[:, 2] / 2) * Tc + a[:, 1]) * Tc + a[:, 6]) + a[:, 0] * np.log(Tc)
    kf = np.zeros(24)
    kr = np.zeros(24)
    for r in range(24):
        Lr = [x for x in t["coeffs"][0][r][1:1 + t["coeffs"][0][r][0]] if x != 10]
        Pr = [x for x in t["coeffs"][1][r][1:1 + t["coeffs"][1][r][0]] if x != 10]
        ds = sum(s[p - 1] for p in Pr) - sum(s[q - 1] for q in Lr)
        dh = sum(h[p - 1] for p in Pr) - sum(h[q - 1] for q in Lr)
        dnu = t["coeffs"][1][r][0] - t["coeffs"][0][r][0]
        kinf = t["A"][r] * Tc ** t["beta"][r] * np.exp(-t["E_act"][r] / R / Tc)
        k = kinf
        if t["reaction_type"][r] in (2, 3):
            k0 = t["A_low"][r] * Tc ** t["beta_low"][r] * np.exp(-t["E_act_low"][r] / R / Tc)
            pr = k0 * mc[r] / kinf
            k = kinf * pr / (1 + pr)
            if t["reaction_type"][r] == 3:
                al, T3, T1, T2 = t["troe"][r]
                Fc = (1 - al) * np.exp(-Tc / T3) + al * np.exp(-Tc / T1) + np.exp(-T2 / Tc)
                c = -0.4 - 0.67 * np.log10(Fc)
                nn = 0.75 - 1.27 * np.log10(Fc)
                if pr > 0:
                    k *= Fc ** (1 / (1 + ((np.log10(pr) + c) / (nn - 0.14 * (np.log10(pr) + c))) ** 2))
                else:
                    k *= Fc ** (-1 / 0.14)
        kf[r] = k
        kr[r] = k / (np.exp(ds / R - dh / R / Tc) * (101325 / R / Tc) ** dnu)
    return kf, kr


def _numpy_rhs(t, z, kf, kr, mc):
    zd = np.zeros(9)
    for r in range(24):
        f, b = kf[r], kr[r]
        L = t["coeffs"][0][r][1:1 + t["coeffs"][0][r][0]]
        P = t["coeffs"][1][r][1:1 + t["coeffs"][1][r][0]]
        for x in L:
            f *= mc[r] if x == 10 else z[x - 1]
        for x in P:
            b *= mc[r] if x == 10 else z[x - 1]
        for x in L:
            if x != 10:
                zd[x - 1] += b - f
        for x in P:
            if x != 10:
                zd[x - 1] += f - b
    return zd


def test_rates_and_rhs_independent_restatement(oracle_mech, W):
    t = oracle_mech.tables()
    f = fields.random_field(W)
    for c in range(0, f.n, 397):
        C0 = f.Y[:, c] * f.rho[c] / W
        mc = np.array([np.sum(C0 * t["eff"][r]) for r in range(24)])
        kf, kr = oracle_mech.rate_constants(f.T[c], mc)
        kf2, kr2 = _numpy_rates(t, f.T[c], mc)
        np.testing.assert_allclose(kf, kf2, rtol=1e-12)
        np.testing.assert_allclose(kr, kr2, rtol=1e-12)
        zd = oracle_mech.rhs(kf, kr, mc, C0)
        zd2 = _numpy_rhs(t, C0, kf, kr, mc)
        np.testing.assert_allclose(zd, zd2, rtol=1e-9, atol=1e-12 * np.max(np.abs(zd)))


def test_oracle_against_scipy_bdf(oracle_mech, W):
    from scipy.integrate import solve_ivp
    t = oracle_mech.tables()
    f = fields.random_field(W)
    sel = np.arange(0, f.n, 256)
    out = oracle_mech.chem_step(f.dt, f.T[sel], f.rho[sel], f.Y[:, sel])
    for j, c in enumerate(sel):
        C0 = f.Y[:, c] * f.rho[c] / W
        mc = np.array([np.sum(C0 * t["eff"][r]) for r in range(24)])
        kf, kr = oracle_mech.rate_constants(f.T[c], mc)
        sol = solve_ivp(lambda tt, z: oracle_mech.rhs(kf, kr, mc, z), (0, f.dt), C0, method="BDF",
                        rtol=1e-13, atol=1e-20)
        dY_ref = (sol.y[:, -1] - C0) * W / f.rho[c]
        dY = out["Y_prod"][:, j] * f.dt / f.rho[c]
        assert np.max(np.abs(dY - dY_ref)) < 5e-10


def test_oracle_conservation_and_skip_rule(oracle_mech, W):
    f = fields.random_field(W)
    n = 512
    T = f.T[:n].copy()
    T[:8] = 300.0  # below the 305 K threshold
    bc = np.zeros(n, np.int8)
    bc[8:16] = 1
    init2 = np.full((9, n), 7.0)
    out = oracle_mech.chem_step(f.dt, T, f.rho[:n], f.Y[:, :n], bc=bc, Y_prod2_init=init2)
    assert np.all(out["Y_prod"][:, :16] == 0.0) and np.all(out["E_f_prod"][:16] == 0.0)
    assert np.all(out["Y_prod2"][:, :16] == 7.0)  # not written for skipped cells
    assert np.all(out["nstate"][16:] == 2)
    # mass sources cancel only to the molar-mass table's consistency
    # (molar_masses.dat: H2 = 2.0159e-3 but 2 H = 2.0160e-3); atoms cancel exactly
    yp = out["Y_prod"][:, 16:]
    assert np.all(np.abs(yp.sum(0)) <= 1e-4 * np.abs(yp).sum(0) + 1e-300)
    E = np.array([[2, 0, 0, 0, 1, 1, 2, 1, 2], [0, 2, 0, 1, 0, 1, 1, 2, 2], [0, 0, 2, 0, 0, 0, 0, 0, 0]], float)
    dC = out["Y_prod2"][:, 16:]
    C = f.Y[:, 16:n] * f.rho[16:n] / W[:, None]
    assert np.max(np.abs(E @ dC) / (E @ C)) < 1e-10


def test_oracle_mxstep_flag(oracle_mech, W):
    f = fields.random_field(W)
    out = oracle_mech.chem_step(f.dt, f.T[:64], f.rho[:64], f.Y[:, :64], mxstep=5)
    assert np.all(out["nstate"] == 3) and np.all(out["nstep"] == 5)


def test_energy_closure_round_trip(oracle_mech, W):
    f = fields.random_field(W)
    n = 64
    zero = np.zeros((9, n))
    T1 = oracle_mech.temperature_after(f.dt, f.T[:n], f.rho[:n], f.Y[:, :n], zero, np.zeros(n))
    np.testing.assert_allclose(T1, f.T[:n], rtol=1e-9)


def _energy_per_mass(m, T, Y, W, v):
    """Total energy per mass of (T, Y, v): sensible internal energy above
    T_ref plus kinetic (the inverse of the state equation's energy)."""
    R = 8.31446261815324
    X = Y / W[:, None]
    Wm = 1.0 / X.sum(0)
    X = X * Wm
    e = np.zeros(T.shape[0])
    h0 = np.zeros(T.shape[0])
    for c in range(T.shape[0]):
        for k in range(W.shape[0]):
            e[c] += (m.enthalpy(T[c], k) - R * T[c]) * X[k, c]
            h0[c] += m.enthalpy(298.15, k) * X[k, c]
    return (e - h0) / Wm + 0.5 * (v * v).sum(0)


def test_state_equation_recovers_temperature(oracle_mech, W):
    """apply_state_equation inverts the energy of a known state: T back to
    the Newton tolerance, p = rho R T / W_mix, gamma and v_s consistent."""
    from nrg_b200 import fields
    f = fields.slice_field(fields.random_field(W), 256)
    rng = np.random.default_rng(5)
    v = rng.uniform(-300.0, 300.0, (2, f.n))
    E = _energy_per_mass(oracle_mech, f.T, f.Y, W, v)
    out = oracle_mech.apply_state(f.rho, f.Y, E, f.T * 0.9, v=v)
    assert np.all(out["status"] == 1)
    assert np.max(np.abs(out["T"] - f.T)) < 1e-6
    Wm = 1.0 / (f.Y / W[:, None]).sum(0)
    np.testing.assert_allclose(out["p"], f.rho * 8.31446261815324 * out["T"] / Wm, rtol=1e-14)
    np.testing.assert_allclose(out["mix_mol_mass"], Wm, rtol=1e-14)
    assert np.all((out["gamma"] > 1.0) & (out["gamma"] < 1.67))
    np.testing.assert_allclose(out["v_s"], np.sqrt(out["gamma"] * out["p"] / f.rho), rtol=1e-14)


def test_state_equation_applies_the_chemistry_sources(oracle_mech, W):
    """Y += Y_prod dt / rho and E_f += E_f_prod dt / rho before the state
    equation; bc cells untouched."""
    from nrg_b200 import fields
    f = fields.slice_field(fields.random_field(W), 64)
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y)
    E = _energy_per_mass(oracle_mech, f.T, f.Y, W, np.zeros((0, f.n)))
    bc = np.zeros(f.n, np.int8)
    bc[:4] = 1
    out = oracle_mech.apply_state(f.rho, f.Y, E, f.T, dt=f.dt, Y_prod=o["Y_prod"], E_f_prod=o["E_f_prod"], bc=bc)
    act = bc == 0
    np.testing.assert_array_equal(out["Y"][:, ~act], f.Y[:, ~act])
    np.testing.assert_allclose(out["Y"][:, act], (f.Y + o["Y_prod"] * f.dt / f.rho)[:, act], rtol=0, atol=1e-15)
    # the closure of the chemistry step gives the same temperature
    T1 = oracle_mech.temperature_after(f.dt, f.T, f.rho, f.Y, o["Y_prod"], o["E_f_prod"])
    assert np.max(np.abs(out["T"][act] - T1[act])) < 1e-6
    assert np.all(out["status"][~act] == 0)

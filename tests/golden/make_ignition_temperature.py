"""Finds the frozen-temperature ignition temperature used by the 262,144-cell
uneven-work field: the T at which the time of peak OH production of the
stoichiometric H2/air mixture (1 atm, radicals 1e-12) is 1e-5 s.

Uses the CPU oracle (test infrastructure) and prints the value that
nrg_b200/fields.py records as T_IGNITION_1E5.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle_py as op  # noqa: E402
from nrg_b200 import fields  # noqa: E402

D = os.path.join(ROOT, "nrg_b200", "data", "mechanism")


def peak_oh_time(m, W, T, t_end=4e-5, n_out=400):
    Yr, Yp, idx = fields._stoich(W)
    Y = Yr.copy()
    for s in fields.RADICALS:
        Y[idx[s]] = 1e-12
    Y /= Y.sum()
    Wmix = 1.0 / np.sum(Y / W)
    rho = fields.P_ATM * Wmix / (fields.R_GAS * T)
    dt = t_end / n_out
    oh = [Y[idx["OH"]]]
    Yc = Y.copy()
    for _ in range(n_out):
        out = m.chem_step(dt, np.array([T]), np.array([rho]), Yc[:, None], threads=1)
        Yc = Yc + out["Y_prod"][:, 0] * dt / rho
        oh.append(Yc[idx["OH"]])
    rate = np.diff(np.array(oh)) / dt
    return (np.argmax(rate) + 0.5) * dt


def main():
    m = op.Mechanism(os.path.join(D, "KEROMNES.txt"), os.path.join(D, "KEROMNES_THERMO.txt"),
                     os.path.join(D, "molar_masses.dat"), 1.0, "cal.mol")
    W = m.tables()["molar_mass"]
    lo, hi = 900.0, 1600.0
    for _ in range(14):
        mid = 0.5 * (lo + hi)
        if peak_oh_time(m, W, mid) > 1e-5:
            lo = mid
        else:
            hi = mid
    print(f"T_IGNITION_1E5 = {0.5 * (lo + hi):.1f}")


if __name__ == "__main__":
    main()

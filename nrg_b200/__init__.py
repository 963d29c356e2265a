"""B200-native chemistry step for NRG (per-cell stiff H2/air kinetics).

nrg_b200.chemistry -- C-ABI bindings and the reference-named operator
nrg_b200.fields    -- seeded synthetic cell fields of the benchmark shapes
nrg_b200.build     -- in-tree nvcc build of libnrg_chem.so (sm_100a)
"""
import os

MECH_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden", "mechanism")


def keromnes_paths():
    """The reference's H2/air input decks (mechanism, thermo, molar masses)."""
    return (os.path.join(MECH_DIR, "KEROMNES.txt"), os.path.join(MECH_DIR, "KEROMNES_THERMO.txt"),
            os.path.join(MECH_DIR, "molar_masses.dat"))

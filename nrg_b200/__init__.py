"""B200-native chemistry step for NRG (per-cell stiff H2/air kinetics).

nrg_b200.chemistry -- C-ABI bindings and the reference-named operator
nrg_b200.fields    -- seeded synthetic cell fields of the benchmark shapes
nrg_b200.build     -- in-tree nvcc build of libnrg_chem.so (sm_100a)
"""
import os

MECH_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden", "mechanism")


MECHANISMS = ("KEROMNES", "ZHANG", "TEREZA", "KONNOV")


def mechanism_paths(name: str = "KEROMNES"):
    """Input decks of one of the reference's H2/air mechanisms (mechanism,
    thermo, molar masses), as in its task_setup directory."""
    if name not in MECHANISMS:
        raise ValueError(f"unknown mechanism {name!r}; have {MECHANISMS}")
    return (os.path.join(MECH_DIR, f"{name}.txt"), os.path.join(MECH_DIR, f"{name}_THERMO.txt"),
            os.path.join(MECH_DIR, "molar_masses.dat"))


def keromnes_paths():
    """The reference's H2/air input decks (mechanism, thermo, molar masses)."""
    return mechanism_paths("KEROMNES")


def transport_path(name: str = "KEROMNES"):
    """The mechanism's transport deck (Lennard-Jones parameters), as in the
    reference's task_setup/thermophysical_data directory."""
    if name not in MECHANISMS:
        raise ValueError(f"unknown mechanism {name!r}; have {MECHANISMS}")
    return os.path.join(MECH_DIR, f"{name}_TRANSDATA.txt")

"""B200-native chemistry step for NRG (per-cell stiff H2/air kinetics).

nrg_b200.chemistry -- C-ABI bindings and the reference-named operator
nrg_b200.fields    -- seeded synthetic cell fields of the benchmark shapes
nrg_b200.build     -- in-tree nvcc build of libnrg_chem.so (sm_100a)
"""
import os

# the reference's input decks (task_setup/chemical_mechanisms, task_setup/thermophysical_data)
MECH_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "mechanism")


# the reference's H2/air mechanisms (task_setup/chemical_mechanisms)
MECHANISMS = ("KEROMNES", "ZHANG", "TEREZA", "KONNOV")
# plus its C2H2/O2 deck, the only one with carbon species, whose thermo and
# transport data are the FFCM-1 files of task_setup/thermophysical_data
ALL_MECHANISMS = MECHANISMS + ("ACETYLENE",)
_DECKS = {"ACETYLENE": ("ACETYLENE_Varatharajan.txt", "FFCM-1_thermo.txt", "FFCM-1_transport.txt")}


def _check_name(name: str) -> None:
    if name not in ALL_MECHANISMS:
        raise ValueError(f"unknown mechanism {name!r}; have {ALL_MECHANISMS}")


def mechanism_paths(name: str = "KEROMNES"):
    """Input decks of one of the reference's mechanisms (mechanism, thermo,
    molar masses), as in its task_setup directory."""
    _check_name(name)
    mech, thermo = (_DECKS[name][:2] if name in _DECKS else (f"{name}.txt", f"{name}_THERMO.txt"))
    return (os.path.join(MECH_DIR, mech), os.path.join(MECH_DIR, thermo), os.path.join(MECH_DIR, "molar_masses.dat"))


def eact_units(name: str = "KEROMNES") -> str:
    """Activation-energy units of the deck (its header comment; the H2/air
    setups use cal.mol, 1D_laminar_velocity.f90:327-336)."""
    _check_name(name)
    return "J.mol" if name == "ACETYLENE" else "cal.mol"


def keromnes_paths():
    """The reference's H2/air input decks (mechanism, thermo, molar masses)."""
    return mechanism_paths("KEROMNES")


def transport_path(name: str = "KEROMNES"):
    """The mechanism's transport deck (Lennard-Jones parameters), as in the
    reference's task_setup/thermophysical_data directory."""
    _check_name(name)
    return os.path.join(MECH_DIR, _DECKS[name][2] if name in _DECKS else f"{name}_TRANSDATA.txt")

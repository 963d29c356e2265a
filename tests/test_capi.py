"""The C-ABI library loads and exports every symbol include/nrg_chem.h declares."""
import os
import re

from nrg_b200 import chemistry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            out |= set(re.findall(r"NRG_API\s+[\w\s\*]+?\b(nrg_\w+)\s*\(", src))
    return out


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) >= 15
    L = chemistry.lib()
    for n in sorted(names):
        assert hasattr(L, n), n


def test_bindings_cover_the_header():
    assert declared_symbols() <= set(chemistry.SIGNATURES)


def test_create_error_is_reported_without_gpu(decks, tmp_path):
    import ctypes
    import pytest
    L = chemistry.lib()
    h = ctypes.c_void_p()
    rc = L.nrg_chem_create(str(tmp_path / "missing.txt").encode(), decks[1].encode(), decks[2].encode(),
                           1.0, 2, ctypes.byref(h))
    assert rc == -2 and b"cannot open" in L.nrg_chem_last_error(None)
    with pytest.raises(chemistry.NrgError):
        chemistry.ChemicalKineticsSolver(None, str(tmp_path / "missing.txt"), *decks[1:])


def build_c_driver(out_dir) -> str:
    """Compiles tests/c_abi_driver.c against include/nrg_chem.h and links it
    with libnrg_chem.so, as a C (or Fortran bind(C)) host code would."""
    import subprocess
    exe = os.path.join(str(out_dir), "c_abi_driver")
    libdir = os.path.dirname(chemistry.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c_abi_driver.c"), "-L", libdir, "-lnrg_chem",
                        "-Wl,-rpath," + libdir, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_driver_compiles_and_links_against_the_header(tmp_path):
    chemistry.lib()  # builds the library if needed
    assert os.path.exists(build_c_driver(tmp_path))

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def decks():
    from nrg_b200 import keromnes_paths
    return keromnes_paths()


@pytest.fixture(scope="session")
def oracle_mech(decks):
    from oracle import oracle_py as op
    return op.Mechanism(*decks, 1.0, "cal.mol")


@pytest.fixture(scope="session")
def W(oracle_mech):
    return oracle_mech.tables()["molar_mass"]


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False

"""nrg_mixture_diffusivity_device (calculate_diffusivity_coeff,
fickean_diffusion_solver.f90:358-395) against the oracle on the wide-range
state distribution (T ~ U[800, 2600] K, p ~ U[0.5, 5] atm) for the four
reference mechanisms.  Tolerance: 1e-12 relative per coefficient (the device
and host pow / exp may differ in the last bit; the rest of the arithmetic is
the reference's, in its order)."""
import numpy as np
import pytest

from nrg_b200 import MECHANISMS, fields, mechanism_paths, transport_path

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.mark.parametrize("name", MECHANISMS)
def test_diffusivity_matches_oracle(name):
    import torch
    from nrg_b200.chemistry import ChemicalKineticsSolver, mechanism_tables
    from oracle import oracle_py as op
    paths = mechanism_paths(name)
    W = mechanism_tables(*paths)["molar_mass"]
    s = ChemicalKineticsSolver(None, *paths, mode="fast")
    try:
        s.load_transport(transport_path(name))
        W9 = mechanism_tables(*mechanism_paths("KEROMNES"))["molar_mass"]
        base = fields.slice_field(fields.wide_range_field(W9, n_side=128), 8192, stride=2)
        f = fields.state_for_species(base, s.species_names, W)
        mm = 1.0 / np.sum(f.Y / W[:, None], axis=0)
        bc = (np.arange(f.n) % 97 == 5).astype(np.int8)
        om = op.Mechanism(*paths, 1.0, "cal.mol")
        om.load_transport(transport_path(name))
        Do = om.mixture_diffusivity(f.T, f.p, f.Y, mm, bc=bc)
        d = torch.device("cuda")
        t = lambda a: torch.tensor(np.ascontiguousarray(a), device=d)
        D = torch.full(f.Y.shape, -1.0, dtype=torch.float64, device=d)
        s.mixture_diffusivity_device(t(f.T), t(f.p), t(f.Y), t(mm), D, bc=t(bc))
        Dg = D.cpu().numpy()
    finally:
        s.close()
    assert np.all((Dg == 0) == (Do == 0))
    assert np.all(Dg[:, bc != 0] == 0)
    nz = Do != 0
    assert np.max(np.abs(Dg[nz] / Do[nz] - 1.0)) <= RTOL

"""The device species predictor (nrg_species_predictor_device, the
low-Mach solver's calculate_interm_Y_predictor,
fds_low_mach_solver.f90:785-954) against the oracle, bit for bit: both
perform the reference's operations in its order without contraction."""
import numpy as np
import pytest

from nrg_b200 import fields

pytestmark = pytest.mark.gpu

OUT = ("rho", "Y", "rho_old", "Y_old", "rho_int", "Y_int")


def run_both(solver, W, b, parts=(), **kw):
    import torch
    from oracle import oracle_py as op
    N = W.shape[0]
    args = dict(x_center=b.x_center, bc=b.bc, Y_prod_diff=b.Y_prod_diff, Y_prod_chem=b.Y_prod_chem)
    args.update(kw)
    o = op.species_predictor(W, b.dims, b.n_cells, b.coord, b.dx, b.dt, b.v_f, b.rho, b.Y, np.full(b.ld, 7.0),
                             np.full((N, b.ld), 7.0), Y_prod_part=parts, rho_old=np.full(b.ld, -1.0),
                             Y_old=np.full((N, b.ld), -1.0), **args)
    d = torch.device("cuda")
    t = lambda a: None if a is None else torch.tensor(np.ascontiguousarray(a), device=d)
    g = dict(rho=t(b.rho), Y=t(b.Y), rho_old=t(np.full(b.ld, -1.0)), Y_old=t(np.full((N, b.ld), -1.0)),
             rho_int=t(np.full(b.ld, 7.0)), Y_int=t(np.full((N, b.ld), 7.0)))
    solver.species_predictor_device(b.dt, b.dims, b.n_cells, b.dx, [t(v) for v in b.v_f], g["rho"], g["Y"],
                                    g["rho_old"], g["Y_old"], g["rho_int"], g["Y_int"], coord=b.coord,
                                    x_center=t(args["x_center"]), bc=t(args["bc"]), Y_prod_diff=t(args["Y_prod_diff"]),
                                    Y_prod_chem=t(args["Y_prod_chem"]), Y_prod_particles=[t(p) for p in parts])
    torch.cuda.synchronize()
    return o, {k: v.cpu().numpy().reshape(o[k].shape) for k, v in g.items()}


def assert_same(o, g):
    for k in OUT:
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    yield s
    s.close()


@pytest.mark.parametrize("dims,n,coord", [(2, (100, 70), 0), (1, (257,), 0), (3, (20, 12, 9), 0),
                                          (2, (64, 40), 1), (1, (50,), 2), (2, (33, 9), 2), (2, (31, 1), 0)])
def test_predictor_matches_oracle(solver, W, dims, n, coord):
    b = fields.predictor_block(W, dims, n, seed=11 + dims, coord=coord)
    o, g = run_both(solver, W, b)
    assert_same(o, g)


def test_predictor_optional_sources_and_particles(solver, W):
    b = fields.predictor_block(W, 2, (70, 45), seed=21)
    rng = np.random.Generator(np.random.PCG64(5))
    parts = [rng.normal(0.0, 30.0, b.Y.shape) for _ in range(2)]
    assert_same(*run_both(solver, W, b, parts=parts))
    assert_same(*run_both(solver, W, b, Y_prod_diff=None, Y_prod_chem=None, bc=None))


def test_predictor_all_clipped_cells(solver, W):
    b = fields.predictor_block(W, 2, (40, 20), seed=22, bc_fraction=0.0)
    b.Y_prod_chem[:, 500:540] = -1e12
    o, g = run_both(solver, W, b)
    assert np.any(o["rho"] == 7.0)
    assert_same(o, g)


def test_predictor_other_species_count(W):
    """A 10-species mechanism (TEREZA) on the same block shape."""
    from nrg_b200 import mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver, mechanism_tables
    paths = mechanism_paths("TEREZA")
    W10 = mechanism_tables(*paths)["molar_mass"]
    s = ChemicalKineticsSolver(None, *paths, mode="fast")
    try:
        b = fields.predictor_block(W, 2, (48, 30), seed=23)
        Y10 = np.zeros((10, b.ld))
        Y10[:9] = b.Y
        b.Y = Y10
        b.Y_prod_diff = np.vstack([b.Y_prod_diff, np.zeros((1, b.ld))])
        b.Y_prod_chem = np.vstack([b.Y_prod_chem, np.zeros((1, b.ld))])
        assert_same(*run_both(s, W10, b))
    finally:
        s.close()

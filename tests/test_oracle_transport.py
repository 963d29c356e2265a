"""The oracle's species predictor (oracle/orc_transport.c, the restatement of
calculate_interm_Y_predictor, fds_low_mach_solver.f90:785-954) against
properties of the scheme: free-stream preservation, conservation with closed
walls, uniform composition kept by the equation-of-state correction, and the
reference's all-clipped rule."""
import numpy as np
import pytest

from nrg_b200 import fields
from oracle import oracle_py as op


def run(W, b, **kw):
    N = W.shape[0]
    args = dict(x_center=b.x_center, bc=b.bc, Y_prod_diff=b.Y_prod_diff, Y_prod_chem=b.Y_prod_chem)
    args.update(kw)
    return op.species_predictor(W, b.dims, b.n_cells, b.coord, b.dx, b.dt, b.v_f, b.rho, b.Y,
                                np.full(b.ld, 7.0), np.full((N, b.ld), 7.0), **args)


def interior_mask(b):
    n = list(b.n_cells) + [1] * (3 - b.dims)
    e = [n[d] + 2 if d < b.dims else 1 for d in range(3)]
    m = np.zeros(e[::-1], bool)
    sl = tuple(slice(1, -1) if d < b.dims else slice(None) for d in (2, 1, 0))
    m[sl] = True
    return m.reshape(-1)


@pytest.mark.parametrize("dims,n", [(1, (50,)), (2, (30, 17)), (3, (9, 7, 6))])
def test_free_stream_is_preserved(W, dims, n):
    """Uniform state and uniform velocity, no sources: nothing changes."""
    b = fields.predictor_block(W, dims, n, seed=3)
    b.rho[:] = b.rho[0]
    b.Y[:] = b.Y[:, :1]
    for v in b.v_f:
        v[:] = 3.0
    o = run(W, b, bc=None, Y_prod_diff=None, Y_prod_chem=None)
    act = interior_mask(b)
    np.testing.assert_allclose(o["rho"][act], b.rho[act], rtol=1e-14)
    np.testing.assert_allclose(o["Y"][:, act], b.Y[:, act], rtol=1e-13, atol=1e-18)
    assert np.all(o["rho_old"][act] == b.rho[act]) and np.all(o["Y_old"][:, act] == b.Y[:, act])


def test_closed_walls_conserve_every_species(W):
    """Zero normal velocity on the domain's faces: sum over the cells of
    rho*Y_k changes only by dt times the (non-negative) sources."""
    b = fields.predictor_block(W, 2, (40, 24), seed=4, bc_fraction=0.0)
    nx, ny = b.n_cells
    fx, fy = nx + 3, ny + 3
    vx = b.v_f[0].reshape(fy, fx, 2)
    vy = b.v_f[1].reshape(fy, fx, 2)
    vx[:, 1, 0] = 0.0
    vx[:, nx + 1, 0] = 0.0
    vy[1, :, 1] = 0.0
    vy[ny + 1, :, 1] = 0.0
    b.v_f = [vx.reshape(-1), vy.reshape(-1)]
    b.Y_prod_chem = np.abs(b.Y_prod_chem)
    b.Y_prod_diff = np.abs(b.Y_prod_diff)
    o = run(W, b, bc=None)
    act = interior_mask(b)
    before = (b.rho[None, act] * b.Y[:, act]).sum(1) + b.dt * (b.Y_prod_diff[:, act] + b.Y_prod_chem[:, act]).sum(1)
    after = (o["rho"][None, act] * o["Y"][:, act]).sum(1)
    np.testing.assert_allclose(after, before, rtol=1e-12, atol=1e-16)


def test_uniform_composition_stays_uniform(W):
    """Same Y everywhere, density and velocities varying: the CHARM limiter
    is scale invariant and the EOS correction keeps sum_k phi_k / W_k on the
    face value of rho / W, so Y is unchanged (to rounding)."""
    b = fields.predictor_block(W, 2, (32, 20), seed=5)
    b.Y[:] = b.Y[:, [b.ld // 2]]
    o = run(W, b, bc=None, Y_prod_diff=None, Y_prod_chem=None)
    act = interior_mask(b)
    np.testing.assert_allclose(o["Y"][:, act], b.Y[:, act], rtol=1e-11, atol=1e-20)


def test_all_clipped_cell_keeps_rho_int(W):
    """Where every rho*Y_k clips to zero the reference leaves rho_int / Y_int
    as they were and then copies them into rho / Y."""
    b = fields.predictor_block(W, 1, (20,), seed=6, bc_fraction=0.0)
    b.Y_prod_chem[:, 5] = -1e12
    o = run(W, b)
    assert o["rho"][5] == 7.0 and np.all(o["Y"][:, 5] == 7.0)
    assert o["rho_old"][5] == b.rho[5]
    assert np.all(o["rho"][6:20] != 7.0)


def test_bc_cells_and_ghosts_untouched(W):
    b = fields.predictor_block(W, 2, (24, 16), seed=7, bc_fraction=0.1)
    o = run(W, b)
    skip = ~interior_mask(b) | (b.bc != 0)
    assert np.all(o["rho"][skip] == b.rho[skip]) and np.all(o["Y"][:, skip] == b.Y[:, skip])
    assert np.all(o["rho_int"][skip] == 7.0) and np.all(o["rho_old"][skip] == 0.0)


def test_bad_arguments_raise(W):
    b = fields.predictor_block(W, 1, (8,), seed=8)
    with pytest.raises(ValueError):
        op.species_predictor(W, 4, (8,), 0, b.dx, b.dt, b.v_f, b.rho, b.Y, b.rho.copy(), b.Y.copy())

"""nrg_chem_step called from a compiled C program (tests/c_abi_driver.c) on a
ghost-layered 3-D block of column-major arrays, the layout a Fortran host
code passes through ISO_C_BINDING (chemical_kinetics_solver.f90:81-107,
175): results against the CPU oracle, ghost cells untouched, skipped cells'
Y_prod2 left as the caller had it."""
import os
import subprocess

import numpy as np
import pytest

from nrg_b200 import fields, keromnes_paths
from tests.test_capi import build_c_driver

pytestmark = pytest.mark.gpu

TOL_Y = 1e-9


def test_c_program_steps_a_ghost_layered_block(tmp_path, oracle_mech, W):
    nx, ny, nz = 16, 12, 6
    n = nx * ny * nz
    f = fields.slice_field(fields.random_field(W), n, stride=3)
    f.T[:25] = 290.0                     # cold: skipped by the reference rule
    bc = np.zeros(n, np.int8)
    bc[25:60] = 1                        # boundary-marked: skipped
    N = f.Y.shape[0]
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as fh:
        np.array([nx, ny, nz, N], np.int32).tofile(fh)
        np.array([f.dt], np.float64).tofile(fh)
        f.T.tofile(fh)
        f.rho.tofile(fh)
        np.ascontiguousarray(f.Y).tofile(fh)
        bc.tofile(fh)
    exe = build_c_driver(tmp_path)
    r = subprocess.run([exe, *keromnes_paths(), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    raw = np.fromfile(out, np.float64, count=(2 * N + 1) * n)
    counts = np.fromfile(out, np.int64, offset=(2 * N + 1) * n * 8)
    Yp, Yp2, Ef = raw[:N * n].reshape(N, n), raw[N * n:2 * N * n].reshape(N, n), raw[2 * N * n:]
    o = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y, bc=bc, Y_prod2_init=np.full((N, n), 3.25))
    skipped = np.arange(n) < 60
    assert counts[0] == n and counts[1] == n - 60 and counts[2] == 0
    assert np.all(Yp[:, skipped] == 0.0) and np.all(Ef[skipped] == 0.0)
    assert np.all(Yp2[:, skipped] == 3.25)
    np.testing.assert_array_equal(Yp2[:, skipped], o["Y_prod2"][:, skipped])
    dy = np.abs(Yp - o["Y_prod"])[:, ~skipped] * f.dt / f.rho[None, ~skipped]
    assert dy.max() <= TOL_Y, dy.max()
    # Y_prod2 is the concentration change: Y_prod * dt / W
    d2 = np.abs(Yp2 - o["Y_prod2"])[:, ~skipped] / (f.rho[None, ~skipped] / W[:, None])
    assert d2.max() <= TOL_Y, d2.max()

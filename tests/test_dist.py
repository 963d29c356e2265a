"""Multi-process plumbing on CPU: the row partition and a two-rank gloo run
(no GPU): ranks step disjoint row blocks, the union equals the one-process
step bit for bit, and the timing reduction returns the slowest rank's value."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from nrg_b200 import dist, fields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("n_rows,world", [(64, 1), (64, 2), (2048, 8), (7, 3), (3, 4)])
def test_row_blocks_cover_every_row_once(n_rows, world):
    blocks = [dist.row_block(n_rows, r, world) for r in range(world)]
    covered = [i for a, b in blocks for i in range(a, b)]
    assert covered == list(range(n_rows))
    sizes = [b - a for a, b in blocks]
    assert max(sizes) - min(sizes) <= 1


def test_row_block_rejects_bad_rank():
    with pytest.raises(ValueError):
        dist.row_block(10, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_step_disjoint_rows(tmp_path, oracle_mech, W):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}",
           os.path.join(ROOT, "tests", "dist_worker.py"), str(tmp_path)]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = np.concatenate([np.load(tmp_path / f"rank{k}.npy") for k in range(2)], axis=1)
    f = fields.random_field(W)
    ref = oracle_mech.chem_step(f.dt, f.T, f.rho, f.Y, threads=1)["Y_prod"]
    np.testing.assert_array_equal(got, ref)
    assert float((tmp_path / "max.txt").read_text()) == 2.0


@pytest.mark.gpu
def test_two_ranks_step_row_blocks_through_the_product(tmp_path, W):
    """Two processes (gloo for the plumbing) step their row blocks of one
    field through nrg_chem_step_device on the one GPU: the blocks put
    together equal a single-process step of the whole field bit for bit."""
    import torch
    from nrg_b200 import keromnes_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver
    cmd = ["timeout", "-k", "30", "600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr=127.0.0.1", f"--master-port={_free_port()}",
           os.path.join(ROOT, "tests", "dist_worker.py"), str(tmp_path), "product"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=700)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = np.concatenate([np.load(tmp_path / f"rank{k}.npy") for k in range(2)], axis=1)
    f = fields.random_field(W)
    dev = torch.device("cuda:0")
    T, rho, Y = (torch.tensor(a, device=dev) for a in (f.T, f.rho, f.Y))
    Yp, Yp2, Ef = torch.zeros_like(Y), torch.zeros_like(Y), torch.zeros_like(T)
    s = ChemicalKineticsSolver(None, *keromnes_paths(), mode="fast")
    try:
        s.step_device(f.dt, T, rho, Y, Yp, Yp2, Ef)
        torch.cuda.synchronize()
    finally:
        s.close()
    np.testing.assert_array_equal(got, Yp.cpu().numpy())
    assert float((tmp_path / "max.txt").read_text()) == 2.0

"""The surrogate's BF16 tensor-core kernels against the float64 CPU reference
of the same network (oracle/mlp_ref.py), training, and the gated path."""
import numpy as np
import pytest

from nrg_b200 import fields
from oracle import mlp_ref
from tests.gpu_util import dY, run_device

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(decks):
    from nrg_b200.chemistry import ChemicalKineticsSolver
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    yield s
    s.close()


@pytest.fixture(scope="module")
def sur(solver):
    from nrg_b200.surrogate import Surrogate
    return Surrogate(solver)


def rand_batch(B, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = np.zeros((B, 16), np.float32)
    x[:, :12] = rng.standard_normal((B, 12))
    y = rng.standard_normal((B, 10)).astype(np.float32)
    xt = torch.tensor(x, device="cuda").to(torch.bfloat16)
    return xt, torch.tensor(y, device="cuda"), mlp_ref.bf16(x), y.astype(np.float64)


def test_forward_matches_cpu_reference(sur):
    sur.init(seed=11)
    p = sur.params()
    xt, _, x, _ = rand_batch(300, 1)
    out = sur.forward(xt).cpu().numpy()
    ref, _ = mlp_ref.forward(p, x)
    scale = np.max(np.abs(ref[:, :10]))
    assert np.max(np.abs(out[:, :10] - ref[:, :10])) <= 2e-2 * scale
    assert np.all(out[:, 10:] == 0.0)


def test_gradients_match_cpu_reference(sur):
    sur.init(seed=5)
    p = sur.params()
    xt, yt, x, y = rand_batch(512, 2)
    g, loss = sur.grad(xt, yt)
    loss_ref, g_ref = mlp_ref.loss_and_grad(p, x, y)
    assert loss == pytest.approx(loss_ref, rel=2e-2)
    off = 0
    for o, i in mlp_ref.SHAPES:
        for n in (o * i, o):
            a, b = g[off:off + n], g_ref[off:off + n]
            off += n
            assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b) + 1e-12, (o, i, n)


def test_training_reduces_loss(solver, sur, W):
    from nrg_b200.surrogate import training_pairs
    x, y, info = training_pairs(solver, W, 65536, seed=9)
    assert info["integrator_stats"]["cells_bad"] == 0
    sur.init(seed=1)
    losses = sur.train(x, y, epochs=4, batch=1024, lr=1e-3, seed=2)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0]


def test_save_load_round_trip(sur, tmp_path):
    sur.init(seed=3)
    p = sur.params()
    nrm = sur.norm()
    path = str(tmp_path / "m.bin")
    sur.save(path)
    sur.init(seed=4)
    sur.load(path)
    np.testing.assert_array_equal(sur.params(), p)
    np.testing.assert_array_equal(sur.norm(), nrm)

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


@pytest.fixture(scope="module")
def fitted(solver, sur, W):
    """Scaling fitted on 65,536 training pairs and a briefly trained network."""
    from nrg_b200.surrogate import training_pairs
    x, y, _ = training_pairs(solver, W, 65536, seed=9)
    sur.init(seed=1)
    sur.train(x, y, epochs=2, batch=1024, lr=1e-3, seed=2)
    return sur


def test_fused_inference_matches_unfused_and_cpu(fitted, W):
    f = fields.slice_field(fields.random_field(W), 2000)  # 15 full 128-cell tiles and a ragged one
    out_tc = fitted.infer(f).cpu().numpy()
    xb, _ = fitted.features(f, xraw=False)
    out_gemm = fitted.forward(xb).cpu().numpy()
    ref, _ = mlp_ref.forward(fitted.params(), xb.float().cpu().numpy().astype(np.float64))
    scale = np.max(np.abs(ref[:, :10]))
    assert np.max(np.abs(out_tc[:, :10] - ref[:, :10])) <= 2e-2 * scale
    assert np.max(np.abs(out_tc[:, :10] - out_gemm[:, :10])) <= 2e-2 * scale
    assert np.all(out_tc[:, 10:] == 0.0)


def test_fused_step_matches_unfused_step(solver, fitted, W):
    f = fields.slice_field(fields.random_field(W), 3000)
    f.T[:40] = 300.0
    f.T[1000:2000] = 700.0  # below the training hull (T >= 800 K less 2 %): FP64 fallback
    bc = np.zeros(f.n, np.int8)
    bc[40:80] = 1
    fitted.set_gate(1e-6, 1e9, 1e9, 1e9)  # open gate: the hull alone decides
    fitted.enable(True)
    res = {}
    try:
        for fused in (True, False):
            fitted.set_inference(fused)
            res[fused] = run_device(solver, f, "surrogate", bc=bc, y_prod2_init=np.full((9, f.n), 3.25))[0]
    finally:
        fitted.set_inference(True)
        solver.set_mode("fast")
    a, b = res[True], res[False]
    assert np.all(a["status"][:80] == 0) and np.all(b["status"][:80] == 0)
    assert np.all(a["Y_prod"][:, :80] == 0.0) and np.all(a["Y_prod2"][:, :80] == 3.25)
    same = a["status"] == b["status"]
    assert same.mean() >= 0.99, same.mean()
    sur_both = same & (a["status"] == 5)
    fb_both = same & (a["status"] == 1)
    assert sur_both.sum() > 1500 and 990 <= fb_both.sum() <= 1000, (sur_both.sum(), fb_both.sum())
    # the FP64 fallback gives the same bits whichever path chose the cell
    np.testing.assert_array_equal(a["Y_prod"][:, fb_both], b["Y_prod"][:, fb_both])
    np.testing.assert_array_equal(a["T_after"][fb_both], b["T_after"][fb_both])
    d = np.abs(a["Y_prod"] - b["Y_prod"])[:, sur_both] * f.dt / f.rho[None, sur_both]
    m = np.abs(b["Y_prod"])[:, sur_both].max() * f.dt / f.rho[sur_both].min()
    assert d.max() <= 2e-2 * m, (d.max(), m)


def test_trained_network_gain_on_flame_rows(decks, W):
    """What the trained network gains over the plain FP64 integrator on 128
    rows (262,144 cells) of the 2048 x 2048 flame field: the same step in less
    device time, accepted cells within |dT| <= 1 K and |dY_k| <= 1e-4 of the
    FP64 result, fallback cells bit-identical to it."""
    from nrg_b200.chemistry import ChemicalKineticsSolver
    from nrg_b200.surrogate import DEFAULT_MODEL, RECIPE, Surrogate
    full = fields.flame_field(W)
    f = fields.slice_field(full, 128 * 2048, offset=960 * 2048)
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        s.set_launch(kernel="thread", block=64)
        sur = Surrogate(s)
        sur.load(DEFAULT_MODEL)
        sur.set_gate(*RECIPE["gate"])
        plain, st_p = run_device(s, f, "fast")
        plain, st_p = run_device(s, f, "fast")
        sg, st_s = run_device(s, f, "surrogate")
        sg, st_s = run_device(s, f, "surrogate")
    finally:
        s.close()
    act = plain["status"] != 0
    acc = sg["status"] == 5
    fb = act & ~acc
    assert np.array_equal(sg["status"] == 0, ~act)
    assert acc.sum() >= 0.5 * act.sum(), (acc.sum(), act.sum())
    dT = np.abs(sg["T_after"] - plain["T_after"])[acc]
    dYk = (np.abs(sg["Y_prod"] - plain["Y_prod"]) * f.dt / f.rho[None, :])[:, acc]
    assert dT.max() <= 1.0 and dYk.max() <= 1e-4, (dT.max(), dYk.max())
    np.testing.assert_array_equal(sg["Y_prod"][:, fb], plain["Y_prod"][:, fb])
    np.testing.assert_array_equal(sg["T_after"][fb], plain["T_after"][fb])
    gain = st_p["device_ms"] / st_s["device_ms"]
    print(f"surrogate answers {acc.sum()} of {act.sum()} active cells; device time "
          f"{st_p['device_ms']:.1f} ms -> {st_s['device_ms']:.1f} ms ({gain:.2f}x)")
    assert gain > 1.2, gain


def test_fallback_order_changes_no_result(decks, W):
    """The surrogate's rejected cells go to the FP64 fallback grouped by
    temperature (default) or in cell order: the same bits and counts."""
    from nrg_b200.chemistry import ChemicalKineticsSolver
    from nrg_b200.surrogate import DEFAULT_MODEL, RECIPE, Surrogate
    f = fields.slice_field(fields.flame_field(W), 16 * 2048, offset=1000 * 2048)
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        s.set_launch(kernel="thread", block=32)
        sur = Surrogate(s)
        sur.load(DEFAULT_MODEL)
        sur.set_gate(*RECIPE["gate"])
        s.set_cell_order(False)
        a, sa = run_device(s, f, "surrogate")
        s.set_cell_order(True)
        b, sb = run_device(s, f, "surrogate")
    finally:
        s.close()
    for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after", "status"):
        np.testing.assert_array_equal(b[k], a[k], err_msg=k)
    for k in ("cells_active", "cells_surrogate", "cells_fallback", "steps", "solves"):
        assert sb[k] == sa[k], (k, sa, sb)
    assert 0 < sb["cells_fallback"] < sb["cells_active"]


def test_gate_sends_longer_steps_to_fp64(decks, W):
    """The gate bounds were calibrated on 1e-6 s steps.  On 1e-5 s steps of
    the wide-range distribution every cell goes to the FP64 integrator by
    default (results bit-equal to the plain step), and a flame sample with
    1e-6 s steps is answered by the network only while the bound admits
    1e-6 s."""
    from nrg_b200.chemistry import ChemicalKineticsSolver
    from nrg_b200.surrogate import DEFAULT_MODEL, RECIPE, Surrogate
    wide = fields.slice_field(fields.wide_range_field(W, n_side=256), 16384, stride=3)
    flame = fields.slice_field(fields.flame_field(W), 8 * 2048, offset=1000 * 2048)
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        s.set_launch(kernel="thread", block=32)
        sur = Surrogate(s)
        sur.load(DEFAULT_MODEL)
        sur.set_gate(*RECIPE["gate"])
        plain, _ = run_device(s, wide, "fast")
        sg, st = run_device(s, wide, "surrogate")
        fl, st_fl = run_device(s, flame, "surrogate")
        sur.set_gate_dt(5e-7)
        fl2, st_fl2 = run_device(s, flame, "surrogate")
    finally:
        s.close()
    assert st["cells_surrogate"] == 0 and st["cells_fallback"] == wide.n
    for k in ("Y_prod", "E_f_prod", "T_after"):
        np.testing.assert_array_equal(sg[k], plain[k])
    assert st_fl["cells_surrogate"] > 0
    assert st_fl2["cells_surrogate"] == 0 and np.all(fl2["status"][fl2["status"] != 0] == 1)


def test_gate_bands_by_step_length(decks, W):
    """nrg_surrogate_set_gate_band: a band admits steps up to its dt_max
    with its own bounds; steps above every band, and a band with dt_max 0 or
    with zero bounds, answer nothing (those cells get the plain step's bits)."""
    from nrg_b200.chemistry import ChemicalKineticsSolver, NrgError
    from nrg_b200.surrogate import DEFAULT_MODEL, RECIPE, Surrogate
    wide = fields.slice_field(fields.wide_range_field(W, n_side=256), 16384, stride=3)
    mid = fields.Field("mid", wide.T, wide.rho, wide.p, wide.Y, 3e-6, wide.shape)
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        s.set_launch(kernel="thread", block=32)
        sur = Surrogate(s)
        sur.load(DEFAULT_MODEL)
        sur.set_gate(*RECIPE["gate"])
        plain, _ = run_device(s, mid, "fast")
        _, st_none = run_device(s, mid, "surrogate")
        sur.set_gate_band(1, 5e-6, 1e-6, 5e-6, 0.2, 80.0)
        got, st_band = run_device(s, mid, "surrogate")
        sur.set_gate_band(2, 2e-6, 1e-6, 5e-6, 0.2, 80.0)  # not above band 1's bound: unused
        _, st_band2 = run_device(s, mid, "surrogate")
        sur.set_gate_band(1, 5e-6, 0.0, 0.0, 0.0, 0.0)
        _, st_zero = run_device(s, mid, "surrogate")
        sur.set_gate_band(1, 2e-6, 1e-6, 5e-6, 0.2, 80.0)
        _, st_short = run_device(s, mid, "surrogate")
        with pytest.raises(NrgError):
            sur.set_gate_band(4, 1e-5)
        with pytest.raises(NrgError):
            sur.set_gate_band(1, -1.0)
    finally:
        s.close()
    assert st_none["cells_surrogate"] == 0
    assert st_band["cells_surrogate"] > 0
    assert st_band2["cells_surrogate"] == st_band["cells_surrogate"]
    assert st_zero["cells_surrogate"] == 0 and st_short["cells_surrogate"] == 0
    rej = (got["status"] != 5) & (got["status"] != 0)
    for k in ("Y_prod", "Y_prod2"):
        np.testing.assert_array_equal(got[k][:, rej], plain[k][:, rej])


def test_step_band_routing(decks, W):
    """nrg_surrogate_set_dt_band: a network is routed only the cells whose
    step lies in its band (dt_lo, dt_hi]; outside it the cells go to FP64
    with the plain step's bits."""
    from nrg_b200.chemistry import ChemicalKineticsSolver, NrgError
    from nrg_b200.surrogate import DEFAULT_MODEL, RECIPE, Surrogate
    flame = fields.slice_field(fields.flame_field(W), 4 * 2048, offset=1000 * 2048)
    s = ChemicalKineticsSolver(None, *decks, mode="fast")
    try:
        s.set_launch(kernel="thread", block=32)
        sur = Surrogate(s)
        sur.load(DEFAULT_MODEL)
        sur.set_gate(*RECIPE["gate"])
        plain, _ = run_device(s, flame, "fast")
        _, st_in = run_device(s, flame, "surrogate")
        sur.set_dt_band(1e-6, 1e-5)  # the flame's 1e-6 s step is outside (1e-6, 1e-5]
        out, st_out = run_device(s, flame, "surrogate")
        sur.set_dt_band(5e-7, 1e-6)
        _, st_back = run_device(s, flame, "surrogate")
        with pytest.raises(NrgError):
            sur.set_dt_band(1e-5, 1e-6)
    finally:
        s.close()
    assert st_in["cells_surrogate"] > 0
    assert st_out["cells_surrogate"] == 0
    assert st_back["cells_surrogate"] == st_in["cells_surrogate"]
    for k in ("Y_prod", "Y_prod2", "E_f_prod", "T_after"):
        np.testing.assert_array_equal(out[k], plain[k])

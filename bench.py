#!/usr/bin/env python
"""Chemistry-step throughput on B200 (cell-updates/s), one JSON line.

Workload (default): the 2048 x 2048 premixed-flame field (4,194,304 cells,
dt = 1e-6 s, p = 1 atm) of the H2/air KEROMNES mechanism, synthetic and seeded
(nrg_b200/fields.py: flame_field).  A step is one chemistry step over the whole
field.  Inputs (370 MB of FP64 state) are larger than the 126 MB L2, so no
flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode surrogate|fast|reference|mixed]
  python bench.py --impl reference ...   # CPU restatement of the reference path

Multi-GPU (torchrun): every rank integrates its own full field (weak scaling,
no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "chem cell-updates/s: surrogate+fallback vs plain FP64, same GPU, |ΔT|≤1 K"
UNIT = "cell-updates/s"
H2D_BYTES_PER_CELL = 11 * 8 + 1   # T, rho, 9 Y, bc
D2H_BYTES_PER_CELL = 10 * 8 + 1   # 9 Y_prod2, E_f_prod, status (the host rebuilds Y_prod = Y_prod2 W / dt)
D2H_BYTES_PER_CELL_TABLE = 19 * 8 + 1  # table mode: 9 Y_prod as well


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="auto", choices=["auto", "surrogate", "fast", "reference", "mixed", "table"])
    p.add_argument("--field", default="flame", choices=["flame", "wide-range", "ignition"],
                   help="flame: 2048^2 flame field, dt=1e-6 s (the headline workload); wide-range: 1024^2 cells, "
                        "T~U[800,2600] K, p~U[0.5,5] atm, dt=1e-5 s; ignition: 512^2 cells, dt=1e-5 s, 20%% of "
                        "them within 50 K of the 1e-5 s ignition temperature")
    p.add_argument("--n-side", type=int, default=None, help="cells per side (default: the field's own size)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--kernel", choices=["thread", "thread_queue", "warp_queue"], default=None,
                   help="fix the integrator launch instead of autotuning it (with --block)")
    p.add_argument("--block", type=int, default=32)
    p.add_argument("--fallback-eps", type=float, default=None,
                   help="integrator tolerance of the surrogate's rejected cells (default: FALLBACK_EPS; 0: 1e-9)")
    p.add_argument("--cell-order", choices=["temperature", "cell"], default="temperature",
                   help="order in which the FP64 integrator takes the cells (same results)")
    p.add_argument("--mechanism", default="KEROMNES", choices=["KEROMNES", "ZHANG", "TEREZA", "KONNOV", "ACETYLENE"],
                   help="reference mechanism; the others run the plain FP64 path on the same flame field "
                        "(ACETYLENE: the same geometry with a C2H2/O2/Ar mixture)")
    p.add_argument("--no-predictor", dest="predictor", action="store_false",
                   help="skip timing the low-Mach species predictor on an n-side x n-side flame block "
                        "(nrg_species_predictor_device)")
    p.add_argument("--no-diffusivity", dest="diffusivity", action="store_false",
                   help="skip timing the mixture-averaged diffusion coefficients of the field "
                        "(nrg_mixture_diffusivity_device)")
    p.add_argument("--no-state-eq", dest="state_eq", action="store_false",
                   help="skip timing the sources + state-equation update of the field "
                        "(nrg_chem_apply_state_device)")
    p.add_argument("--no-table", dest="table", action="store_false",
                   help="skip timing the table_approximated mode on the field (a table of the flame's first "
                        "row, made by the plain integrator)")
    a = p.parse_args()
    if a.n_side is None:
        a.n_side = {"flame": 2048, "wide-range": 1024, "ignition": 512}[a.field]
    return a


def make_field(F, W, args):
    """The workload's synthetic cell field and its one-line description."""
    if args.field == "wide-range":
        f = F.wide_range_field(W, n_side=args.n_side)
        return f, (f"wide-range field {args.n_side}x{args.n_side} ({f.n:,} cells), dt=1e-5 s, "
                   "T~U[800,2600] K, p~U[0.5,5] atm")
    if args.field == "ignition":
        f = F.ignition_field(W, n_side=args.n_side)
        return f, (f"ignition field {args.n_side}x{args.n_side} ({f.n:,} cells), dt=1e-5 s, p=1 atm, 20% of cells "
                   "within 50 K of the 1e-5 s ignition temperature")
    f = F.flame_field(W, n_side=args.n_side)
    return f, f"flame field {args.n_side}x{args.n_side} ({f.n:,} cells), dt=1e-6 s, p=1 atm"


# --------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, kept for the timed region only.

    The sampler starts before the warm-up steps (nvidia-smi needs a moment
    before its first sample); begin() and end() mark the timed region and
    summary() keeps the samples whose nvidia-smi timestamps fall inside it."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self._p = None
        self._t = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits", "-lms", "100"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._p = None
        return self

    def _read(self):
        for line in self._p.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def __exit__(self, *a):
        if self._p:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()

    @staticmethod
    def _when(ts: str):
        import datetime
        try:
            return datetime.datetime.strptime(ts, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                t = self._when(r[0])
                if t is None or self.t0 is None or not (self.t0 <= t <= self.t1):
                    continue
                sm.append(float(r[2]))
                mx = float(r[3])
                for i, nm in enumerate(names):
                    if r[6 + i].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "window_s": None if self.t0 is None else round(self.t1 - self.t0, 3)}


def flop_model(tables: dict, mode: str) -> dict:
    """Algorithmic FP64 flops per counted event (reference formulation).

    rhs   : per reaction, one multiply per reactant and product factor and two
            adds per species update (chemical_kinetics_solver.f90:509-536)
    lu    : DGEFA on N x N: sum_k (N-k) + 2 (N-k)^2
    solve : DGESL: N(N-1) forward + N + N(N-1) backward, plus the corrector's
            residual and weighted norm (6N)
    jac   : FD (reference): 2N^2 to form columns and the matrix (its N right-hand
            sides are counted as rhs); analytic: partial products and updates
    step  : predictor, Nordsieck update, error weights and norms (~30N)
    setup : 9 NASA-7 species x 40 + 24 reactions x 30 (transcendentals as 1)
    """
    co = tables["coeffs"].tolist()
    N, R = int(tables["n_species"]), int(tables["n_reactions"])
    f_rhs = 0
    f_jac = 0
    for r in range(R):
        nl, nr = co[0][r][0], co[1][r][0]
        left = [x for x in co[0][r][1:1 + nl] if x != N + 1]
        right = [x for x in co[1][r][1:1 + nr] if x != N + 1]
        nupd = len(left) + len(right)
        f_rhs += nl + nr + 2 * nupd
        for side in (left, right):
            f_jac += len(side) * (max(len(side) - 1, 0) + 1 + nupd)
    f_lu = sum((N - k) + 2 * (N - k) ** 2 for k in range(1, N))
    f_sol = N * (N - 1) + N + N * (N - 1) + 6 * N
    f_jacform = 2 * N * N if mode == "reference" else f_jac + N * N
    return dict(rhs=f_rhs, lu=f_lu, solve=f_sol, jac=f_jacform + f_lu, step=30 * N,
                setup=9 * 40 + 24 * 30)


def algorithmic_flops(st: dict, fm: dict) -> float:
    st = {k: float(v) for k, v in st.items() if not isinstance(v, (list, tuple))}
    return ((st["cells_active"] - st.get("cells_surrogate", 0.0)) * fm["setup"] + st["rhs_evals"] * fm["rhs"] + st["jacobians"] * fm["jac"]
            + st["solves"] * fm["solve"] + st["steps"] * fm["step"])


def energy_per_mass(field, tables) -> np.ndarray:
    """Sensible internal energy per mass above T_ref of each cell (the energy
    the state equation inverts), from the NASA-7 tables: measurement set-up
    for --state-eq."""
    R = 8.31446261815324
    a = tables["a_coeffs"]  # (N, 2, 7), times R
    W = tables["molar_mass"]
    X = field.Y / W[:, None]
    Wm = 1.0 / X.sum(0)
    X = X * Wm

    def h(T):
        t = np.minimum(T, 6000.0)
        s = (t >= 1000.0).astype(int)
        out = np.zeros((W.shape[0], T.shape[0]))
        for k in range(W.shape[0]):
            c = a[k][s]  # (n, 7)
            v = c[:, 4] / 5.0
            for i in (3, 2, 1):
                v = v * t + c[:, i] / (i + 1.0)
            v = v * t + c[:, 0]
            out[k] = (v + c[:, 5] / t) * t
        return out

    e = ((h(field.T) - R * field.T[None, :]) * X).sum(0)
    h0 = (h(np.full_like(field.T, 298.15)) * X).sum(0)
    return (e - h0) / Wm


def load_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "fallback": True}


def cpu_baseline(field, W, decks, seconds: float, units: str = "cal.mol") -> dict:
    """CPU restatement of the reference path (oracle, all host cores) on a
    strided sample of the same field, sized to about `seconds` of work."""
    from oracle import oracle_py as op
    m = op.Mechanism(*decks, 1.0, units)
    cores = os.cpu_count() or 1
    probe = sample_cells(field, 4096, seed=1)
    t0 = time.perf_counter()
    m.chem_step(probe.dt, probe.T, probe.rho, probe.Y, threads=cores)
    rate = probe.n / max(time.perf_counter() - t0, 1e-6)
    n = int(min(field.n, max(probe.n, rate * seconds)))
    samp = sample_cells(field, n, seed=7)
    t0 = time.perf_counter()
    m.chem_step(samp.dt, samp.T, samp.rho, samp.Y, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} cells drawn uniformly (seeded) from the {field.name.replace('_', ' ')} "
                      f"({dt:.1f} s, OpenMP dynamic schedule)"}


def oracle_sample_index(field, seed: int = 21):
    """Cells of the workload on which the GPU results are checked against the
    oracle: for the flame field 34,816 cells drawn per temperature band (cold
    pass-through, preheat, front, trailing edge, burnt); otherwise 16,384
    cells drawn uniformly."""
    rng = np.random.default_rng(seed)
    if field.name != "flame_field":
        return np.sort(rng.choice(field.n, size=min(16384, field.n), replace=False))
    bands = [(0.0, 305.0, 2048), (305.0, 800.0, 8192), (800.0, 2380.0, 14336), (2380.0, 2399.9, 4096),
             (2399.9, 1e9, 6144)]
    idx = []
    for lo, hi, k in bands:
        band = np.flatnonzero((field.T >= lo) & (field.T < hi))
        idx.append(rng.choice(band, size=min(k, band.size), replace=False))
    return np.sort(np.concatenate(idx))


def accuracy_vs_oracle(field, decks, units, arms: dict) -> dict:
    """Maxima of |dY_k| and |dT| of each measured arm's outputs (from the
    full-field GPU run) against the oracle on a seeded sample of the same
    cells; the oracle is the checker here, not a timed path."""
    from oracle import oracle_py as op
    m = op.Mechanism(*decks, 1.0, units)
    idx = oracle_sample_index(field)
    samp = F_slice(field, idx)
    o = m.chem_step(samp.dt, samp.T, samp.rho, samp.Y)
    To = m.temperature_after(samp.dt, samp.T, samp.rho, samp.Y, o["Y_prod"], o["E_f_prod"])
    act = samp.T >= 305.0
    out = {"sample_cells": int(idx.size), "active_in_sample": int(act.sum()),
           "sample": ("cells drawn per temperature band (seeded)" if field.name == "flame_field"
                      else "cells drawn uniformly (seeded)")}
    for name, (Yp, Ta, st) in arms.items():
        Yp, Ta, st = Yp[:, idx], Ta[idx], st[idx]
        dY = (np.abs(Yp - o["Y_prod"]) * samp.dt / samp.rho[None, :])[:, act]
        dT = np.abs(Ta - To)[act]
        out[name] = {"max_abs_dY": float(dY.max()) if dY.size else 0.0,
                     "max_abs_dY_per_species": [float(v) for v in dY.max(1)] if dY.size else [],
                     "max_abs_dT_K": float(dT.max()) if dT.size else 0.0,
                     "max_rel_dT": float((dT / samp.T[act]).max()) if dT.size else 0.0,
                     "answered_by_network": int((st[act] == 5).sum())}
    return out


def F_slice(field, idx):
    from nrg_b200 import fields as F
    return F.Field(field.name, field.T[idx].copy(), field.rho[idx].copy(), field.p[idx].copy(),
                   np.ascontiguousarray(field.Y[:, idx]), field.dt, (len(idx),))


def sample_cells(field, n: int, seed: int):
    """n cells drawn uniformly without replacement (seeded), in cell order."""
    from nrg_b200 import fields as F
    idx = np.sort(np.random.default_rng(seed).choice(field.n, size=min(n, field.n), replace=False))
    return F.Field(field.name, field.T[idx].copy(), field.rho[idx].copy(), field.p[idx].copy(),
                   np.ascontiguousarray(field.Y[:, idx]), field.dt, (len(idx),))


# ------------------------------------------------------------ reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # the reference arm maps no library of the product: the field generator
    # is numpy only and the molar masses come from the oracle's own reader
    from nrg_b200 import fields as F, keromnes_paths
    from oracle import oracle_py as op
    decks = keromnes_paths()
    m = op.Mechanism(*decks, 1.0, "cal.mol")
    W = m.tables()["molar_mass"]
    field, desc = make_field(F, W, args)
    cores = os.cpu_count() or 1
    # sample sized so that a step takes ~ cpu-seconds
    probe = sample_cells(field, 4096, seed=1)
    t0 = time.perf_counter()
    m.chem_step(probe.dt, probe.T, probe.rho, probe.Y, threads=cores)
    rate = probe.n / max(time.perf_counter() - t0, 1e-6)
    n = int(min(field.n, max(probe.n, rate * args.cpu_seconds)))
    samp = sample_cells(field, n, seed=7)
    for _ in range(args.warmup):
        m.chem_step(samp.dt, samp.T, samp.rho, samp.Y, threads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        m.chem_step(samp.dt, samp.T, samp.rho, samp.Y, threads=cores)
    el = time.perf_counter() - t0
    value = args.steps * n / el
    sample = (f"{n} cells per step drawn uniformly (seeded) from the {desc}; "
              f"C restatement of the reference Fortran + SLATEC DDRIV3 path (no Fortran compiler on the box)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": f"{desc}, KEROMNES H2/air; CPU sample"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
MLP_FLOPS_PER_CELL = 2 * (12 * 128 + 3 * 128 * 128 + 128 * 10)
PROFILE = os.path.join(ROOT, "profiles", "fp64_integrator_flame.md")


def integrator_traffic(cells_integrated: float):
    """DRAM bytes (read + write) of one integrator launch: the per-cell figure
    of the committed ncu capture (line 'traffic_bytes_per_integrated_cell: N')
    times the cells this launch integrated."""
    try:
        with open(PROFILE) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_integrated_cell:"):
                    return float(line.split(":", 1)[1].split()[0]) * cells_integrated
    except OSError:
        pass
    return None


# Algorithmic HBM bytes per interior cell of the species predictor (N species):
# read rho, Y_k, the two normal face velocities, the diffusion and chemistry
# sources, bc; write rho_old, Y_old, rho_int, Y_int; the commit reads rho_int,
# Y_int and writes rho, Y.
def predictor_bytes_per_cell(N: int, dims: int = 2) -> int:
    return 8 * (N + 1) + 8 * dims + 8 * 2 * N + 1 + 8 * 2 * (N + 1) + 8 * 2 * (N + 1)


def time_predictor(solver, tables, args, dev, peaks) -> dict:
    """nrg_species_predictor_device on a 2048 x 2048 flame block (ghost layer
    included), 9 species, dt = 1e-7 s, seeded face velocities of both signs;
    inputs restored before each call (outside the timed region)."""
    import torch
    from nrg_b200 import fields as F
    N = int(tables["n_species"])
    W = np.asarray(tables["molar_mass"])
    b = F.predictor_block(W, 2, (args.n_side, args.n_side), seed=31, bc_fraction=0.0)
    if N != b.Y.shape[0]:
        return None
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    rho0, Y0 = t(b.rho), t(b.Y)
    rho, Y = rho0.clone(), Y0.clone()
    rho_old, Y_old, rho_int, Y_int = (torch.empty_like(x) for x in (rho0, Y0, rho0, Y0))
    v_f = [t(v) for v in b.v_f]
    diff, chem = t(b.Y_prod_diff), t(b.Y_prod_chem)
    times = []
    for rep in range(args.warmup + args.steps):
        rho.copy_(rho0)
        Y.copy_(Y0)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        solver.species_predictor_device(b.dt, 2, b.n_cells, b.dx, v_f, rho, Y, rho_old, Y_old, rho_int, Y_int,
                                        Y_prod_diff=diff, Y_prod_chem=chem)
        a1.record()
        torch.cuda.synchronize()
        if rep >= args.warmup:
            times.append(a0.elapsed_time(a1))
    ms = statistics.median(times)
    cells = args.n_side * args.n_side
    bpc = predictor_bytes_per_cell(N)
    gbs = bpc * cells / (ms * 1e-3) * 1e-9
    return {"ms": ms, "cells_per_s": cells / (ms * 1e-3), "bytes_per_cell": bpc, "algorithmic_GB_s": gbs,
            "frac_of_measured_hbm": gbs / peaks["hbm_gbs"], "launches": 2,
            "what": "nrg_species_predictor_device (k_predictor + k_predictor_commit): CHARM convective update "
                    "of rho*Y_k with the EOS correction, diffusion + chemistry sources, clip, renormalise; "
                    f"{args.n_side} x {args.n_side} cells, 2-D, inputs larger than L2"}


def time_diffusivity(solver, tables, args, dev, field, T, Y) -> dict:
    """nrg_mixture_diffusivity_device over the flame field (the mechanism's
    transport deck; mixture molar mass from Y)."""
    import torch
    from nrg_b200 import transport_path
    solver.load_transport(transport_path(args.mechanism))
    W = np.asarray(tables["molar_mass"])
    N = int(tables["n_species"])
    mm = torch.tensor(1.0 / np.sum(field.Y / W[:, None], axis=0), device=dev)
    p = torch.tensor(field.p, device=dev)
    D = torch.empty_like(Y)
    times = []
    for rep in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        solver.mixture_diffusivity_device(T, p, Y, mm, D)
        a1.record()
        torch.cuda.synchronize()
        if rep >= args.warmup:
            times.append(a0.elapsed_time(a1))
    ms = statistics.median(times)
    n = field.n
    bpc = 8 * (N + 3) + 8 * N  # read T, p, mix_mol_mass, Y; write D
    return {"ms": ms, "cells_per_s": n / (ms * 1e-3), "bytes_per_cell": bpc,
            "algorithmic_GB_s": bpc * n / (ms * 1e-3) * 1e-9, "pairs_per_cell": N * (N - 1) // 2,
            "what": "nrg_mixture_diffusivity_device: Chapman-Enskog binary coefficients (Neufeld collision "
                    "integral: one pow and three exp per species pair) and the mixture-averaged coefficient "
                    "of every species, every cell of the field"}


def table_bytes(n: int, active: int, N: int) -> int:
    """Algorithmic HBM bytes of one table-mode step without T_after or bc:
    every cell reads T and writes Y_prod, E_f_prod and its status byte;
    an active cell also reads Y and writes Y_prod2."""
    return n * (8 + 8 * N + 8 + 1) + active * (8 * N + 8 * N)


def make_flame_table(solver, W, path, n_side: int = 2048) -> None:
    """The table of the reference's table_approximated mode, made as the
    reference makes one: the first row of the flame field (a 1-D flame,
    300 K to 2400 K) stepped by the plain FP64 integrator, its T and Y_prod2
    written with the table writer (nrg_table_write)."""
    import torch
    from nrg_b200 import fields as F
    from nrg_b200.chemistry import DataManager, write_table
    row = F.slice_field(F.flame_field(W, n_side=n_side), n_side)
    dev = torch.device("cuda", torch.cuda.current_device())
    T, rho, Y = (torch.tensor(a, device=dev) for a in (row.T, row.rho, row.Y))
    Yp, Yp2, Ef = torch.zeros_like(Y), torch.zeros_like(Y), torch.zeros_like(T)
    solver.set_mode("fast")
    solver.step_device(row.dt, T, rho, Y, Yp, Yp2, Ef)
    torch.cuda.synchronize()
    m = DataManager((0, 1, 1), (n_side + 1, 1, 1), (1, 1, 1), (n_side, 1, 1))
    Tf = m.create_scalar_field("temperature")
    y2 = m.create_vector_field("specie_production_chemistry2", Y.shape[0])
    m.interior(Tf)[:, 0, 0] = row.T
    Yp2h = Yp2.cpu().numpy()
    for k in range(Y.shape[0]):
        m.interior(y2[k])[:, 0, 0] = Yp2h[k]
    write_table(path, solver.species_names, m)


def time_table(solver, W, args, dev, field, T, rho, Y, peaks, table_path, decks, units) -> dict:
    """The table_approximated mode over the whole field (nrg_chem_step_device,
    no T_after): device time, algorithmic HBM rate, and its sources against
    the oracle's table step on a sample of the field (bit for bit)."""
    import torch
    if not os.path.exists(table_path):
        make_flame_table(solver, W, table_path)
    solver.read_chemical_kinetics_table(table_path)
    solver.set_mode("table")
    n, N = field.n, Y.shape[0]
    Yp, Yp2, Ef = torch.zeros_like(Y), torch.zeros_like(Y), torch.zeros_like(T)
    st = torch.zeros(n, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        solver.step_device(field.dt, T, rho, Y, Yp, Yp2, Ef, status=st)
    torch.cuda.synchronize()
    times, stats = [], None
    for _ in range(args.steps):
        torch.cuda.synchronize()
        stats = solver.step_device(field.dt, T, rho, Y, Yp, Yp2, Ef, status=st)
        times.append(stats["device_ms"])
    ms = statistics.median(times)
    active = int(stats["cells_active"])
    nbytes = table_bytes(n, active, N)
    gbs = nbytes / (ms * 1e-3) * 1e-9
    from oracle import oracle_py as op
    idx = oracle_sample_index(field)
    samp = F_slice(field, idx)
    om = op.Mechanism(*decks, 1.0, units)
    T_t, Y_t = op.table_read(table_path, N)
    o = om.table_step(T_t, Y_t, samp.dt, samp.T, samp.Y)
    same = bool(np.array_equal(Yp[:, idx].cpu().numpy(), o["Y_prod"], equal_nan=True) and
                np.array_equal(Ef[idx].cpu().numpy(), o["E_f_prod"], equal_nan=True))
    solver.set_mode("fast")
    return {"ms": ms, "cells_per_s": n / (ms * 1e-3), "table_rows": int(T_t.size), "active_cells": active,
            "bytes_per_launch": nbytes, "algorithmic_GB_s": gbs, "frac_of_measured_hbm": gbs / peaks["hbm_gbs"],
            "sources_equal_oracle_on_sample": same, "sample_cells": int(idx.size),
            "what": "NRG_MODE_TABLE (ODE_solver = 'table_approximated'): Y_prod2 interpolated in T from a table of "
                    "the flame's first row (k_table_step; reads T and Y, writes Y_prod, Y_prod2, E_f_prod, status)"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as tdist
    from nrg_b200 import dist
    rank, world, local = dist.world()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init("nccl", timeout_s=600)
    from nrg_b200 import eact_units, fields as F, keromnes_paths, mechanism_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver, DataManager, fp64_peak_tflops, mechanism_tables
    from nrg_b200.surrogate import (DEFAULT_MODEL, FALLBACK_EPS, PREHEAT_MODEL, RECIPE, Surrogate, load_default,
                                    train_default)
    decks = mechanism_paths(args.mechanism)
    units = eact_units(args.mechanism)
    tables = mechanism_tables(*decks, 1.0, units)
    W = tables["molar_mass"]
    dev = torch.device("cuda", local)
    solver = ChemicalKineticsSolver(None, *decks, E_act_units=units, mode="fast")
    field, desc = make_field(F, mechanism_tables(*keromnes_paths())["molar_mass"], args)
    if args.field != "flame":
        # the widened rows are timed on flame blocks only
        args.predictor = args.diffusivity = args.state_eq = False
        if args.mechanism != "KEROMNES":
            raise SystemExit("--field other than flame is for the KEROMNES mechanism")
    if args.mechanism == "ACETYLENE":
        # the same flame geometry with the C2H2/O2/Ar mixture
        field = F.acetylene_flame(solver.species_names[:tables["n_species"]], W, n_side=args.n_side)
        args.no_e2e = True
        args.predictor = args.diffusivity = False
    elif args.mechanism != "KEROMNES":
        # the same flame, in the mechanism's species (others start at zero)
        field = F.state_for_species(field, solver.species_names[:tables["n_species"]], W)
        args.no_e2e = True
    n = field.n
    T, rho, Y = (torch.tensor(a, device=dev) for a in (field.T, field.rho, field.Y))
    in_bytes = n * (8 * (2 + Y.shape[0]) + 1)
    # inputs smaller than L2 (126 MB): a 256 MB buffer is rewritten between
    # timed steps so that every step reads its inputs from HBM
    l2_flush = torch.empty(32 << 20, dtype=torch.float64, device=dev) if in_bytes < (126 << 20) else None
    l2_note = (f"inputs ({in_bytes / 1e6:.0f} MB) larger than L2; no flush" if l2_flush is None else
               f"inputs ({in_bytes / 1e6:.0f} MB) smaller than L2: 256 MB written between timed steps (in the timed time)")

    solver.set_cell_order(args.cell_order == "temperature")
    # launch shape of the FP64 integrator: autotuned on a contiguous block of
    # 512 rows (a quarter of the field: large enough that the plain grid's last
    # wave weighs as little as on the whole field)
    if args.kernel:
        solver.set_launch(kernel=args.kernel, block=args.block)
    else:
        nsamp = min(n, 1048576)
        samp = F.slice_field(field, nsamp, stride=1, offset=(n - nsamp) // 2)
        sT, sr, sY = (torch.tensor(a, device=dev) for a in (samp.T, samp.rho, samp.Y))
        solver.autotune(samp.dt, sT, sr, sY, torch.zeros_like(sY), torch.zeros_like(sY), torch.zeros_like(sT))
        del sT, sr, sY
    launch = solver.get_launch()

    mode = args.mode
    if args.mechanism != "KEROMNES" and mode == "auto":
        mode = "fast"
    train_info = None
    if mode in ("auto", "surrogate"):
        if os.path.exists(DEFAULT_MODEL):
            nets = load_default(solver, args.fallback_eps)
            train_info = {"model": os.path.relpath(DEFAULT_MODEL, ROOT), "trained": "loaded",
                          "gate": list(RECIPE["gate"]),
                          "fallback_eps": FALLBACK_EPS if args.fallback_eps is None else args.fallback_eps}
            if len(nets) > 1:
                from nrg_b200.surrogate import RECIPE_PREHEAT
                train_info["preheat_model"] = os.path.relpath(PREHEAT_MODEL, ROOT)
                train_info["preheat_gate"] = list(RECIPE_PREHEAT["gate"])
        else:
            sur = Surrogate(solver)
            info = train_default(solver, W)
            sur.save(DEFAULT_MODEL)
            train_info = {"trained": "in this run", "pairs": info["n"], "epochs": info["recipe"]["epochs"],
                          "pairs_s": info["pairs_s"], "train_s": info["train_s"], "final_loss": info["losses"][-1],
                          "gate": list(RECIPE["gate"])}
        mode = "surrogate"
    peak_fp64 = fp64_peak_tflops()

    def make_out():
        return (torch.zeros_like(Y), torch.zeros_like(Y), torch.zeros_like(T), torch.zeros_like(T),
                torch.zeros(n, dtype=torch.uint8, device=dev))

    def time_arm(arm_mode):
        Yp, Yp2, Ef, Ta, st = make_out()
        solver.set_mode(arm_mode)
        stats = []
        with ClockSampler(local) as clk:
            for _ in range(args.warmup):
                solver.step_device(field.dt, T, rho, Y, Yp, Yp2, Ef, T_after=Ta, status=st)
            torch.cuda.synchronize()
            dist.barrier()
            torch.cuda.synchronize()
            clk.begin()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                if l2_flush is not None:
                    l2_flush.fill_(1.0)
                stats.append(solver.step_device(field.dt, T, rho, Y, Yp, Yp2, Ef, T_after=Ta, status=st))
            e1.record()
            torch.cuda.synchronize()
            clk.end()
        el = dist.max_over_ranks(e0.elapsed_time(e1), dev)  # the job's time: its slowest rank
        # one untimed step with per-phase events for the roofline
        solver.set_timing(True)
        ph = solver.step_device(field.dt, T, rho, Y, Yp, Yp2, Ef, T_after=Ta, status=st)
        solver.set_timing(False)
        return el, stats, ph, clk.summary(), (Yp, Yp2, Ef, Ta, st)

    import tempfile
    table_path = os.path.join(tempfile.mkdtemp(prefix="nrg_table_"), "flame_table(T).dat")
    if mode == "table":
        make_flame_table(solver, W, table_path)
        solver.read_chemical_kinetics_table(table_path)
    el_plain, st_plain, ph_plain, clk_plain, out_plain = time_arm("fast")
    if mode == "surrogate":
        el, stats, ph, clocks, out = time_arm("surrogate")
    else:
        solver.set_mode(mode)
        el, stats, ph, clocks, out = (el_plain, st_plain, ph_plain, clk_plain, out_plain) if mode == "fast" \
            else time_arm(mode)
    value = args.steps * n * world / (el * 1e-3)
    plain_value = args.steps * n * world / (el_plain * 1e-3)

    # accuracy of the measured path against the plain FP64 integrator
    acc = None
    if mode != "fast":
        Yp_p, _, _, Ta_p, st_p = (x.cpu().numpy() for x in out_plain)
        Yp_s, _, _, Ta_s, st_s = (x.cpu().numpy() for x in out)
        act = st_p != 0
        dT = np.abs(Ta_s - Ta_p)[act]
        dYk = (np.abs(Yp_s - Yp_p) * field.dt / field.rho[None, :])[:, act]
        acc = {"vs": "plain FP64 GPU integrator (same inputs)", "active_cells": int(act.sum()),
               "max_abs_dT_K": float(dT.max()), "p99_abs_dT_K": float(np.percentile(dT, 99)),
               "max_abs_dY": float(dYk.max()), "max_abs_dY_per_species": [float(v) for v in dYk.max(1)],
               "accepted_cells": int((st_s == 5).sum()), "fallback_cells": int(ph["cells_fallback"]),
               "fallback_fraction_of_active": float(ph["cells_fallback"]) / max(1, int(act.sum()))}
        if mode == "surrogate":
            # the integrated (rejected) cells alone: the fallback tolerance's share
            fb = (st_s[act] != 5)
            acc["fallback_max_abs_dT_K"] = float(dT[fb].max()) if fb.any() else 0.0
            acc["fallback_max_abs_dY"] = float(dYk[:, fb].max()) if fb.any() else 0.0

    state_eq = None
    if args.state_eq:
        # sources of the last plain step into (Y, E_f), then the state
        # equation, over the whole field; inputs restored before each call
        Yp_p, _, Ef_p, _, _ = out_plain
        E0 = torch.tensor(energy_per_mass(field, tables), device=dev)
        Yw, Ew, Tw = torch.empty_like(Y), torch.empty_like(E0), torch.empty_like(T)
        outs = [torch.empty_like(T) for _ in range(7)]
        stq = torch.empty(n, dtype=torch.uint8, device=dev)
        times = []
        for rep in range(args.warmup + args.steps):
            Yw.copy_(Y)
            Ew.copy_(E0)
            Tw.copy_(T)
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record()
            solver.apply_state_device(rho, Yw, Ew, Tw, outs[0], outs[1], time_step=field.dt, Y_prod=Yp_p,
                                      E_f_prod=Ef_p, cp_mass=outs[2], h_s=outs[3], h_full=outs[4], v_s=outs[5],
                                      mix_mol_mass=outs[6], status=stq)
            a1.record()
            torch.cuda.synchronize()
            if rep >= args.warmup:
                times.append(a0.elapsed_time(a1))
        ms = statistics.median(times)
        nsp = int(tables["n_species"])
        bpc = 8 * (2 * nsp + 5) + 8 * (nsp + 9) + 1  # read rho,Y,E_f,T,Y_prod,E_f_prod; write Y,E_f,T,7 props,status
        dT = np.abs(Tw.cpu().numpy() - out_plain[3].cpu().numpy())
        state_eq = {"ms": ms, "cells_per_s": n / (ms * 1e-3), "bytes_per_cell": bpc,
                    "algorithmic_GB_s": bpc * n / (ms * 1e-3) * 1e-9,
                    "max_abs_T_minus_step_closure_K": float(dT[out_plain[4].cpu().numpy() != 0].max()),
                    "what": "nrg_chem_apply_state_device: sources of the plain step into Y, E_f, then the state "
                            "equation (T Newton, p, gamma, cp, h_s, h_full, sound speed)"}

    predictor = None
    if args.predictor:
        predictor = time_predictor(solver, tables, args, dev, load_peaks())

    table_leg = None
    if args.table and args.mechanism == "KEROMNES":
        table_leg = time_table(solver, W, args, dev, field, T, rho, Y, load_peaks(), table_path, decks, units)

    diffusivity = None
    if args.diffusivity:
        diffusivity = time_diffusivity(solver, tables, args, dev, field, T, Y)

    e2e = None
    if not args.no_e2e:
        nx, ny = field.shape
        m = DataManager.block(nx, ny)
        for name in ("temperature", "pressure", "density"):
            m.create_scalar_field(name)
        m.create_vector_field("specie_mass_fraction", 9)
        m.interior(m.fields["temperature"])[...] = field.T.reshape(ny, nx).T[:, :, None]
        m.interior(m.fields["density"])[...] = field.rho.reshape(ny, nx).T[:, :, None]
        for k in range(9):
            m.interior(m.fields["specie_mass_fraction"][k])[...] = field.Y[k].reshape(ny, nx).T[:, :, None]
        host = ChemicalKineticsSolver(m, *decks, mode="fast")
        host.set_launch(**launch)
        host.set_cell_order(args.cell_order == "temperature")
        if mode == "surrogate":
            load_default(host, args.fallback_eps)
        if mode == "table":
            host.read_chemical_kinetics_table(table_path)
        host.set_mode(mode)
        host.solve_chemical_kinetics(field.dt)
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            host.solve_chemical_kinetics(field.dt)
        el2 = dist.max_over_ranks(time.perf_counter() - t0, dev)
        e2e = {"value": args.steps * n * world / el2, "unit": UNIT,
               "h2d_bytes_per_step": n * H2D_BYTES_PER_CELL, "d2h_bytes_per_step": n * (D2H_BYTES_PER_CELL_TABLE if mode == "table" else D2H_BYTES_PER_CELL),
               "path": "nrg_chem_step (host Fortran-layout arrays: chunks gathered and copied in while the "
                       "networks and gate run per chunk; FP64 fallback per half of the field; copied out and scattered)"}
        host.close()

    if rank == 0:
        st = stats[-1]
        peaks = load_peaks()
        arms = {"plain_fp64": tuple(out_plain[i].cpu().numpy() for i in (0, 3, 4))}
        if mode != "fast":
            arms[mode] = tuple(out[i].cpu().numpy() for i in (0, 3, 4))
        acc_oracle = accuracy_vs_oracle(field, decks, units, arms)
        fm = flop_model(tables, "fast")
        phases = {"inference_ms": ph["phase_ms"][0], "fallback_order_ms": ph["phase_ms"][1],
                  "integrator_ms": ph["phase_ms"][2]}
        integ_flops = algorithmic_flops(ph, fm)
        integ_tf = integ_flops / max(phases["integrator_ms"], 1e-9) * 1e-9
        roof = {"bound": "fp64", "achieved": integ_tf, "peak": peak_fp64, "unit": "TFLOP/s",
                "frac": integ_tf / peak_fp64,
                "traffic": integrator_traffic(float(ph["cells_active"]) - float(ph.get("cells_surrogate", 0))),
                "kernel": "FP64 BDF integrator (" + launch["kernel"] + "), the dominant kernel",
                "peak_source": "measured live: dependent-FMA FP64 probe (MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_launch": integ_flops, "flop_model": fm}
        roof_mlp = None
        if mode == "surrogate":
            # fused kernel: MLP of every active cell + the FP64 gate; tensor
            # share is a lower bound because the gate is inside the same time
            mlp_flops = MLP_FLOPS_PER_CELL * float(ph["cells_active"])
            mlp_tf = mlp_flops / max(phases["inference_ms"], 1e-9) * 1e-9
            roof_mlp = {"bound": "tensor", "achieved": mlp_tf, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                        "frac": mlp_tf / peaks["bf16_tflops"], "kernel": "k_mlp_gate_tc (features + 5 tcgen05 "
                        "layers + FP64 gate)", "flops_per_launch": mlp_flops,
                        "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst), of measured"}
        cpu = cpu_baseline(field, W, decks, args.cpu_seconds, units)
        # per step: fused MLP + gate (surrogate), the cell order (3 radix passes of
        # count / tile scan / digit scan / scatter, or 3 compaction kernels for the
        # fallback in cell order), the integrator
        if args.cell_order == "temperature":
            launches = 14 if mode == "surrogate" else 13
        else:
            launches = 5 if mode == "surrogate" else 1
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+bf16" if mode == "surrogate" else "f64",
            "data": "synthetic",
            "config": {"workload": f"{desc}, "
                                   f"{args.mechanism} {'C2H2/O2/Ar' if args.mechanism == 'ACETYLENE' else 'H2/air'} ({tables['n_species']} species, "
                                   f"{tables['n_reactions']} reactions)",
                       "path": {"fast": "plain FP64 integrator, analytic Jacobian",
                                "reference": "plain FP64 integrator, reference FD Jacobian",
                                "mixed": "FP32 LU + FP64 residual/refinement",
                                "surrogate": "BF16 MLP surrogate + gated FP64 fallback",
                                "table": "table_approximated: Y_prod2 interpolated in T"}[mode],
                       "launch": launch, "cell_order": args.cell_order, "l2": l2_note,
                       "active_cells": int(ph["cells_active"])},
            # long per-kernel blocks first; the headline figures close the line
            "accuracy": acc,
            "surrogate_model": train_info,
            "phases_ms": phases,
            "roofline_mlp": roof_mlp,
            "state_equation": state_eq,
            "species_predictor": predictor,
            "mixture_diffusivity": diffusivity,
            "table_mode": table_leg,
            "peaks_file": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained")},
            "accuracy_vs_oracle": acc_oracle,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps * launches,
            "clocks": clocks,
            "plain_fp64": {"value": plain_value, "ms_per_step": el_plain / args.steps},
            "plain_fp64_value": plain_value,
            "ratio_surrogate_over_plain": value / plain_value,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.barrier()
        tdist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

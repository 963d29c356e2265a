"""Seeded synthetic cell fields for the chemistry-step workloads.

Composition model (as the reference's H2/air set-ups,
package_interface/src/tests/classic_tests/1D_laminar_velocity.f90:269-271,
477-480): stoichiometric H2/air reactants H2:O2:N2 = 2:1:3.762 (mole), products
H2O:N2 = 2:3.762, blended in mass by a progress variable c, radicals
H, O, OH, HO2, H2O2 set separately, renormalised; rho = p W / (R T).
Species order is the mechanism's (KEROMNES: H2 O2 N2 O H OH H2O HO2 H2O2).
Arrays are species-major: Y[k, cell].
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

R_GAS = 8.31446261815324
P_ATM = 101325.0
SPECIES = ["H2", "O2", "N2", "O", "H", "OH", "H2O", "HO2", "H2O2"]
RADICALS = ["H", "O", "OH", "HO2", "H2O2"]
# Frozen-temperature ignition temperature of the stoichiometric mixture at
# 1 atm for which the time of peak OH production is 1e-5 s (oracle bisection,
# tests/golden/make_ignition_temperature.py).
T_IGNITION_1E5 = 1586.9


@dataclass
class Field:
    name: str
    T: np.ndarray       # (n,)
    rho: np.ndarray     # (n,)
    p: np.ndarray       # (n,)
    Y: np.ndarray       # (N, n)
    dt: float
    shape: tuple
    dt_cells: np.ndarray | None = None  # per-cell dt (training pairs)

    @property
    def n(self) -> int:
        return self.T.shape[0]


def _stoich(W: np.ndarray):
    idx = {s: i for i, s in enumerate(SPECIES)}
    Xr = np.zeros(len(SPECIES))
    Xr[idx["H2"]], Xr[idx["O2"]], Xr[idx["N2"]] = 2.0, 1.0, 3.762
    Xp = np.zeros(len(SPECIES))
    Xp[idx["H2O"]], Xp[idx["N2"]] = 2.0, 3.762
    Yr = Xr * W / np.sum(Xr * W)
    Yp = Xp * W / np.sum(Xp * W)
    return Yr, Yp, idx


def _finish(name, T, p, Y, W, dt, shape, dt_cells=None) -> Field:
    Y = Y / Y.sum(axis=0, keepdims=True)
    Wmix = 1.0 / np.sum(Y / W[:, None], axis=0)
    rho = p * Wmix / (R_GAS * T)
    return Field(name, np.ascontiguousarray(T), np.ascontiguousarray(rho), np.ascontiguousarray(p),
                 np.ascontiguousarray(Y), dt, shape, dt_cells)


def radical_mask() -> int:
    """Bit k set for each radical species k (mechanism order)."""
    return sum(1 << SPECIES.index(s) for s in RADICALS)


def random_state(n: int, rng: np.random.Generator, W: np.ndarray, T_lo: float, T_hi: float,
                 p_lo: float = 1.0, p_hi: float = 1.0, coupled: float = 0.0):
    """Each radical mass fraction is log-uniform on [1e-8, 1e-3].  The five
    radicals are drawn independently, except in a fraction `coupled` of the
    cells where they share one draw (same marginals, radical pools of one
    size, as at a flame front)."""
    Yr, Yp, idx = _stoich(W)
    T = rng.uniform(T_lo, T_hi, n)
    c = rng.uniform(0.0, 1.0, n)
    p = P_ATM * (rng.uniform(p_lo, p_hi, n) if p_hi > p_lo else np.full(n, p_lo))
    Y = (1.0 - c)[None, :] * Yr[:, None] + c[None, :] * Yp[:, None]
    u = rng.uniform(0.0, 1.0, (len(RADICALS), n))
    if coupled > 0.0:
        same = rng.uniform(0.0, 1.0, n) < coupled
        u[:, same] = u[0, same][None, :]
    for i, s in enumerate(RADICALS):
        Y[idx[s]] = 10.0 ** (-8.0 + 5.0 * u[i])
    return T, p, Y


def random_field(W: np.ndarray, n_side: int = 64) -> Field:
    """4,096 cells, T ~ U[1000, 2400] K, p = 1 atm, dt = 1e-6 s."""
    rng = np.random.Generator(np.random.PCG64(0))
    n = n_side * n_side
    T, p, Y = random_state(n, rng, W, 1000.0, 2400.0)
    return _finish("random_field", T, p, Y, W, 1e-6, (n_side, n_side))


def ignition_field(W: np.ndarray, n_side: int = 512) -> Field:
    """262,144 cells, dt = 1e-5 s; 20 % of cells within +-50 K of the
    temperature whose ignition delay is 1e-5 s (uneven substep counts)."""
    rng = np.random.Generator(np.random.PCG64(1))
    n = n_side * n_side
    T, p, Y = random_state(n, rng, W, 1000.0, 2400.0)
    hot = rng.uniform(0.0, 1.0, n) < 0.2
    T[hot] = T_IGNITION_1E5 + rng.uniform(-50.0, 50.0, int(hot.sum()))
    return _finish("ignition_field", T, p, Y, W, 1e-5, (n_side, n_side))


def wide_range_field(W: np.ndarray, n_side: int = 1024, seed: int = 2) -> Field:
    """1,048,576 cells, T ~ U[800, 2600] K, p ~ U[0.5, 5] atm, dt = 1e-5 s."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = n_side * n_side
    T, p, Y = random_state(n, rng, W, 800.0, 2600.0, 0.5, 5.0)
    return _finish("wide_range_field", T, p, Y, W, 1e-5, (n_side, n_side))


def training_states(W: np.ndarray, n: int, seed: int = 3, coupled: float = 0.0, T_lo: float = 800.0,
                    T_hi: float = 2600.0, dt_lo: float = 1e-7, dt_hi: float = 1e-5) -> Field:
    """Training states: the wide-range distribution with dt ~ log-U[dt_lo,
    dt_hi] (default [1e-7, 1e-5] s; radicals shared in a fraction `coupled`
    of the states); [T_lo, T_hi] is [800, 2600] K for the wide-range
    distribution itself and [305, 800] K for a flame's preheat zone."""
    rng = np.random.Generator(np.random.PCG64(seed))
    T, p, Y = random_state(n, rng, W, T_lo, T_hi, 0.5, 5.0, coupled)
    dts = 10.0 ** rng.uniform(np.log10(dt_lo), np.log10(dt_hi), n)
    return _finish("training_states", T, p, Y, W, float("nan"), (n,), dts)


def flame_field(W: np.ndarray, n_side: int = 2048, seed: int = 4) -> Field:
    """Premixed-flame-like field: 2048 x 2048 cells of 10 um, tanh front
    (delta = 0.5 mm) from 300 K to 2400 K along x, front position perturbed in
    y by 8 seeded sinusoids of amplitude 0.2 mm, radicals Gaussian at the front
    with peak mass fraction 1e-3, p = 1 atm, dt = 1e-6 s."""
    T, c, g = _flame_geometry(n_side, seed)
    Yr, Yp, idx = _stoich(W)
    Y = (1.0 - c)[None, :] * Yr[:, None] + c[None, :] * Yp[:, None]
    for sp in RADICALS:
        Y[idx[sp]] = 1e-3 * g
    n = n_side * n_side
    return _finish("flame_field", T, np.full(n, P_ATM), Y, W, 1e-6, (n_side, n_side))


def _flame_geometry(n_side: int, seed: int):
    """Flat (T, progress c, front Gaussian g) of the flame geometry."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dx = 10e-6
    delta = 0.5e-3
    L = n_side * dx
    x = (np.arange(n_side) + 0.5) * dx
    y = (np.arange(n_side) + 0.5) * dx
    modes = rng.integers(1, 17, 8)
    phases = rng.uniform(0.0, 2.0 * np.pi, 8)
    xf = 0.5 * L + np.sum(0.2e-3 * np.sin(2.0 * np.pi * modes[:, None] * y[None, :] / L + phases[:, None]), axis=0)
    # cell (i, j) with i along x fastest: flat index j * n_side + i
    s = (x[None, :] - xf[:, None]) / delta
    c = 0.5 * (1.0 + np.tanh(s))
    T = 300.0 + 2100.0 * c
    return T.reshape(-1), c.reshape(-1), np.exp(-0.5 * (s.reshape(-1)) ** 2)


ACETYLENE_RADICALS = ["H", "O", "OH", "HO2", "HCO", "CH3", "HCCO"]


def _acetylene_mix(names, W):
    """Stoichiometric C2H2/O2 in 70 % argon (mole) and its complete products."""
    idx = {s: i for i, s in enumerate(names)}
    Xr, Xp = np.zeros(len(names)), np.zeros(len(names))
    Xr[idx["C2H2"]], Xr[idx["O2"]], Xr[idx["AR"]] = 2.0, 5.0, 16.33
    Xp[idx["CO2"]], Xp[idx["H2O"]], Xp[idx["AR"]] = 4.0, 2.0, 16.33
    return Xr * W / np.sum(Xr * W), Xp * W / np.sum(Xp * W), idx


def acetylene_state(names, W: np.ndarray, n: int, seed: int = 0, T_lo: float = 1000.0, T_hi: float = 2600.0,
                    dt: float = 1e-6) -> Field:
    """Random cells of the C2H2/O2/Ar mechanism: T ~ U[T_lo, T_hi], p = 1
    atm, progress c ~ U[0, 1] between the stoichiometric mixture and its
    products, radicals log-uniform on [1e-8, 1e-4]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Yr, Yp, idx = _acetylene_mix(names, W)
    T = rng.uniform(T_lo, T_hi, n)
    c = rng.uniform(0.0, 1.0, n)
    Y = (1.0 - c)[None, :] * Yr[:, None] + c[None, :] * Yp[:, None]
    for sp in ACETYLENE_RADICALS:
        Y[idx[sp]] = 10.0 ** rng.uniform(-8.0, -4.0, n)
    return _finish("acetylene", T, np.full(n, P_ATM), Y, W, dt, (n,))


def acetylene_flame(names, W: np.ndarray, n_side: int = 2048, seed: int = 4) -> Field:
    """The flame flame geometry with the C2H2/O2/Ar mixture: same
    temperature field, reactants to products along the front, radicals
    Gaussian at the front with peak mass fraction 1e-4."""
    T, c, g = _flame_geometry(n_side, seed)
    Yr, Yp, idx = _acetylene_mix(names, W)
    Y = (1.0 - c)[None, :] * Yr[:, None] + c[None, :] * Yp[:, None]
    for sp in ACETYLENE_RADICALS:
        Y[idx[sp]] = 1e-4 * g
    n = n_side * n_side
    return _finish("acetylene_flame", T, np.full(n, P_ATM), Y, W, 1e-6, (n_side, n_side))


def slice_field(f: Field, n: int, stride: int = 1, offset: int = 0) -> Field:
    sel = np.arange(offset, offset + n * stride, stride) % f.n
    return Field(f.name + f"[{n}]", f.T[sel].copy(), f.rho[sel].copy(), f.p[sel].copy(),
                 np.ascontiguousarray(f.Y[:, sel]), f.dt, (n,),
                 None if f.dt_cells is None else f.dt_cells[sel].copy())


def state_for_species(f: Field, names, W: np.ndarray) -> Field:
    """The same cells for a mechanism with other species: H2, O2, N2, H2O
    and the five radicals keep their mass fractions, species the field does
    not carry (excited or other states) start at zero; rho is recomputed from
    p, T and the new mixture molar mass."""
    idx = {s: i for i, s in enumerate(SPECIES)}
    Y = np.zeros((len(names), f.n))
    for k, nm in enumerate(names):
        if nm in idx:
            Y[k] = f.Y[idx[nm]]
    return _finish(f.name, f.T.copy(), f.p.copy(), Y, W, f.dt, f.shape, f.dt_cells)


@dataclass
class PredictorBlock:
    """Cell and face fields of one block of the low-Mach solver, flat with the
    ghost layer (layout of nrg_grid_desc / nrg_species_predictor_device)."""
    dims: int
    n_cells: tuple
    dx: float
    dt: float
    coord: int
    rho: np.ndarray          # (ld,)
    Y: np.ndarray            # (N, ld)
    v_f: list                # dims face fields, each (dims * f0 * f1 * f2,)
    x_center: np.ndarray     # (e0,)
    bc: np.ndarray           # (ld,) int8
    Y_prod_diff: np.ndarray  # (N, ld)
    Y_prod_chem: np.ndarray  # (N, ld)

    @property
    def ld(self) -> int:
        return self.rho.shape[0]


def predictor_block(W: np.ndarray, dims: int, n_cells, seed: int = 0, coord: int = 0, dx: float = 10e-6,
                    dt: float = 1e-7, bc_fraction: float = 0.02, zero_face_fraction: float = 0.05) -> PredictorBlock:
    """A flame front along x (as the flame field: tanh profile from 300 K
    to 2400 K, radicals Gaussian at the front) on a block with its ghost
    layer, plus seeded face velocities of both signs (some exactly zero),
    diffusion and chemistry sources of the size the step produces, and a few
    cells with bc /= 0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = list(n_cells) + [1] * (3 - len(n_cells))
    e = [n[d] + 2 if d < dims else 1 for d in range(3)]
    f = [e[d] + 1 if d < dims else 1 for d in range(3)]
    ld = e[0] * e[1] * e[2]
    i = np.arange(ld) % e[0]
    j = (np.arange(ld) // e[0]) % e[1]
    k = np.arange(ld) // (e[0] * e[1])
    x = (i - 0.5) * dx
    xf = 0.5 * n[0] * dx + 0.15 * n[0] * dx * np.sin(2.0 * np.pi * (j + 0.5 * k) / max(e[1], 4))
    s = (x - xf) / (0.1 * n[0] * dx)
    c = 0.5 * (1.0 + np.tanh(s))
    T = 300.0 + 2100.0 * c
    Yr, Yp, idx = _stoich(W)
    Y = (1.0 - c)[None, :] * Yr[:, None] + c[None, :] * Yp[:, None]
    g = np.exp(-0.5 * s ** 2)
    for sp in RADICALS:
        Y[idx[sp]] = 1e-3 * g * rng.uniform(0.5, 1.5, ld)
    fl = _finish("predictor", T, np.full(ld, P_ATM), Y, W, dt, (ld,))
    v_f = []
    for d in range(dims):
        v = rng.uniform(-6.0, 10.0, dims * f[0] * f[1] * f[2])
        v[rng.uniform(0.0, 1.0, v.shape[0]) < zero_face_fraction] = 0.0
        v_f.append(v)
    x_center = (np.arange(e[0]) - 0.5) * dx + (20.0 * dx if coord else 0.0)
    bc = (rng.uniform(0.0, 1.0, ld) < bc_fraction).astype(np.int8)
    N = W.shape[0]
    Y_prod_diff = rng.normal(0.0, 50.0, (N, ld))
    Y_prod_chem = rng.normal(0.0, 200.0, (N, ld)) * g[None, :]
    return PredictorBlock(dims, tuple(n[:dims]), dx, dt, coord, fl.rho, np.ascontiguousarray(fl.Y), v_f, x_center,
                          bc, Y_prod_diff, Y_prod_chem)

"""ctypes front-end to the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product path never imports
this module.  Parity status of the oracle: unpinned (no Fortran compiler, no
reference golden vectors); see oracle/oracle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

NMAX = 64
RMAX = 512


class OrcMech(ctypes.Structure):
    _fields_ = [
        ("n_species", ctypes.c_int),
        ("n_reactions", ctypes.c_int),
        ("species_names", (ctypes.c_char * 21) * (NMAX + 1)),
        ("reaction_type", ctypes.c_int * RMAX),
        ("coeffs", ((ctypes.c_int * 4) * RMAX) * 2),
        ("A", ctypes.c_double * RMAX),
        ("beta", ctypes.c_double * RMAX),
        ("E_act", ctypes.c_double * RMAX),
        ("A_low", ctypes.c_double * RMAX),
        ("beta_low", ctypes.c_double * RMAX),
        ("E_act_low", ctypes.c_double * RMAX),
        ("troe", (ctypes.c_double * 4) * RMAX),
        ("eff", (ctypes.c_double * NMAX) * RMAX),
        ("a_coeffs", ((ctypes.c_double * 7) * 2) * NMAX),
        ("molar_mass", ctypes.c_double * NMAX),
    ]


class OrcTransport(ctypes.Structure):
    _fields_ = [
        ("n_species", ctypes.c_int),
        ("well_depth", ctypes.c_double * NMAX),
        ("collision_diameter", ctypes.c_double * NMAX),
        ("bdc", (ctypes.c_double * NMAX) * NMAX),
    ]


class OrcCounters(ctypes.Structure):
    _fields_ = [("nstate", ctypes.c_int), ("nstep", ctypes.c_int),
                ("nfe", ctypes.c_int), ("nje", ctypes.c_int)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_load_mechanism.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_double, ctypes.c_char_p,
                                                                 ctypes.POINTER(OrcMech)]
        L.orc_load_mechanism.restype = ctypes.c_int
        L.orc_chem_step_mx.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_long, ctypes.c_double,
                                       dp, dp, dp, ctypes.c_void_p, dp, dp, dp,
                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_chem_step_mx.restype = ctypes.c_int
        L.orc_temperature_after.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_long, ctypes.c_double,
                                            dp, dp, dp, dp, dp, dp, ctypes.c_int]
        L.orc_apply_state.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_long, ctypes.c_int, ctypes.c_double,
                                      dp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, dp, dp,
                                      ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_void_p,
                                      ctypes.c_int]
        L.orc_apply_state.restype = ctypes.c_int
        L.orc_species_predictor.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.c_long, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_void_p * 3] + [ctypes.c_void_p] * 4 + [
                                            ctypes.c_int, ctypes.c_void_p] + [dp] * 6
        L.orc_species_predictor.restype = ctypes.c_int
        L.orc_load_transport.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_char_p, ctypes.POINTER(OrcTransport)]
        L.orc_load_transport.restype = ctypes.c_int
        L.orc_omega.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_omega.restype = ctypes.c_double
        L.orc_binary_diffusion.argtypes = [ctypes.POINTER(OrcMech), ctypes.POINTER(OrcTransport), ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_binary_diffusion.restype = ctypes.c_double
        L.orc_mixture_diffusivity.argtypes = [ctypes.POINTER(OrcMech), ctypes.POINTER(OrcTransport), ctypes.c_long,
                                              dp, dp, dp, dp, ctypes.c_void_p, dp, ctypes.c_int]
        L.orc_mixture_diffusivity.restype = None
        L.orc_rate_constants.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_double, dp, dp, dp]
        L.orc_rate_constants.restype = None
        L.orc_rhs.argtypes = [ctypes.POINTER(OrcMech), dp, dp, dp, dp, dp]
        L.orc_rhs.restype = None
        for f in ("orc_specie_enthalpy", "orc_specie_entropy", "orc_specie_cp"):
            getattr(L, f).argtypes = [ctypes.POINTER(OrcMech), ctypes.c_double, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_double
        L.orc_dnrm2.argtypes = [ctypes.c_int, dp, ctypes.c_int]
        L.orc_dnrm2.restype = ctypes.c_double
        L.orc_ddcst.argtypes = [ctypes.c_int, dp, dp]
        L.orc_ddcst.restype = None
        L.orc_format_e14_7.argtypes = [ctypes.c_double, ctypes.c_char_p]
        L.orc_format_e14_7.restype = None
        L.orc_parse_e14_7.argtypes = [ctypes.c_char_p, ctypes.c_int, dp]
        L.orc_parse_e14_7.restype = ctypes.c_int
        L.orc_table_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_long, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        L.orc_table_read.restype = ctypes.c_int
        L.orc_table_write.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p] + [ctypes.c_int] * 4 + [dp, dp]
        L.orc_table_write.restype = ctypes.c_int
        L.orc_table_step.argtypes = [ctypes.POINTER(OrcMech), ctypes.c_long, dp, dp, ctypes.c_long, ctypes.c_double,
                                     dp, dp, ctypes.c_void_p, dp, dp, dp, ctypes.c_int]
        L.orc_table_step.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Mechanism:
    """Parsed mechanism held by the oracle."""

    def __init__(self, mech_path, thermo_path, molar_path, eff_default=1.0, eact_units="cal.mol"):
        self.m = OrcMech()
        rc = lib().orc_load_mechanism(mech_path.encode(), thermo_path.encode(), molar_path.encode(),
                                      float(eff_default), eact_units.encode(), ctypes.byref(self.m))
        if rc != 0:
            raise RuntimeError(f"oracle mechanism load failed: {rc}")

    @property
    def n_species(self):
        return self.m.n_species

    @property
    def n_reactions(self):
        return self.m.n_reactions

    def species(self):
        return [self.m.species_names[i].value.decode() for i in range(self.m.n_species + 1)]

    def tables(self) -> dict:
        """Constant tables as numpy arrays (reference layouts)."""
        N, R = self.m.n_species, self.m.n_reactions
        m = self.m
        coeffs = np.array([[list(m.coeffs[s][r]) for r in range(R)] for s in range(2)], dtype=np.int32)
        return dict(
            species=self.species(),
            reaction_type=np.array(m.reaction_type[:R], dtype=np.int32),
            coeffs=coeffs,
            A=np.array(m.A[:R]), beta=np.array(m.beta[:R]), E_act=np.array(m.E_act[:R]),
            A_low=np.array(m.A_low[:R]), beta_low=np.array(m.beta_low[:R]),
            E_act_low=np.array(m.E_act_low[:R]),
            troe=np.array([list(m.troe[r]) for r in range(R)]),
            eff=np.array([list(m.eff[r])[:N] for r in range(R)]),
            a_coeffs=np.array([[list(m.a_coeffs[k][s]) for s in range(2)] for k in range(N)]),
            molar_mass=np.array(m.molar_mass[:N]),
        )

    def chem_step(self, dt, T, rho, Y, bc=None, threads=0, mxstep=10000, Y_prod2_init=None):
        """Y is (N, n) SoA.  Returns dict of outputs and per-cell counters."""
        n = T.shape[0]
        N = self.m.n_species
        T = np.ascontiguousarray(T, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64).reshape(N, n)
        Yp = np.zeros((N, n))
        Yp2 = np.zeros((N, n)) if Y_prod2_init is None else np.array(Y_prod2_init, dtype=np.float64)
        Ef = np.zeros(n)
        cnt = (OrcCounters * n)()
        bcp = None
        if bc is not None:
            bc = np.ascontiguousarray(bc, dtype=np.int8)
            bcp = bc.ctypes.data_as(ctypes.c_void_p)
        lib().orc_chem_step_mx(ctypes.byref(self.m), n, float(dt), _dp(T), _dp(rho), _dp(Y), bcp,
                               _dp(Yp), _dp(Yp2), _dp(Ef), ctypes.cast(cnt, ctypes.c_void_p),
                               int(threads), int(mxstep))
        c = np.frombuffer(cnt, dtype=np.int32).reshape(n, 4)
        return dict(Y_prod=Yp, Y_prod2=Yp2, E_f_prod=Ef, nstate=c[:, 0].copy(), nstep=c[:, 1].copy(),
                    nfe=c[:, 2].copy(), nje=c[:, 3].copy())

    def table_step(self, T_t, Y_t, dt, T, Y, bc=None, Y_prod2_init=None, threads=0):
        """table_approximated mode (orc_table_step): T_t (M,), Y_t (N, M)."""
        n = T.shape[0]
        N = self.m.n_species
        T_t = np.ascontiguousarray(T_t, dtype=np.float64)
        Y_t = np.ascontiguousarray(Y_t, dtype=np.float64).reshape(N, T_t.shape[0])
        T = np.ascontiguousarray(T, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64).reshape(N, n)
        Yp = np.zeros((N, n))
        Yp2 = np.zeros((N, n)) if Y_prod2_init is None else np.array(Y_prod2_init, dtype=np.float64)
        Ef = np.zeros(n)
        bcp = None
        if bc is not None:
            bc = np.ascontiguousarray(bc, dtype=np.int8)
            bcp = bc.ctypes.data_as(ctypes.c_void_p)
        rc = lib().orc_table_step(ctypes.byref(self.m), T_t.shape[0], _dp(T_t), _dp(Y_t), n, float(dt), _dp(T),
                                  _dp(Y), bcp, _dp(Yp), _dp(Yp2), _dp(Ef), int(threads))
        if rc != 0:
            raise RuntimeError(f"orc_table_step: {rc}")
        return dict(Y_prod=Yp, Y_prod2=Yp2, E_f_prod=Ef)

    def table_write(self, path, lb, ub, lo, hi, T_row, Y_prod2_row):
        """write_chemical_kinetics_table on one row (orc_table_write):
        T_row (ub-lb+1,), Y_prod2_row (N, ub-lb+1), Fortran indices."""
        N = self.m.n_species
        T_row = np.ascontiguousarray(T_row, dtype=np.float64)
        Y2 = np.ascontiguousarray(Y_prod2_row, dtype=np.float64).reshape(N, T_row.shape[0])
        rc = lib().orc_table_write(str(path).encode(), N, ctypes.cast(self.m.species_names, ctypes.c_void_p),
                                   lb, ub, lo, hi, _dp(T_row), _dp(Y2))
        if rc != 0:
            raise RuntimeError(f"orc_table_write: {rc}")

    def table_read(self, path):
        """read_chemical_kinetics_table (orc_table_read): (T_t, Y_t (N, M))."""
        return table_read(path, self.m.n_species)

    def temperature_after(self, dt, T, rho, Y, Y_prod, E_f_prod, threads=0):
        n = T.shape[0]
        out = np.zeros(n)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (T, rho, Y, Y_prod, E_f_prod)]
        lib().orc_temperature_after(ctypes.byref(self.m), n, float(dt), *[_dp(a) for a in args],
                                    _dp(out), int(threads))
        return out

    def apply_state(self, rho, Y, E_f, T, v=None, dt=0.0, Y_prod=None, E_f_prod=None, bc=None, threads=0):
        """Chemistry sources applied to (Y, E_f), then the state equation
        (orc_apply_state).  Y is (N, n) SoA, v (dims, n) or None.  Returns the
        updated Y, E_f, T and p, gamma, cp, h_s, h_full, v_s, mix_mol_mass,
        status."""
        n = rho.shape[0]
        N = self.m.n_species
        Y = np.array(Y, dtype=np.float64).reshape(N, n)
        E_f = np.array(E_f, dtype=np.float64)
        T = np.array(T, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        dims = 0 if v is None else int(np.asarray(v).shape[0])
        vv = np.zeros((1, n)) if v is None else np.ascontiguousarray(v, dtype=np.float64)
        out = {k: np.zeros(n) for k in ("p", "gamma", "cp", "h_s", "h_full", "v_s", "mix_mol_mass")}
        st = np.zeros(n, np.uint8)
        yp = None if Y_prod is None else np.ascontiguousarray(Y_prod, dtype=np.float64)
        ep = None if E_f_prod is None else np.ascontiguousarray(E_f_prod, dtype=np.float64)
        bcv = None if bc is None else np.ascontiguousarray(bc, dtype=np.int8)
        vp = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        lib().orc_apply_state(ctypes.byref(self.m), n, dims, float(dt), _dp(rho), vp(yp), vp(ep), vp(bcv),
                              _dp(Y), _dp(E_f), vv.ctypes.data_as(ctypes.c_void_p), _dp(T), _dp(out["p"]),
                              _dp(out["gamma"]), _dp(out["cp"]), _dp(out["h_s"]), _dp(out["h_full"]),
                              _dp(out["v_s"]), _dp(out["mix_mol_mass"]), st.ctypes.data_as(ctypes.c_void_p),
                              int(threads))
        out.update(Y=Y, E_f=E_f, T=T, status=st)
        return out

    def load_transport(self, transport_path) -> None:
        """Transport deck for this mechanism's species (orc_load_transport)."""
        self.tr = OrcTransport()
        rc = lib().orc_load_transport(ctypes.byref(self.m), transport_path.encode(), ctypes.byref(self.tr))
        if rc != 0:
            raise RuntimeError(f"oracle transport load failed: {rc}")

    def transport_tables(self) -> dict:
        N = self.m.n_species
        return {"well_depth": np.array(self.tr.well_depth[:N]),
                "collision_diameter": np.array(self.tr.collision_diameter[:N]),
                "binary_diffusivity_constant": np.array([[self.tr.bdc[i][j] for j in range(N)] for i in range(N)])}

    def binary_diffusion(self, T, p, i, j) -> float:
        return lib().orc_binary_diffusion(ctypes.byref(self.m), ctypes.byref(self.tr), float(T), float(p), i, j)

    def mixture_diffusivity(self, T, p, Y, m_mix, bc=None) -> np.ndarray:
        """calculate_diffusivity_coeff over n cells: (N, n) mixture-averaged
        diffusion coefficients (zero where bc /= 0)."""
        n = T.shape[0]
        N = self.m.n_species
        T, p, m_mix = (np.ascontiguousarray(a, dtype=np.float64) for a in (T, p, m_mix))
        Y = np.ascontiguousarray(Y, dtype=np.float64).reshape(N, n)
        D = np.zeros((N, n))
        bcv = None if bc is None else np.ascontiguousarray(bc, dtype=np.int8)
        lib().orc_mixture_diffusivity(ctypes.byref(self.m), ctypes.byref(self.tr), n, _dp(T), _dp(p), _dp(Y),
                                      _dp(m_mix), None if bcv is None else bcv.ctypes.data_as(ctypes.c_void_p),
                                      _dp(D), 0)
        return D

    def rate_constants(self, T, mix_conc):
        R = self.m.n_reactions
        mc = np.ascontiguousarray(mix_conc, dtype=np.float64)
        kf = np.zeros(R)
        kr = np.zeros(R)
        lib().orc_rate_constants(ctypes.byref(self.m), float(T), _dp(mc), _dp(kf), _dp(kr))
        return kf, kr

    def rhs(self, kf, kr, mix_conc, Z):
        out = np.zeros(self.m.n_species)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (kf, kr, mix_conc, Z)]
        lib().orc_rhs(ctypes.byref(self.m), *[_dp(x) for x in a], _dp(out))
        return out

    def enthalpy(self, T, k):
        return lib().orc_specie_enthalpy(ctypes.byref(self.m), float(T), int(k))

    def entropy(self, T, k):
        return lib().orc_specie_entropy(ctypes.byref(self.m), float(T), int(k))

    def cp(self, T, k):
        return lib().orc_specie_cp(ctypes.byref(self.m), float(T), int(k))


def dnrm2(x) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().orc_dnrm2(x.shape[0], _dp(x), 1)


def ddcst(maxord=5):
    el = np.zeros(13 * 12)
    tq = np.zeros(3 * 12)
    lib().orc_ddcst(maxord, _dp(el), _dp(tq))
    return el.reshape(12, 13).T, tq.reshape(12, 3).T


def species_predictor(W, dims, n_cells, coord, dx, dt, v_f, rho, Y, rho_int, Y_int, x_center=None, bc=None,
                      Y_prod_diff=None, Y_prod_chem=None, Y_prod_part=(), rho_old=None, Y_old=None):
    """The low-Mach species predictor (orc_species_predictor) on copies of
    the cell fields.  Cell fields are flat (ld,) or (N, ld) arrays in the
    layout of orc_transport.c; v_f is a list of `dims` face fields.  Returns
    dict(rho, Y, rho_old, Y_old, rho_int, Y_int)."""
    W = np.ascontiguousarray(W, dtype=np.float64)
    N = W.shape[0]
    ld = rho.shape[0]
    c = lambda a: np.array(a, dtype=np.float64, copy=True)
    out = dict(rho=c(rho), Y=c(Y).reshape(N, ld), rho_int=c(rho_int), Y_int=c(Y_int).reshape(N, ld),
               rho_old=np.zeros(ld) if rho_old is None else c(rho_old),
               Y_old=np.zeros((N, ld)) if Y_old is None else c(Y_old).reshape(N, ld))
    keep = []

    def vp(a, dtype=np.float64):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a.ctypes.data_as(ctypes.c_void_p)

    vf = (ctypes.c_void_p * 3)(*([vp(v) for v in v_f] + [None] * (3 - len(v_f))))
    parts = (ctypes.c_void_p * max(1, len(Y_prod_part)))(*[vp(a) for a in Y_prod_part])
    nc = (ctypes.c_int * 3)(*(list(n_cells) + [1] * (3 - len(n_cells))))
    rc = lib().orc_species_predictor(N, _dp(W), int(dims), nc, ld, int(coord), float(dx), float(dt), vf,
                                     vp(x_center), vp(bc, np.int8), vp(Y_prod_diff), vp(Y_prod_chem),
                                     len(Y_prod_part), ctypes.cast(parts, ctypes.c_void_p),
                                     _dp(out["rho"]), _dp(out["Y"]), _dp(out["rho_old"]), _dp(out["Y_old"]),
                                     _dp(out["rho_int"]), _dp(out["Y_int"]))
    if rc != 0:
        raise ValueError(f"orc_species_predictor: bad arguments ({rc})")
    return out


def format_e14_7(x: float) -> str:
    """Fortran E14.7 output of one value."""
    buf = ctypes.create_string_buffer(15)
    lib().orc_format_e14_7(float(x), buf)
    return buf.value.decode()


def parse_e14_7(field: str) -> float:
    """Fortran E14.7 input of one field."""
    v = ctypes.c_double()
    raw = field.encode()
    if lib().orc_parse_e14_7(raw, len(raw), ctypes.byref(v)) != 0:
        raise ValueError(f"malformed E14.7 field {field!r}")
    return v.value


def table_read(path, n_species: int):
    """read_chemical_kinetics_table (orc_table_read): (T_t, Y_t (N, M))."""
    rows = ctypes.c_long()
    rc = lib().orc_table_read(str(path).encode(), n_species, 0, None, None, ctypes.byref(rows))
    if rc != 0:
        raise RuntimeError(f"orc_table_read: {rc}")
    M = rows.value
    T_t = np.zeros(M)
    Y_t = np.zeros((n_species, M))
    rc = lib().orc_table_read(str(path).encode(), n_species, M, T_t.ctypes.data, Y_t.ctypes.data,
                              ctypes.byref(rows))
    if rc != 0:
        raise RuntimeError(f"orc_table_read: {rc}")
    return T_t, Y_t

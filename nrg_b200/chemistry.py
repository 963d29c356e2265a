"""Host-side mirror of NRG's chemistry operator over the libnrg_chem C ABI.

Reference interface (computing_module/src/current_build/
chemical_kinetics_solver.f90):

    type(chemical_kinetics_solver) function chemical_kinetics_solver_c(manager)   ! :111-173
    subroutine solve_chemical_kinetics(this, time_step)                           ! :175-358

The constructor finds 'temperature', 'pressure', 'density' and
'specie_mass_fraction' in the data manager and creates
'energy_production_chemistry', 'specie_production_chemistry' and
'specie_production_chemistry2' (:121-138).  This module keeps those names and
that behaviour; the arithmetic runs in libnrg_chem.so on the GPU.  There is no
CPU fallback: a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnrg_chem.so")
NRG_MAX_SPECIES = 24

MODES = {"reference": 0, "fast": 1, "mixed": 2, "surrogate": 3, "table": 4}
EACT_UNITS = {"J.mol": 0, "kJ.mol": 1, "cal.mol": 2, "kcal.mol": 3}
CELL_STATUS = {0: "skipped", 1: "ok", 2: "mxstep", 3: "fatal", 4: "nonfinite", 5: "surrogate"}


class NrgError(RuntimeError):
    pass


class FieldDesc(ctypes.Structure):
    _fields_ = [
        ("lb", ctypes.c_int * 3), ("ub", ctypes.c_int * 3),
        ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3),
        ("T", ctypes.c_void_p), ("p", ctypes.c_void_p), ("rho", ctypes.c_void_p),
        ("Y", ctypes.c_void_p * NRG_MAX_SPECIES),
        ("Y_prod", ctypes.c_void_p * NRG_MAX_SPECIES),
        ("Y_prod2", ctypes.c_void_p * NRG_MAX_SPECIES),
        ("E_f_prod", ctypes.c_void_p),
        ("bc_markers", ctypes.c_void_p),
    ]


class GridDesc(ctypes.Structure):
    """nrg_grid_desc: a block of the low-Mach solver's cell fields."""
    _fields_ = [("dims", ctypes.c_int), ("n", ctypes.c_int * 3), ("ld", ctypes.c_longlong),
                ("coord", ctypes.c_int), ("dx", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("cells", ctypes.c_longlong), ("cells_active", ctypes.c_longlong),
        ("cells_bad", ctypes.c_longlong), ("cells_surrogate", ctypes.c_longlong),
        ("cells_fallback", ctypes.c_longlong),
        ("steps", ctypes.c_longlong), ("rhs_evals", ctypes.c_longlong),
        ("jacobians", ctypes.c_longlong), ("solves", ctypes.c_longlong),
        ("device_ms", ctypes.c_double),
        ("phase_ms", ctypes.c_double * 4),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["phase_ms"] = list(self.phase_ms)
        return d


# every symbol include/nrg_chem.h declares, with its ctypes signature
_VP, _I, _D, _L, _CP = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long, ctypes.c_char_p
SIGNATURES = {
    "nrg_chem_create": (_I, [_CP, _CP, _CP, _D, _I, ctypes.POINTER(_VP)]),
    "nrg_chem_destroy": (_I, [_VP]),
    "nrg_chem_step": (_I, [_VP, _D, ctypes.POINTER(FieldDesc), ctypes.POINTER(Stats)]),
    "nrg_chem_step_device": (_I, [_VP, _D, _L, _L, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                  ctypes.POINTER(Stats)]),
    "nrg_chem_step_device_noalloc": (_I, [_VP, _D, _L, _L, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                          ctypes.POINTER(Stats)]),
    "nrg_chem_set_mode": (_I, [_VP, _I]),
    "nrg_chem_set_launch": (_I, [_VP, _I, _I, _I, _I]),
    "nrg_chem_get_launch": (_I, [_VP] + [ctypes.POINTER(_I)] * 4),
    "nrg_chem_autotune": (_I, [_VP, _D, _L, _L, _VP, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.POINTER(_D)]),
    "nrg_chem_set_graph": (_I, [_VP, _I]),
    "nrg_chem_set_cell_order": (_I, [_VP, _I]),
    "nrg_chem_set_timing": (_I, [_VP, _I]),
    "nrg_chem_set_eps": (_I, [_VP, _D]),
    "nrg_surrogate_set_fallback_eps": (_I, [_VP, _D]),
    "nrg_chem_set_lu_form": (_I, [_VP, _I]),
    "nrg_chem_get_lu_form": (_I, [_VP, ctypes.POINTER(_I)]),
    "nrg_surrogate_set_dt_band": (_I, [_VP, _D, _D]),
    "nrg_surrogate_set_gate_band": (_I, [_VP, _I, _D, _D, _D, _D, _D]),
    "nrg_chem_info": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "nrg_chem_tables": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nrg_chem_species_name": (_I, [_VP, _I, ctypes.c_char_p, _I]),
    "nrg_mech_tables": (_I, [_CP, _CP, _CP, _D, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)] + [_VP] * 7),
    "nrg_chem_last_error": (ctypes.c_char_p, [_VP]),
    "nrg_surrogate_param_count": (_I, []),
    "nrg_surrogate_norm_count": (_I, []),
    "nrg_surrogate_select": (_I, [_VP, _I]),
    "nrg_surrogate_init": (_I, [_VP, ctypes.c_ulonglong]),
    "nrg_surrogate_get_params": (_I, [_VP, _VP]),
    "nrg_surrogate_set_params": (_I, [_VP, _VP]),
    "nrg_surrogate_get_norm": (_I, [_VP, _VP]),
    "nrg_surrogate_set_norm": (_I, [_VP, _VP]),
    "nrg_surrogate_prepare": (_I, [_VP, _L, _L, _D, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nrg_surrogate_features": (_I, [_VP, _L, _L, _D, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nrg_surrogate_forward": (_I, [_VP, _L, _VP, _VP]),
    "nrg_surrogate_grad": (_I, [_VP, _L, _VP, _VP, _VP, ctypes.POINTER(_D)]),
    "nrg_surrogate_train": (_I, [_VP, _L, _VP, _VP, _I, _I, ctypes.c_float, ctypes.c_ulonglong, _VP]),
    "nrg_surrogate_set_gate": (_I, [_VP, _D, _D, _D, _D]),
    "nrg_surrogate_set_gate_dt": (_I, [_VP, _D]),
    "nrg_surrogate_set_partner": (_I, [_VP, _I, _D, _D]),
    "nrg_surrogate_set_band": (_I, [_VP, _D, _D]),
    "nrg_chem_set_specialised": (_I, [_VP, _I]),
    "nrg_chem_apply_state_device": (_I, [_VP, _D, _L, _L, _I] + [_VP] * 17),
    "nrg_surrogate_set_inference": (_I, [_VP, _I]),
    "nrg_surrogate_infer": (_I, [_VP, _L, _L, _D, _VP, _VP, _VP, _VP, _VP]),
    "nrg_surrogate_enable": (_I, [_VP, _I]),
    "nrg_surrogate_save": (_I, [_VP, _CP]),
    "nrg_surrogate_load": (_I, [_VP, _CP]),
    "nrg_chem_integrate": (_I, [_VP, _L, _L, _D, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                ctypes.POINTER(Stats)]),
    "nrg_fp64_peak_tflops": (_I, [ctypes.POINTER(_D)]),
    "nrg_table_read": (_I, [_CP, _I, _L, _VP, _VP, ctypes.POINTER(_L)]),
    "nrg_table_write": (_I, [_CP, _I, _VP, ctypes.POINTER(FieldDesc)]),
    "nrg_chem_set_table": (_I, [_VP, _L, _VP, _VP]),
    "nrg_chem_load_table": (_I, [_VP, _CP]),
    "nrg_selftest_bounded_wait": (_I, [ctypes.c_longlong, ctypes.POINTER(_I), ctypes.POINTER(_D)]),
    "nrg_chem_load_transport": (_I, [_VP, _CP]),
    "nrg_mech_transport_tables": (_I, [_CP] * 4 + [_VP] * 3),
    "nrg_mixture_diffusivity_device": (_I, [_VP, _L, _L] + [_VP] * 7),
    "nrg_species_predictor_device": (_I, [_VP, _D, ctypes.POINTER(GridDesc), _VP, _VP, _VP, _VP, _VP, _I, _VP]
                                     + [_VP] * 7),
}

_lib = None


def lib():
    """Loads libnrg_chem.so; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NrgError(f"{LIB_PATH} not built: run __graft_entry__.build() or python nrg_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a) -> int | None:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _check(rc: int, h=None) -> None:
    if rc != 0:
        msg = lib().nrg_chem_last_error(h)
        raise NrgError(f"libnrg_chem error {rc}: {msg.decode() if msg else ''}")


def mechanism_tables(mechanism, thermo, molar_masses, default_enhanced_efficiencies=1.0,
                     E_act_units="cal.mol") -> dict:
    """Parsed constant tables (host only, no GPU)."""
    L = lib()
    n, r = ctypes.c_int(), ctypes.c_int()
    args = [str(mechanism).encode(), str(thermo).encode(), str(molar_masses).encode(),
            float(default_enhanced_efficiencies), EACT_UNITS[E_act_units]]
    _check(L.nrg_mech_tables(*args, ctypes.byref(n), ctypes.byref(r), *([None] * 7)))
    N, R = n.value, r.value
    t = dict(reaction_type=np.zeros(R, np.int32), coeffs=np.zeros((2, R, 4), np.int32),
             arrhenius=np.zeros((R, 9)), troe3=np.zeros(R), eff=np.zeros((R, N)),
             a_coeffs=np.zeros((N, 2, 7)), molar_mass=np.zeros(N))
    _check(L.nrg_mech_tables(*args, ctypes.byref(n), ctypes.byref(r),
                             *[_ptr(t[k]) for k in ("reaction_type", "coeffs", "arrhenius", "troe3",
                                                    "eff", "a_coeffs", "molar_mass")]))
    t["n_species"], t["n_reactions"] = N, R
    return t


def transport_tables(mechanism, thermo, molar_masses, transport) -> dict:
    """Transport deck of the mechanism's species as the library reads it
    (host only, no GPU): well depths, collision diameters [nm], binary
    diffusivity constants."""
    N = mechanism_tables(mechanism, thermo, molar_masses)["n_species"]
    eps, sg, bdc = np.zeros(N), np.zeros(N), np.zeros((N, N))
    _check(lib().nrg_mech_transport_tables(str(mechanism).encode(), str(thermo).encode(),
                                           str(molar_masses).encode(), str(transport).encode(),
                                           _ptr(eps), _ptr(sg), _ptr(bdc)))
    return {"well_depth": eps, "collision_diameter": sg, "binary_diffusivity_constant": bdc}


@dataclass
class DataManager:
    """Named Fortran-layout fields of one block: cells(lb:ub) per axis, ghost
    layer included, column-major (data_manager_class.f90:55-68)."""

    lb: tuple
    ub: tuple
    lo: tuple
    hi: tuple
    fields: dict = field(default_factory=dict)

    @classmethod
    def block(cls, nx: int, ny: int, nz: int = 1, ghost: int = 1) -> "DataManager":
        lb = (1 - ghost, 1 - ghost, 1 - ghost if nz > 1 else 1)
        ub = (nx + ghost, ny + ghost, nz + ghost if nz > 1 else 1)
        return cls(lb, ub, (1, 1, 1), (nx, ny, nz))

    @property
    def shape(self):
        return tuple(u - l + 1 for l, u in zip(self.lb, self.ub))

    def create_scalar_field(self, name: str) -> np.ndarray:
        self.fields[name] = np.zeros(self.shape, order="F")
        return self.fields[name]

    def create_vector_field(self, name: str, n: int) -> list:
        self.fields[name] = [np.zeros(self.shape, order="F") for _ in range(n)]
        return self.fields[name]

    def get_field_pointer_by_name(self, name: str):
        return self.fields[name]

    def interior(self, a: np.ndarray) -> np.ndarray:
        sl = tuple(slice(lo - l, hi - l + 1) for lo, hi, l in zip(self.lo, self.hi, self.lb))
        return a[sl]


class ChemicalKineticsSolver:
    """GPU chemistry operator with the reference's constructor and step."""

    def __init__(self, manager: DataManager | None, mechanism, thermo, molar_masses,
                 default_enhanced_efficiencies: float = 1.0, E_act_units: str = "cal.mol",
                 mode: str = "fast"):
        L = lib()
        h = ctypes.c_void_p()
        _check(L.nrg_chem_create(str(mechanism).encode(), str(thermo).encode(), str(molar_masses).encode(),
                                 float(default_enhanced_efficiencies), EACT_UNITS[E_act_units],
                                 ctypes.byref(h)))
        self._h = h
        n, r = ctypes.c_int(), ctypes.c_int()
        _check(L.nrg_chem_info(h, ctypes.byref(n), ctypes.byref(r)), h)
        self.species_number, self.reactions_number = n.value, r.value
        buf = ctypes.create_string_buffer(32)
        self.species_names = []
        for k in range(self.species_number):
            _check(L.nrg_chem_species_name(h, k, buf, 32), h)
            self.species_names.append(buf.value.decode())
        self.set_mode(mode)
        self.manager = manager
        if manager is not None:
            for name in ("temperature", "density", "specie_mass_fraction"):
                if name not in manager.fields:
                    raise NrgError(f"field '{name}' not registered in the data manager")
            manager.create_scalar_field("energy_production_chemistry")
            manager.create_vector_field("specie_production_chemistry", self.species_number)
            manager.create_vector_field("specie_production_chemistry2", self.species_number)

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().nrg_chem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- options -----------------------------------------------------------
    def set_mode(self, mode: str) -> None:
        _check(lib().nrg_chem_set_mode(self._h, MODES[mode]), self._h)
        self.mode = mode

    KERNELS = {"thread": 0, "thread_queue": 1, "warp_queue": 2}

    def set_launch(self, kernel="warp_queue", block=256, grid=0, chunk=1, lu_rolled=None) -> None:
        """kernel: 'thread' (one thread per cell), 'thread_queue' (thread per
        cell with a work queue) or 'warp_queue' (warp per cell, work queue);
        lu_rolled: the thread kernels' LU as a loop (None: unchanged)."""
        k = self.KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        _check(lib().nrg_chem_set_launch(self._h, k, block, grid, chunk), self._h)
        if lu_rolled is not None:
            _check(lib().nrg_chem_set_lu_form(self._h, int(bool(lu_rolled))), self._h)

    def get_launch(self) -> dict:
        v = [ctypes.c_int() for _ in range(4)]
        _check(lib().nrg_chem_get_launch(self._h, *[ctypes.byref(x) for x in v]), self._h)
        d = dict(zip(("kernel", "block", "grid", "chunk"), [x.value for x in v]))
        d["kernel"] = {v: k for k, v in self.KERNELS.items()}[d["kernel"]]
        r = ctypes.c_int()
        _check(lib().nrg_chem_get_lu_form(self._h, ctypes.byref(r)), self._h)
        d["lu_rolled"] = bool(r.value)
        return d

    def set_graph(self, enable: bool) -> None:
        _check(lib().nrg_chem_set_graph(self._h, int(enable)), self._h)

    def set_cell_order(self, by_temperature: bool) -> None:
        """Integrator takes the cells grouped by temperature (default) or in
        cell order; the results are the same."""
        _check(lib().nrg_chem_set_cell_order(self._h, int(by_temperature)), self._h)

    def apply_state_device(self, rho, Y, E_f, T, p, gamma, v=None, time_step=0.0, Y_prod=None, E_f_prod=None,
                           bc=None, cp_mass=None, h_s=None, h_full=None, v_s=None, mix_mol_mass=None,
                           status=None) -> None:
        """Chemistry sources into (Y, E_f) and the state equation, on torch
        CUDA tensors (Y species-major (N, n); v (dims, n) or None)."""
        import torch
        n = T.numel()
        dims = 0 if v is None else int(v.shape[0])
        _check(lib().nrg_chem_apply_state_device(
            self._h, float(time_step), n, Y.shape[1], dims, _ptr(rho), _ptr(Y_prod), _ptr(E_f_prod), _ptr(bc),
            _ptr(Y), _ptr(E_f), _ptr(v), _ptr(T), _ptr(p), _ptr(gamma), _ptr(cp_mass), _ptr(h_s), _ptr(h_full),
            _ptr(v_s), _ptr(mix_mol_mass), _ptr(status),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), self._h)

    def species_predictor_device(self, time_step, dims, n_cells, dx, v_f, rho, Y, rho_old, Y_old, rho_int, Y_int,
                                 coord=0, x_center=None, bc=None, Y_prod_diff=None, Y_prod_chem=None,
                                 Y_prod_particles=()) -> None:
        """calculate_interm_Y_predictor on torch CUDA tensors: cell fields
        flat over the block with its ghost layer (Y-like fields (N, ld)), v_f a
        list of `dims` face fields in the reference's layout
        (nrg_species_predictor_device)."""
        import torch
        g = GridDesc(int(dims), (ctypes.c_int * 3)(*(list(n_cells) + [1] * (3 - len(n_cells)))), rho.numel(),
                     int(coord), float(dx))
        vf = (ctypes.c_void_p * 3)(*([_ptr(v) for v in v_f] + [None] * (3 - len(v_f))))
        parts = (ctypes.c_void_p * max(1, len(Y_prod_particles)))(*[_ptr(a) for a in Y_prod_particles])
        _check(lib().nrg_species_predictor_device(
            self._h, float(time_step), ctypes.byref(g), ctypes.cast(vf, ctypes.c_void_p), _ptr(x_center), _ptr(bc),
            _ptr(Y_prod_diff), _ptr(Y_prod_chem), len(Y_prod_particles), ctypes.cast(parts, ctypes.c_void_p),
            _ptr(rho), _ptr(Y), _ptr(rho_old), _ptr(Y_old), _ptr(rho_int), _ptr(Y_int),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), self._h)

    def load_transport(self, transport_path: str) -> None:
        """Transport deck of the mechanism's species (nrg_chem_load_transport)."""
        _check(lib().nrg_chem_load_transport(self._h, transport_path.encode()), self._h)

    def mixture_diffusivity_device(self, T, p, Y, mix_mol_mass, D, bc=None) -> None:
        """calculate_diffusivity_coeff on torch CUDA tensors (Y, D: (N, n))."""
        import torch
        _check(lib().nrg_mixture_diffusivity_device(
            self._h, T.numel(), Y.shape[1], _ptr(T), _ptr(p), _ptr(Y), _ptr(mix_mol_mass), _ptr(bc), _ptr(D),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), self._h)

    def set_specialised(self, enable: bool) -> None:
        """Generated mechanism-specialised RHS / iteration matrix (default when
        the mechanism matches) or the table-driven loops."""
        _check(lib().nrg_chem_set_specialised(self._h, int(enable)), self._h)

    def set_eps(self, eps: float = 0.0) -> None:
        """Integrator tolerance EPS (0: the reference's 1e-9)."""
        _check(lib().nrg_chem_set_eps(self._h, float(eps)), self._h)

    def set_fallback_eps(self, eps: float = 0.0) -> None:
        """Integrator tolerance of the surrogate's rejected cells (0: the
        handle's EPS)."""
        _check(lib().nrg_surrogate_set_fallback_eps(self._h, float(eps)), self._h)

    def set_timing(self, enable: bool) -> None:
        _check(lib().nrg_chem_set_timing(self._h, int(enable)), self._h)

    @property
    def handle(self):
        return self._h

    # -- the reference step on host fields -------------------------------------
    def solve_chemical_kinetics(self, time_step: float) -> dict:
        m = self.manager
        if m is None:
            raise NrgError("no data manager attached")
        d, keep = field_desc(m, self.species_number)
        st = Stats()
        _check(lib().nrg_chem_step(self._h, float(time_step), ctypes.byref(d), ctypes.byref(st)), self._h)
        del keep
        return st.as_dict()

    # -- table_approximated mode --------------------------------------------
    def set_table(self, T_t, Y_t) -> None:
        """Table of the table mode: T_t (rows,), Y_t (N, rows)."""
        T_t = np.ascontiguousarray(T_t, dtype=np.float64)
        Y_t = np.ascontiguousarray(Y_t, dtype=np.float64).reshape(self.species_number, T_t.shape[0])
        _check(lib().nrg_chem_set_table(self._h, T_t.shape[0], _ptr(T_t), _ptr(Y_t)), self._h)

    def read_chemical_kinetics_table(self, table_file) -> None:
        """read_chemical_kinetics_table (chemical_kinetics_solver.f90:608-650)."""
        _check(lib().nrg_chem_load_table(self._h, str(table_file).encode()), self._h)

    def write_chemical_kinetics_table(self, table_file) -> None:
        """write_chemical_kinetics_table (chemical_kinetics_solver.f90:542-607)
        from the attached data manager's temperature and Y_prod2 fields."""
        if self.manager is None:
            raise NrgError("no data manager attached")
        write_table(table_file, self.species_names, self.manager)

    # -- device-resident step (torch CUDA tensors) ---------------------------
    def step_device(self, time_step, T, rho, Y, Y_prod, Y_prod2, E_f_prod, bc=None, T_after=None,
                    status=None, stream=None) -> dict:
        """Species-major device arrays: Y has shape (N, ld) with cells in the
        first n = T.numel() columns."""
        n = T.numel()
        ld = Y.shape[1]
        if stream is None and hasattr(T, "device"):
            import torch
            stream = torch.cuda.current_stream(T.device).cuda_stream
        st = Stats()
        _check(lib().nrg_chem_step_device(
            self._h, float(time_step), n, ld, _ptr(T), _ptr(rho), _ptr(Y), _ptr(bc), _ptr(Y_prod),
            _ptr(Y_prod2), _ptr(E_f_prod), _ptr(T_after), _ptr(status),
            ctypes.c_void_p(stream) if stream else None, ctypes.byref(st)), self._h)
        return st.as_dict()

    def integrate(self, dt, T, rho, Y, Y_prod, Y_prod2, E_f_prod, dt_cells=None, bc=None, T_after=None,
                  status=None) -> dict:
        """FP64 integration (never the surrogate) with an optional per-cell dt."""
        import torch
        st = Stats()
        stream = torch.cuda.current_stream(T.device).cuda_stream
        _check(lib().nrg_chem_integrate(
            self._h, T.numel(), Y.shape[1], float(dt), _ptr(dt_cells), _ptr(T), _ptr(rho), _ptr(Y), _ptr(bc),
            _ptr(Y_prod), _ptr(Y_prod2), _ptr(E_f_prod), _ptr(T_after), _ptr(status),
            ctypes.c_void_p(stream) if stream else None, ctypes.byref(st)), self._h)
        return st.as_dict()

    def step_device_noalloc(self, time_step, T, rho, Y, Y_prod, Y_prod2, E_f_prod, bc=None, T_after=None,
                            status=None, stream=None) -> dict:
        """step_device for callers that cannot allocate device memory during a
        step: the library uses a fixed scratch array of its own (at most
        1,048,576 cells per call) and allocates nothing."""
        n = T.numel()
        ld = Y.shape[1]
        if stream is None and hasattr(T, "device"):
            import torch
            stream = torch.cuda.current_stream(T.device).cuda_stream
        st = Stats()
        _check(lib().nrg_chem_step_device_noalloc(
            self._h, float(time_step), n, ld, _ptr(T), _ptr(rho), _ptr(Y), _ptr(bc), _ptr(Y_prod),
            _ptr(Y_prod2), _ptr(E_f_prod), _ptr(T_after), _ptr(status),
            ctypes.c_void_p(stream) if stream else None, ctypes.byref(st)), self._h)
        return st.as_dict()

    def autotune(self, time_step, T, rho, Y, Y_prod, Y_prod2, E_f_prod, bc=None) -> float:
        ms = ctypes.c_double()
        _check(lib().nrg_chem_autotune(self._h, float(time_step), T.numel(), Y.shape[1], _ptr(T), _ptr(rho),
                                       _ptr(Y), _ptr(bc), _ptr(Y_prod), _ptr(Y_prod2), _ptr(E_f_prod),
                                       ctypes.byref(ms)), self._h)
        return ms.value


def chemical_kinetics_solver_c(manager: DataManager, mechanism, thermo, molar_masses, ODE_solver: str = "slatec",
                               table_file=None, **kw) -> ChemicalKineticsSolver:
    """Constructor with the reference's name (chemical_kinetics_solver.f90:105-107,
    111-173).  ODE_solver 'table_approximated' reads table_file and steps in
    table mode (:168-170); 'slatec' (the reference's default) integrates."""
    if ODE_solver not in ("slatec", "table_approximated"):
        raise NrgError(f"unknown ODE_solver {ODE_solver!r}")
    if ODE_solver == "table_approximated":
        if table_file is None:
            raise NrgError("table_approximated needs a table_file")
        s = ChemicalKineticsSolver(manager, mechanism, thermo, molar_masses, **dict(kw, mode="fast"))
        try:
            s.read_chemical_kinetics_table(table_file)
            s.set_mode("table")
        except Exception:
            s.close()
            raise
        return s
    return ChemicalKineticsSolver(manager, mechanism, thermo, molar_masses, **kw)


def field_desc(m: DataManager, N: int):
    """nrg_field_desc of a data manager's fields (and the arrays it points
    into, which the caller keeps alive while the descriptor is used)."""
    d = FieldDesc()
    for i in range(3):
        d.lb[i], d.ub[i], d.lo[i], d.hi[i] = m.lb[i], m.ub[i], m.lo[i], m.hi[i]
    keep = []

    def fptr(a):
        if not (a.flags.f_contiguous and a.dtype == np.float64):
            raise NrgError("fields must be float64 Fortran-ordered arrays")
        keep.append(a)
        return a.ctypes.data

    f = m.fields
    d.T = fptr(f["temperature"])
    if "density" in f:
        d.rho = fptr(f["density"])
    d.p = fptr(f["pressure"]) if "pressure" in f else None
    for k in range(N):
        if "specie_mass_fraction" in f:
            d.Y[k] = fptr(f["specie_mass_fraction"][k])
        if "specie_production_chemistry" in f:
            d.Y_prod[k] = fptr(f["specie_production_chemistry"][k])
        d.Y_prod2[k] = fptr(f["specie_production_chemistry2"][k])
    if "energy_production_chemistry" in f:
        d.E_f_prod = fptr(f["energy_production_chemistry"])
    if "bc_markers" in f:
        bc = f["bc_markers"]
        if bc.dtype != np.int8 or not bc.flags.f_contiguous:
            raise NrgError("bc_markers must be int8 Fortran-ordered")
        keep.append(bc)
        d.bc_markers = bc.ctypes.data
    return d, keep


def table_read(path, n_species: int):
    """A chemistry table file as the library reads it (host only, no GPU):
    (T_t (rows,), Y_t (N, rows))."""
    rows = ctypes.c_long()
    _check(lib().nrg_table_read(str(path).encode(), n_species, 0, None, None, ctypes.byref(rows)))
    M = rows.value
    T_t, Y_t = np.zeros(M), np.zeros((n_species, M))
    _check(lib().nrg_table_read(str(path).encode(), n_species, M, _ptr(T_t), _ptr(Y_t), ctypes.byref(rows)))
    return T_t, Y_t


def write_table(path, species_names, m: DataManager) -> None:
    """write_chemical_kinetics_table on a data manager's 'temperature' and
    'specie_production_chemistry2' fields (host only, no GPU)."""
    N = len(species_names)
    d, keep = field_desc(m, N)
    names = (ctypes.c_char_p * N)(*[n.encode() for n in species_names])
    _check(lib().nrg_table_write(str(path).encode(), N, ctypes.cast(names, ctypes.c_void_p), ctypes.byref(d)))
    del keep


def fp64_peak_tflops() -> float:
    v = ctypes.c_double()
    _check(lib().nrg_fp64_peak_tflops(ctypes.byref(v)))
    return v.value

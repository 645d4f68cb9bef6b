"""ctypes binding of libclb.so (include/clb.h), the C-ABI of the B200 reactive-transport step.

This module is what a Python caller (and this repository's tests and benchmark) uses; a C++
host links the same library directly. There is no fallback: if libclb.so is missing or no CUDA
device is present, every call fails with an exception naming the cause.

Arrays follow the library's layout: x slowest, z fastest, index (x*ny + y)*nz + z; population
arrays are [q][N] in Palabos' velocity order, shifted by the weights.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclb.so")

F64, F32, F16S = 0, 1, 2
DIRICHLET, NEUMANN, CLOSED = 0, 1, 2
LAW_NONE, LAW_DECAY, LAW_MONOD, LAW_DUAL_MONOD = 0, 1, 2, 3
LAW_PRECIP, LAW_MINERAL = 4, 5  # abiotic laws
DISSOL_NONE, DISSOL_FIRST_ORDER, DISSOL_MINERAL = 0, 1, 2
FIELD_MATERIAL, FIELD_FLOW_VELOCITY, FIELD_FLOW_POPULATIONS = 0, 1, 2
FIELD_CONCENTRATION, FIELD_ADE_POPULATIONS, FIELD_BIOMASS, FIELD_ADE_VELOCITY = 3, 4, 5, 6
FIELD_CA_TOTAL, FIELD_CA_AGE = 7, 8
CKPT_FLOW, CKPT_TRANSPORT = 1, 2

STATUS = {0: "OK", 1: "INVALID_ARG", 2: "NOT_CONVERGED", 3: "NONFINITE", 4: "PERCOLATION_LOST",
          5: "CUDA_ERROR", 6: "TIMEOUT", 7: "NOT_INITIALIZED", 8: "OUT_OF_MEMORY"}

MAX_MICROBES, MAX_PORE_CODES, MAX_SPECIES = 8, 8, 16
MAX_EQ_SPECIES, MAX_COMPONENTS = 16, 8
SPEC_OFF, SPEC_NR, SPEC_MLP, SPEC_MLP_NR = 0, 1, 2, 3


class DomainDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("flow_precision", C.c_int32), ("ade_precision", C.c_int32),
                ("solid_code", C.c_int32), ("bounce_back_code", C.c_int32),
                ("n_pore_codes", C.c_int32), ("pore_codes", C.c_int32 * MAX_PORE_CODES),
                ("n_microbes", C.c_int32), ("bio_codes", C.c_int32 * MAX_MICROBES),
                ("perm_ratio", C.c_double * MAX_MICROBES), ("tau", C.c_double)]


class SpeciesDesc(C.Structure):
    _fields_ = [("omega_pore", C.c_double), ("omega_biofilm", C.c_double), ("mobile", C.c_int32),
                ("left_type", C.c_int32), ("right_type", C.c_int32),
                ("left_bc", C.c_double), ("right_bc", C.c_double), ("c0", C.c_double)]


class FlowStats(C.Structure):
    _fields_ = [("pore_mean_u", C.c_double), ("pore_max_ux", C.c_double), ("darcy_outlet_ux", C.c_double),
                ("permeability", C.c_double), ("energy", C.c_double), ("iterations", C.c_int64),
                ("bgk_nodes", C.c_int64), ("active_nodes", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [("total", C.c_double * MAX_SPECIES), ("content", C.c_double * MAX_SPECIES),
                ("biomass", C.c_double * MAX_MICROBES), ("min_c", C.c_double * MAX_SPECIES),
                ("max_c", C.c_double * MAX_SPECIES), ("open_voxels", C.c_int64),
                ("nonfinite", C.c_int64), ("ade_iterations", C.c_int64)]


class GeomOptions(C.Structure):
    _fields_ = [("kind", C.c_char_p), ("porosity", C.c_double), ("radius", C.c_double),
                ("aperture", C.c_double), ("roughness", C.c_double), ("count", C.c_int32),
                ("layers", C.c_int32), ("seed", C.c_uint64), ("walls", C.c_char_p)]


class Inspection(C.Structure):
    _fields_ = [("porosity", C.c_double), ("open_voxels", C.c_int64), ("isolated_voxels", C.c_int64),
                ("clusters", C.c_int32), ("spanning_clusters", C.c_int32), ("percolates", C.c_int32),
                ("quasi_2d", C.c_int32)]


class SpeciationDesc(C.Structure):
    _fields_ = [("n_species", C.c_int32), ("n_components", C.c_int32),
                ("stoich", (C.c_double * MAX_COMPONENTS) * MAX_EQ_SPECIES), ("logK", C.c_double * MAX_EQ_SPECIES),
                ("component_species", C.c_int32 * MAX_COMPONENTS), ("tolerance", C.c_double),
                ("max_iterations", C.c_int32)]


class ThermoDesc(C.Structure):
    _fields_ = [("n_terms", C.c_int32), ("species", C.c_int32 * MAX_SPECIES), ("nu", C.c_double * MAX_SPECIES),
                ("dG0", C.c_double), ("atp", C.c_double), ("dGatp", C.c_double), ("chi", C.c_double),
                ("cmin", C.c_double), ("dGloss", C.c_double), ("temperature", C.c_double),
                ("gas_constant", C.c_double), ("conc_scale", C.c_double)]


class SurrogateDesc(C.Structure):
    _fields_ = [("half_saturation", C.c_double * MAX_SPECIES), ("max_uptake_flux", C.c_double * MAX_SPECIES),
                ("biomass_molar_mass", C.c_double), ("decay", C.c_double)]


class PrecipDesc(C.Structure):
    _fields_ = [("mineral_species", C.c_int32), ("full_density", C.c_double), ("precip_code", C.c_int32),
                ("seal_flow", C.c_int32), ("seal_perm_ratio", C.c_double), ("flow_max_iterations", C.c_int32),
                ("flow_eps", C.c_double), ("dissolution", C.c_int32), ("reopen_fraction", C.c_double),
                ("pore_code", C.c_int32), ("dissolution_law", C.c_int32),
                ("dissolution_params", C.c_double * (MAX_SPECIES + 2)), ("dissolution_surface_only", C.c_int32)]


class CaDesc(C.Structure):
    _fields_ = [("max_biomass", C.c_double), ("biofilm_fraction", C.c_double), ("seed", C.c_uint64),
                ("push_mode", C.c_int32)]


class RunDesc(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("ca", C.c_int32), ("ade_update_interval", C.c_int32),
                ("ns_update_interval", C.c_int32), ("resolve_every", C.c_int32), ("geometry_interval", C.c_int32),
                ("flow_max_iterations", C.c_int32), ("flow_eps", C.c_double)]


class RunReport(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("ca_sweeps", C.c_int64), ("mask_changes", C.c_int64),
                ("flow_resolves", C.c_int64), ("flow_iterations", C.c_int64), ("flow_unconverged", C.c_int64),
                ("sealed", C.c_int64), ("reopened", C.c_int64), ("ms_transport", C.c_double), ("ms_ca", C.c_double),
                ("ms_flow", C.c_double), ("ms_geometry", C.c_double), ("seconds", C.c_double),
                ("launches", C.c_int64)]


class SpeciationStats(C.Structure):
    _fields_ = [("solves", C.c_int64), ("converged", C.c_int64), ("surrogate_used", C.c_int64),
                ("fallbacks", C.c_int64), ("iterations", C.c_int64)]


class SurrogateTrainDesc(C.Structure):
    _fields_ = [("n_samples", C.c_int32), ("epochs", C.c_int32), ("batch", C.c_int32), ("patience", C.c_int32),
                ("learning_rate", C.c_double), ("val_fraction", C.c_double), ("seed", C.c_uint64),
                ("log_c_lo", C.c_double * MAX_EQ_SPECIES), ("log_c_hi", C.c_double * MAX_EQ_SPECIES),
                ("source", C.c_int32), ("jitter", C.c_double)]


class SurrogateReport(C.Structure):
    _fields_ = [("train_mse", C.c_double), ("val_mse", C.c_double), ("seconds", C.c_double),
                ("epochs", C.c_int32), ("steps", C.c_int32), ("n_train", C.c_int32), ("n_val", C.c_int32)]


# every symbol include/clb.h declares, with its argument types
SIGNATURES = {
    "clb_set_device": [C.c_int],
    "clb_create": [C.POINTER(DomainDesc), C.c_void_p, C.POINTER(C.c_void_p)],
    "clb_destroy": [C.c_void_p],
    "clb_last_error": [C.c_void_p],
    "clb_global_error": [],
    "clb_synchronize": [C.c_void_p],
    "clb_set_stream": [C.c_void_p, C.c_void_p],
    "clb_tune": [C.c_void_p, C.c_char_p, C.c_int],
    "clb_autotune": [C.c_void_p, C.c_int, C.c_char_p, C.c_int],
    "clb_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "clb_flow_init": [C.c_void_p, C.c_double],
    "clb_flow_step": [C.c_void_p, C.c_int],
    "clb_flow_solve": [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int)],
    "clb_flow_stats_get": [C.c_void_p, C.c_double, C.POINTER(FlowStats)],
    "clb_flow_solve_peclet": [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                              C.POINTER(C.c_double), C.POINTER(C.c_int)],
    "clb_ade_init": [C.c_void_p, C.POINTER(SpeciesDesc), C.c_int],
    "clb_couple_velocity": [C.c_void_p],
    "clb_set_kinetics": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double],
    "clb_set_biomass": [C.c_void_p, C.c_int, C.c_void_p],
    "clb_set_thermo_gate": [C.c_void_p, C.POINTER(ThermoDesc)],
    "clb_set_symbolic_kinetics": [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int, C.c_char_p],
    "clb_symbolic_eval": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)],
    "clb_set_graph_network": [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int],
    "clb_set_surrogate_organism": [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int, C.c_void_p],
    "clb_surrogate_eval": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int),
                           C.POINTER(C.c_long)],
    "clb_graph_network_eval": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int),
                               C.POINTER(C.c_long)],
    "clb_write_vti": [C.c_void_p, C.c_int, C.c_int, C.c_char_p],
    "clb_checkpoint_save": [C.c_void_p, C.c_char_p, C.c_int],
    "clb_checkpoint_load": [C.c_void_p, C.c_char_p],
    "clb_vti_write": [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p],
    "clb_ade_step": [C.c_void_p, C.c_int],
    "clb_reduce": [C.c_void_p, C.POINTER(Stats)],
    "clb_reduce_noalloc": [C.c_void_p, C.POINTER(Stats)],
    "clb_set_abiotic_kinetics": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int],
    "clb_ca_setup": [C.c_void_p, C.POINTER(CaDesc)],
    "clb_run": [C.c_void_p, C.POINTER(RunDesc), C.POINTER(RunReport)],
    "clb_batch_create": [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)],
    "clb_batch_step": [C.c_void_p, C.c_int, C.c_int, C.c_int],
    "clb_batch_autotune": [C.c_void_p, C.c_int, C.c_char_p, C.c_int],
    "clb_batch_counts": [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "clb_batch_destroy": [C.c_void_p],
    "clb_batch_schedule": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
    "clb_batch_get_schedule": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "clb_batch_set_stream": [C.c_void_p, C.c_void_p],
    "clb_batch_set_wait_limit": [C.c_void_p, C.c_int64],
    "clb_ca_step": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "clb_refresh_dynamics": [C.c_void_p, C.c_int, C.c_int],
    "clb_precip_setup": [C.c_void_p, C.POINTER(PrecipDesc)],
    "clb_geometry_update": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "clb_speciation_setup": [C.c_void_p, C.POINTER(SpeciationDesc)],
    "clb_set_speciation_mode": [C.c_void_p, C.c_int],
    "clb_speciation_stats_get": [C.c_void_p, C.POINTER(SpeciationStats)],
    "clb_speciation_solve": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "clb_surrogate_train": [C.c_void_p, C.POINTER(SurrogateTrainDesc), C.POINTER(SurrogateReport)],
    "clb_surrogate_set_check": [C.c_void_p, C.c_double, C.c_int, C.c_double],
    "clb_surrogate_predict": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int],
    "clb_surrogate_params": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "clb_surrogate_param_count": [],
    "clb_surrogate_gradient": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "clb_get_field": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int],
    "clb_set_field": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int],
    "clb_case_load": [C.c_char_p, C.POINTER(C.c_void_p)],
    "clb_case_free": [C.c_void_p],
    "clb_case_error": [],
    "clb_case_get": [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)],
    "clb_case_setup": [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "clb_case_run": [C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.POINTER(RunReport)],
    "clb_geom_generate": [C.POINTER(GeomOptions), C.c_int, C.c_int, C.c_int, C.c_void_p],
    "clb_geom_sphere_pack": [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64,
                             C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "clb_geom_read_dat": [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "clb_geom_inspect": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(Inspection)],
}

_lib = None


def lib():
    """Load libclb.so once; raise if it is missing (no silent fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libclb.so not built at {LIB_PATH}; run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_char_p if name in ("clb_last_error", "clb_global_error", "clb_case_error") else C.c_int
        _lib = L
    return _lib


class ClbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check_global(st):
    if st != 0:
        raise ClbError(st, lib().clb_global_error().decode())


# ------------------------------------------------------------------------------ geometry
def geom_generate(kind, nx, ny, nz, porosity=0.4, radius=6.0, aperture=6.0, roughness=2.0, count=20,
                  layers=4, seed=1, walls="y"):
    out = np.empty(nx * ny * nz, dtype=np.int8)
    o = GeomOptions(kind.encode(), porosity, radius, aperture, roughness, count, layers, seed, walls.encode())
    _check_global(lib().clb_geom_generate(C.byref(o), nx, ny, nz, _ptr(out)))
    return out


def sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed, walls="yz", grain=1, wall=1, pore=2):
    out = np.empty(nx * ny * nz, dtype=np.int8)
    _check_global(lib().clb_geom_sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed, walls.encode(),
                                             grain, wall, pore, _ptr(out)))
    return out


def read_dat(path, nx_inner, ny, nz):
    out = np.empty((nx_inner + 2) * ny * nz, dtype=np.int8)
    _check_global(lib().clb_geom_read_dat(path.encode(), nx_inner, ny, nz, _ptr(out)))
    return out


def inspect(mat, nx, ny, nz):
    r = Inspection()
    m = np.ascontiguousarray(mat, dtype=np.int8)
    _check_global(lib().clb_geom_inspect(_ptr(m), nx, ny, nz, C.byref(r)))
    return {k: getattr(r, k) for k, _ in Inspection._fields_}


# ------------------------------------------------------------------------------ domain
class Domain:
    """One handle of the library (a domain with its flow and species lattices)."""

    def __init__(self, material, nx, ny, nz, tau, flow_precision=F32, ade_precision=F32,
                 solid_code=0, bounce_back_code=1, pore_codes=(2,), bio_codes=(), perm_ratio=(), device=None):
        L = lib()
        if device is not None:
            _check_global(L.clb_set_device(int(device)))
        d = DomainDesc()
        d.nx, d.ny, d.nz = nx, ny, nz
        d.flow_precision, d.ade_precision = flow_precision, ade_precision
        d.solid_code, d.bounce_back_code = solid_code, bounce_back_code
        d.n_pore_codes = len(pore_codes)
        for k, c in enumerate(pore_codes):
            d.pore_codes[k] = c
        d.n_microbes = len(bio_codes)
        for k, c in enumerate(bio_codes):
            d.bio_codes[k] = c
            d.perm_ratio[k] = perm_ratio[k] if k < len(perm_ratio) else 1.0
        d.tau = tau
        self.desc = d
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.S = 0
        m = np.ascontiguousarray(material, dtype=np.int8)
        assert m.size == self.N
        h = C.c_void_p()
        _check_global(L.clb_create(C.byref(d), _ptr(m), C.byref(h)))
        self.h = h

    def _check(self, st):
        if st != 0:
            raise ClbError(st, lib().clb_last_error(self.h).decode())
        return st

    def close(self):
        if self.h:
            lib().clb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tune(self, key, value):
        self._check(lib().clb_tune(self.h, key.encode(), int(value)))

    def autotune(self, steps=20):
        buf = C.create_string_buffer(512)
        self._check(lib().clb_autotune(self.h, steps, buf, 512))
        return buf.value.decode()

    def set_stream(self, stream_ptr):
        self._check(lib().clb_set_stream(self.h, C.c_void_p(stream_ptr)))

    def stream(self):
        p = C.c_void_p()
        self._check(lib().clb_get_stream(self.h, C.byref(p)))
        return p.value

    def sync(self):
        self._check(lib().clb_synchronize(self.h))

    # ---- flow
    def flow_init(self, delta_p):
        self._check(lib().clb_flow_init(self.h, delta_p))

    def flow_step(self, n=1):
        self._check(lib().clb_flow_step(self.h, n))

    def flow_solve(self, max_it, eps, allow_unconverged=False):
        it = C.c_int(0)
        st = lib().clb_flow_solve(self.h, max_it, eps, C.byref(it))
        if not (st == 0 or (allow_unconverged and st == 2)):
            self._check(st)
        return it.value, st == 0

    def flow_solve_peclet(self, peclet, char_length, tau_ade_fixed, max_it, eps):
        dp = C.c_double(0)
        it = C.c_int(0)
        st = lib().clb_flow_solve_peclet(self.h, peclet, char_length, tau_ade_fixed, max_it, eps,
                                         C.byref(dp), C.byref(it))
        if st not in (0, 2):
            self._check(st)
        return dp.value, it.value, st == 0

    def flow_stats(self, char_length=1.0):
        s = FlowStats()
        self._check(lib().clb_flow_stats_get(self.h, char_length, C.byref(s)))
        return {k: getattr(s, k) for k, _ in FlowStats._fields_}

    def velocity(self, dtype=np.float64, out=None):
        """Flow velocity [3][N]; dtype float64 or float32 (the copy to the host is then half as large).
        `out`: a contiguous array of 3 N elements of that dtype to fill (for example in pinned memory)."""
        dt = np.dtype(dtype)
        if dt not in (np.dtype(np.float64), np.dtype(np.float32)):
            raise ValueError("velocity dtype is float64 or float32")
        if out is None:
            u = np.empty(3 * self.N, dtype=dt)
        else:
            if out.dtype != dt or out.size != 3 * self.N or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous array of 3 N elements of the requested dtype")
            u = out.reshape(-1)
        self._check(lib().clb_get_field(self.h, FIELD_FLOW_VELOCITY, 0, _ptr(u), 0 if dt == np.float64 else 1))
        return u.reshape(3, self.N)

    def flow_populations(self):
        f = np.empty(19 * self.N, dtype=np.float64)
        self._check(lib().clb_get_field(self.h, FIELD_FLOW_POPULATIONS, 0, _ptr(f), 0))
        return f.reshape(19, self.N)

    def set_flow_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._check(lib().clb_set_field(self.h, FIELD_FLOW_POPULATIONS, 0, _ptr(f), 0))

    # ---- transport
    def ade_init(self, species):
        arr = (SpeciesDesc * len(species))()
        for k, s in enumerate(species):
            arr[k] = SpeciesDesc(s["omega_pore"], s.get("omega_biofilm", s["omega_pore"]), s.get("mobile", 1),
                                 s.get("left_type", NEUMANN), s.get("right_type", NEUMANN),
                                 s.get("left_bc", 0.0), s.get("right_bc", 0.0), s.get("c0", 0.0))
        self.S = len(species)
        self._check(lib().clb_ade_init(self.h, arr, len(species)))

    def couple_velocity(self):
        self._check(lib().clb_couple_velocity(self.h))

    def set_velocity(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._check(lib().clb_set_field(self.h, FIELD_ADE_VELOCITY, 0, _ptr(u), 0))

    def set_kinetics(self, law, params, dt):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._check(lib().clb_set_kinetics(self.h, law, _ptr(p), p.size, dt))

    def set_abiotic_kinetics(self, law, params, surface_only=0):
        p = np.ascontiguousarray(params if len(params) else [0.0], dtype=np.float64)
        self._check(lib().clb_set_abiotic_kinetics(self.h, law, _ptr(p), len(params), int(surface_only)))

    def precip_setup(self, mineral, full_density, precip_code=-1, seal_flow=0, seal_perm_ratio=0.0,
                     flow_max_iterations=100000, flow_eps=1e-6, dissolution=0, reopen_fraction=0.9, pore_code=-1,
                     dissolution_law=DISSOL_NONE, dissolution_params=(), dissolution_surface_only=1):
        d = PrecipDesc()
        d.mineral_species, d.full_density, d.precip_code = int(mineral), float(full_density), int(precip_code)
        d.seal_flow, d.seal_perm_ratio = int(seal_flow), float(seal_perm_ratio)
        d.flow_max_iterations, d.flow_eps = int(flow_max_iterations), float(flow_eps)
        d.dissolution, d.reopen_fraction, d.pore_code = int(dissolution), float(reopen_fraction), int(pore_code)
        d.dissolution_law, d.dissolution_surface_only = int(dissolution_law), int(dissolution_surface_only)
        for i, v in enumerate(dissolution_params):
            d.dissolution_params[i] = float(v)
        self._check(lib().clb_precip_setup(self.h, C.byref(d)))

    def geometry_update(self, allow_unconverged=False):
        """Seal / reopen voxels; returns (sealed, reopened)."""
        a, b = C.c_int(), C.c_int()
        st = lib().clb_geometry_update(self.h, C.byref(a), C.byref(b))
        if not (allow_unconverged and st == 2):
            self._check(st)
        return a.value, b.value

    def ca_setup(self, max_biomass, biofilm_fraction, seed, half=False):
        """half: the 'half' push (halfPushExcessBiomass3D) instead of 'fraction'."""
        d = CaDesc(float(max_biomass), float(biofilm_fraction), int(seed), 1 if half else 0)
        self._check(lib().clb_ca_setup(self.h, C.byref(d)))

    def ca_step(self, allow_stall=False):
        """One iteration's biofilm automaton; returns (status, sweeps, mask_changed)."""
        a, b = C.c_int(), C.c_int()
        st = lib().clb_ca_step(self.h, C.byref(a), C.byref(b))
        if not (allow_stall and st == 2):
            self._check(st)
        return st, a.value, bool(b.value)

    def run(self, iterations, ca=False, ade_update_interval=1, ns_update_interval=0, resolve_every=0,
            geometry_interval=0, flow_max_iterations=100000, flow_eps=1e-6, allow_stop=False):
        """clb_run: `iterations` coupled iterations in the reference's loop order; returns the
        report as a dict (its "status" is the call's status when allow_stop lets a stop through)."""
        d = RunDesc(int(iterations), int(bool(ca)), int(ade_update_interval), int(ns_update_interval),
                    int(resolve_every), int(geometry_interval), int(flow_max_iterations), float(flow_eps))
        r = RunReport()
        st = lib().clb_run(self.h, C.byref(d), C.byref(r))
        if not (allow_stop and st in (2, 3, 4)):
            self._check(st)
        out = {k: getattr(r, k) for k, _ in RunReport._fields_}
        out["status"] = st
        return out

    def refresh_dynamics(self, species=True, flow=True):
        self._check(lib().clb_refresh_dynamics(self.h, int(species), int(flow)))

    def ca_total(self):
        t = np.empty(self.N)
        self._check(lib().clb_get_field(self.h, FIELD_CA_TOTAL, 0, _ptr(t), 0))
        return t

    def ca_age(self):
        a = np.empty(self.N)
        self._check(lib().clb_get_field(self.h, FIELD_CA_AGE, 0, _ptr(a), 0))
        return a.astype(np.int64)

    def material(self):
        m = np.empty(self.N, dtype=np.int8)
        self._check(lib().clb_get_field(self.h, FIELD_MATERIAL, 0, _ptr(m), 2))
        return m

    def set_biomass(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        M = b.size // self.N
        self._check(lib().clb_set_biomass(self.h, M, _ptr(b)))

    def set_thermo_gate(self, species=(), nu=(), dG0=0.0, atp=0.0, dGatp=50.0, chi=1.0, cmin=1e-9, dGloss=0.0,
                        temperature=298.15, gas_constant=8.314462618e-3, conc_scale=1.0):
        """The thermodynamic gate of the biotic rates: one reaction block (user species indices
        and stoichiometric numbers, energies in kJ/mol). No terms turns it off."""
        d = ThermoDesc()
        d.n_terms = len(species)
        for i, (sp, v) in enumerate(zip(species, nu)):
            d.species[i], d.nu[i] = int(sp), float(v)
        d.dG0, d.atp, d.dGatp, d.chi, d.cmin, d.dGloss = dG0, atp, dGatp, chi, cmin, dGloss
        d.temperature, d.gas_constant, d.conc_scale = temperature, gas_constant, conc_scale
        self._check(lib().clb_set_thermo_gate(self.h, C.byref(d)))

    def set_symbolic_kinetics(self, path, species_names, microbe=-1, microbe_name=""):
        """A rate law read from a .sym file: microbe m's law (its biomass variable named
        microbe_name in the file), or the abiotic law for microbe = -1; species_names name the
        handle's species in user order."""
        arr = (C.c_char_p * len(species_names))(*[n.encode() for n in species_names])
        self._check(lib().clb_set_symbolic_kinetics(self.h, os.fsencode(path), C.cast(arr, C.c_void_p), int(microbe),
                                                    microbe_name.encode()))

    def symbolic_eval(self, microbe, X):
        """The bound law's rates on the rows of X (its variables in file order), by the device
        interpreter."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        nr = C.c_int()
        self._check(lib().clb_symbolic_eval(self.h, int(microbe), None, 0, None, C.byref(nr)))
        out = np.zeros((X.shape[0], nr.value))
        self._check(lib().clb_symbolic_eval(self.h, int(microbe), _ptr(X), X.shape[0], _ptr(out), C.byref(nr)))
        return out

    def set_graph_network(self, path, species_names, microbe=-1):
        """A rate law given as a .gnn graph network: microbe m's law, or the abiotic law for
        microbe = -1; species_names name the handle's species in user order."""
        arr = (C.c_char_p * len(species_names))(*[n.encode() for n in species_names])
        self._check(lib().clb_set_graph_network(self.h, os.fsencode(path), C.cast(arr, C.c_void_p), int(microbe)))

    def graph_network_eval(self, microbe, X):
        """The bound network's outputs on the rows of X (concentrations in the file's species
        order), evaluated on the device; returns (out [n][n_out], rows clamped to the training box)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        no, nc = C.c_int(), C.c_long()
        self._check(lib().clb_graph_network_eval(self.h, int(microbe), None, 0, None, C.byref(no), None))
        out = np.zeros((X.shape[0], no.value))
        self._check(lib().clb_graph_network_eval(self.h, int(microbe), _ptr(X), X.shape[0], _ptr(out), C.byref(no),
                                                 C.byref(nc)))
        return out, nc.value

    def set_surrogate_organism(self, path, species_names, microbe, half_saturation, max_uptake_flux,
                               biomass_molar_mass, decay):
        """Microbe `microbe` as a surrogate organism: a .srg network fed with its Michaelis-Menten
        uptake estimates (half_saturation, max_uptake_flux per species in user order)."""
        S = len(species_names)
        d = SurrogateDesc()
        for s in range(S):
            d.half_saturation[s] = float(half_saturation[s])
            d.max_uptake_flux[s] = float(max_uptake_flux[s])
        d.biomass_molar_mass = float(biomass_molar_mass)
        d.decay = float(decay)
        arr = (C.c_char_p * S)(*[n.encode() for n in species_names])
        self._check(lib().clb_set_surrogate_organism(self.h, os.fsencode(path), C.cast(arr, C.c_void_p),
                                                     int(microbe), C.cast(C.byref(d), C.c_void_p)))

    def surrogate_eval(self, microbe, X):
        """Every output of the bound surrogate network on the rows of X (its inputs), by the device;
        returns (out [n][n_out], rows clamped to the training box)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        no, nc = C.c_int(), C.c_long()
        self._check(lib().clb_surrogate_eval(self.h, int(microbe), None, 0, None, C.byref(no), None))
        out = np.zeros((X.shape[0], no.value))
        self._check(lib().clb_surrogate_eval(self.h, int(microbe), _ptr(X), X.shape[0], _ptr(out), C.byref(no),
                                             C.byref(nc)))
        return out, nc.value

    def checkpoint_save(self, path, flow=True, transport=True):
        """A restart file of the flow and/or transport lattices (FP64, exact)."""
        what = (CKPT_FLOW if flow else 0) | (CKPT_TRANSPORT if transport else 0)
        self._check(lib().clb_checkpoint_save(self.h, os.fsencode(path), what))

    def checkpoint_load(self, path):
        """Restores a restart file into this handle (same material map, same set-up)."""
        self._check(lib().clb_checkpoint_load(self.h, os.fsencode(path)))

    def write_vti(self, field, path, index=0):
        """One .vti file of the flow velocity (FIELD_FLOW_VELOCITY), the material map
        (FIELD_MATERIAL), a species' concentration or a microbe's biomass (FIELD_CONCENTRATION /
        FIELD_BIOMASS with `index`) over the interior x-planes."""
        self._check(lib().clb_write_vti(self.h, int(field), int(index), os.fsencode(path)))

    def ade_step(self, n=1):
        self._check(lib().clb_ade_step(self.h, n))

    def concentration(self, s):
        c = np.empty(self.N, dtype=np.float64)
        self._check(lib().clb_get_field(self.h, FIELD_CONCENTRATION, s, _ptr(c), 0))
        return c

    def set_concentration(self, s, c):
        """A species' concentration field: immobile species take it as it is, mobile ones the
        equilibrium populations at rest with that density."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        self._check(lib().clb_set_field(self.h, FIELD_CONCENTRATION, s, _ptr(c), 0))

    def set_ade_populations(self, s, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        self._check(lib().clb_set_field(self.h, FIELD_ADE_POPULATIONS, s, _ptr(g), 0))

    def ade_populations(self, s):
        g = np.empty(7 * self.N, dtype=np.float64)
        self._check(lib().clb_get_field(self.h, FIELD_ADE_POPULATIONS, s, _ptr(g), 0))
        return g.reshape(7, self.N)

    def biomass(self, m):
        b = np.empty(self.N, dtype=np.float64)
        self._check(lib().clb_get_field(self.h, FIELD_BIOMASS, m, _ptr(b), 0))
        return b

    def reduce(self):
        s = Stats()
        self._check(lib().clb_reduce(self.h, C.byref(s)))
        S = self.S
        return {"total": np.array(s.total[:S]), "content": np.array(s.content[:S]),
                "biomass": np.array(s.biomass[:]), "min": np.array(s.min_c[:S]), "max": np.array(s.max_c[:S]),
                "open_voxels": s.open_voxels, "nonfinite": s.nonfinite, "ade_iterations": s.ade_iterations}

    def reduce_noalloc(self):
        """clb_reduce_noalloc: the reductions of reduce() from the library's fixed per-device
        buffer, with no allocation; calls on one device must not overlap in time."""
        s = Stats()
        self._check(lib().clb_reduce_noalloc(self.h, C.byref(s)))
        S = self.S
        return {"total": np.array(s.total[:S]), "content": np.array(s.content[:S]),
                "biomass": np.array(s.biomass[:]), "min": np.array(s.min_c[:S]), "max": np.array(s.max_c[:S]),
                "open_voxels": s.open_voxels, "nonfinite": s.nonfinite, "ade_iterations": s.ade_iterations}

    # ---- equilibrium speciation and its surrogate
    def speciation_setup(self, stoich, logK, component_species, tol=1e-10, max_iterations=200):
        S = np.asarray(stoich, dtype=np.float64)
        d = SpeciationDesc()
        d.n_species, d.n_components = S.shape
        for i in range(S.shape[0]):
            for j in range(S.shape[1]):
                d.stoich[i][j] = S[i, j]
            d.logK[i] = float(logK[i])
        for j, cs in enumerate(component_species):
            d.component_species[j] = int(cs)
        d.tolerance, d.max_iterations = tol, max_iterations
        self.eq_ns = S.shape[0]
        self._check(lib().clb_speciation_setup(self.h, C.byref(d)))

    def set_speciation_mode(self, mode):
        self._check(lib().clb_set_speciation_mode(self.h, mode))

    def speciation_stats(self):
        s = SpeciationStats()
        self._check(lib().clb_speciation_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in SpeciationStats._fields_}

    def speciation_solve(self, conc):
        c = np.ascontiguousarray(conc, dtype=np.float64)
        n = c.shape[0]
        out = np.empty_like(c)
        it = np.empty(n, dtype=np.int32)
        self._check(lib().clb_speciation_solve(self.h, _ptr(c), n, _ptr(out), _ptr(it)))
        return out, it

    def surrogate_train(self, log_c_lo, log_c_hi, n_samples=200000, epochs=60, batch=1024, patience=8,
                        learning_rate=3e-3, val_fraction=0.15, seed=1, from_domain=False, jitter=0.0):
        """from_domain: train on the species states of the domain's open voxels (each species
        scaled by 10^U(-jitter, jitter)) instead of states drawn from [log_c_lo, log_c_hi]."""
        d = SurrogateTrainDesc()
        d.n_samples, d.epochs, d.batch, d.patience = n_samples, epochs, batch, patience
        d.learning_rate, d.val_fraction, d.seed = learning_rate, val_fraction, seed
        d.source, d.jitter = int(bool(from_domain)), float(jitter)
        for i, (lo, hi) in enumerate(zip(log_c_lo, log_c_hi)):
            d.log_c_lo[i], d.log_c_hi[i] = lo, hi
        r = SurrogateReport()
        self._check(lib().clb_surrogate_train(self.h, C.byref(d), C.byref(r)))
        return {k: getattr(r, k) for k, _ in SurrogateReport._fields_}

    def surrogate_set_check(self, range_margin=0.02, newton_polish=2, residual_tol=1e-6):
        self._check(lib().clb_surrogate_set_check(self.h, range_margin, int(newton_polish), residual_tol))

    def surrogate_predict(self, conc, residual_check=True):
        c = np.ascontiguousarray(conc, dtype=np.float64)
        n = c.shape[0]
        out = np.empty_like(c)
        acc = np.empty(n, dtype=np.int32)
        self._check(lib().clb_surrogate_predict(self.h, _ptr(c), n, _ptr(out), _ptr(acc), int(residual_check)))
        return out, acc.astype(bool)

    def surrogate_params(self, params=None, scaling=None):
        n = lib().clb_surrogate_param_count()
        out = np.empty(n, dtype=np.float32)
        sc = np.empty(64, dtype=np.float32)
        pin = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        sin = None if scaling is None else np.ascontiguousarray(scaling, dtype=np.float32)
        self._check(lib().clb_surrogate_params(self.h, _ptr(out), None if pin is None else _ptr(pin), _ptr(sc),
                                               None if sin is None else _ptr(sin)))
        return out, sc

    def surrogate_gradient(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        n = X.shape[0]
        g = np.empty(lib().clb_surrogate_param_count(), dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._check(lib().clb_surrogate_gradient(self.h, _ptr(X), _ptr(Y), n, _ptr(g), _ptr(loss)))
        return g, float(loss[0])


def vti_write(path, shape, arrays):
    """Writes host arrays as one .vti file over the interior x-planes: `arrays` maps a name to a
    float64 or float32 array of shape [N] or [components][N] (x slowest, N = nx ny nz)."""
    nx, ny, nz = shape
    N = nx * ny * nz
    keep, names, comps, types = [], [], [], []
    for name, a in arrays.items():
        a = np.asarray(a)
        dt = np.float32 if a.dtype == np.float32 else np.float64
        a = np.ascontiguousarray(a, dtype=dt).reshape(-1, N)
        keep.append(a)
        names.append(name.encode())
        comps.append(a.shape[0])
        types.append(1 if dt == np.float32 else 0)
    n = len(keep)
    cn = (C.c_char_p * max(n, 1))(*names)
    cc = (C.c_int32 * max(n, 1))(*comps)
    ct = (C.c_int32 * max(n, 1))(*types)
    cd = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in keep])
    _check_global(lib().clb_vti_write(os.fsencode(path), nx, ny, nz, n, cn, cc, ct, cd))


class Case:
    """A CompLaB.xml run description (clb_case_*): parse, set up a Domain from it with the
    reference's unit chain, run it."""

    def __init__(self, xml_path):
        c = C.c_void_p()
        st = lib().clb_case_load(os.fsencode(xml_path), C.byref(c))
        if st != 0:
            raise ClbError(st, lib().clb_case_error().decode())
        self.c = c

    def get(self, key):
        v = C.c_double()
        st = lib().clb_case_get(self.c, key.encode(), C.byref(v))
        if st != 0:
            raise ClbError(st, lib().clb_case_error().decode())
        return v.value

    def setup(self, flow_precision=F64, ade_precision=F64):
        """The Domain the description builds (its handle owned by the returned object)."""
        h = C.c_void_p()
        st = lib().clb_case_setup(self.c, int(flow_precision), int(ade_precision), C.byref(h))
        if st != 0:
            raise ClbError(st, lib().clb_case_error().decode())
        D = Domain.__new__(Domain)
        D.h = h
        D.nx, D.ny, D.nz = int(self.get("nx")), int(self.get("ny")), int(self.get("nz"))
        D.N = D.nx * D.ny * D.nz
        D.S = int(self.get("n_substrates"))
        return D

    def run(self, D, iterations=-1, output_dir=None):
        r = RunReport()
        st = lib().clb_case_run(self.c, D.h, int(iterations), None if output_dir is None else os.fsencode(output_dir),
                                C.byref(r))
        if st != 0:
            raise ClbError(st, lib().clb_case_error().decode())
        return {k: getattr(r, k) for k, _ in RunReport._fields_}

    def close(self):
        if getattr(self, "c", None):
            lib().clb_case_free(self.c)
            self.c = None

    def __del__(self):
        self.close()


class Batch:
    """An ensemble of Domains advanced together (clb_batch_*): by default one persistent launch
    runs several steps of every lattice of every domain (a table of tiles with per-domain
    dependencies), launches replayed from a CUDA graph; or one launch per lattice and step.
    Results equal stepping each domain on its own. The domains must stay alive and unchanged
    while the batch exists."""

    def __init__(self, domains):
        self.domains = list(domains)
        arr = (C.c_void_p * len(self.domains))(*[d.h for d in self.domains])
        b = C.c_void_p()
        _check_global(lib().clb_batch_create(arr, len(self.domains), C.byref(b)))
        self.b = b

    def step(self, n=1, flow=True, transport=True):
        _check_global(lib().clb_batch_step(self.b, int(n), int(flow), int(transport)))

    def schedule(self, persistent=True, tile=2048, lag=8, steps_per_launch=2, ctas_per_sm=4, staged_flow=False):
        """persistent: the item-table schedule; else one launch per lattice and step, the flow step
        through the staged kernels when staged_flow (4- and 8-byte storage)."""
        mode = 1 if persistent else (2 if staged_flow else 0)
        _check_global(lib().clb_batch_schedule(self.b, mode, int(tile), int(lag), int(steps_per_launch),
                                               int(ctas_per_sm)))

    def get_schedule(self):
        v = [C.c_int() for _ in range(5)]
        _check_global(lib().clb_batch_get_schedule(self.b, *[C.byref(x) for x in v]))
        return dict(persistent=v[0].value == 1, staged_flow=v[0].value == 2, tile=v[1].value, lag=v[2].value,
                    steps_per_launch=v[3].value, ctas_per_sm=v[4].value)

    def set_stream(self, stream):
        """stream: a cudaStream_t as an integer (torch.cuda.Stream().cuda_stream), or None."""
        _check_global(lib().clb_batch_set_stream(self.b, C.c_void_p(stream) if stream else None))

    def set_wait_limit(self, ns):
        """Limit of one dependency wait of the persistent schedule, in nanoseconds."""
        _check_global(lib().clb_batch_set_wait_limit(self.b, int(ns)))

    def autotune(self, steps=20):
        buf = C.create_string_buffer(4096)
        _check_global(lib().clb_batch_autotune(self.b, int(steps), buf, 4096))
        return buf.value.decode()

    def counts(self):
        a, t = C.c_int64(), C.c_int64()
        _check_global(lib().clb_batch_counts(self.b, C.byref(a), C.byref(t)))
        return a.value, t.value

    def close(self):
        if getattr(self, "b", None):
            lib().clb_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        self.close()

"""ctypes front end of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
baseline leg, never by the product. The per-material dynamics tables are derived here from the
reference's setup rules, independently of the product's own table code:

  flow lattice (complab_functions.hh:296-345): every code IncBGK(omega) by default; the
  bounce-back code BounceBack; the solid code NoDynamics; each microbe's code IncBGK(omega_bio)
  with omega_bio = 1/(r (1/omega - 1/2) + 1/2), or BounceBack when r <= 1e-14.

  species lattices (complab_functions.hh:347-442, complab.cpp:1589-1656): pore BGK, biofilm
  BGK with the biofilm omega, wall and solid BounceBack for a mobile species; kinetics where
  the mask is neither solid nor wall (complab3d_processors_part1.hh:96-99).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

DYN_BB, DYN_NONE, DYN_BGK = 0, 1, 2
ADE_BB, ADE_NONE, ADE_PORE, ADE_BIO = 0, 1, 2, 3

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, dp, ip = C.c_void_p, C.c_double, C.c_int
        sig = {
            "orc_set_threads": ([ip], None), "orc_max_threads": ([], ip),
            "orc_flow_create": ([ip, ip, ip, vp, vp, vp, dp], vp), "orc_flow_destroy": ([vp], None),
            "orc_flow_step": ([vp, ip], None), "orc_flow_solve": ([vp, ip, dp], ip),
            "orc_flow_energy": ([vp], dp), "orc_flow_iterations": ([vp], C.c_long),
            "orc_flow_velocity": ([vp, vp], None), "orc_flow_populations": ([vp, vp], None),
            "orc_flow_set_populations": ([vp, vp], None),
            "orc_ade_create": ([ip, ip, ip, vp, ip, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], vp),
            "orc_ade_destroy": ([vp], None), "orc_ade_set_kinetics": ([vp, ip, vp, ip, dp], None),
            "orc_ade_set_biomass": ([vp, ip, vp], None), "orc_ade_step": ([vp, ip], None),
            "orc_ade_density": ([vp, ip, vp], None), "orc_ade_populations": ([vp, ip, vp], None),
            "orc_ade_biomass": ([vp, vp], None), "orc_ade_set_velocity": ([vp, vp], None),
            "orc_eq_nr": ([ip, ip, vp, vp, vp, dp, ip, vp, vp, vp], ip),
            "orc_ade_set_speciation": ([vp, ip, ip, vp, vp, vp, dp, ip], None),
            "orc_ade_set_abiotic": ([vp, ip, vp, ip, ip], None),
            "orc_ade_set_precip": ([vp, ip, dp, ip, ip, dp, ip, ip, vp, ip, ip], None),
            "orc_ade_geometry_update": ([vp, vp, vp], None),
            "orc_ade_material": ([vp, vp], None),
            "orc_ca_setup": ([vp, dp, dp, C.c_uint64, ip, vp, ip, ip, vp], None),
            "orc_ca_step": ([vp, vp, vp], ip),
            "orc_ade_refresh_dynamics": ([vp], None),
            "orc_ca_fields": ([vp, vp, vp], None),
            "orc_flow_set_material": ([vp, vp], None),
            "orc_flow_set_dynamics": ([vp, ip, ip, dp], None),
            "orc_biotic_increments": ([vp, vp, vp, vp, vp], None), "orc_abiotic_increments": ([vp, vp, vp], None),
            "orc_ade_set_thermo": ([vp, ip, vp, vp, vp], None), "orc_thermo_factor": ([vp, vp], dp),
            "orc_ade_set_immobile": ([vp, ip, vp], None), "orc_ade_set_stamp": ([vp, vp], None),
            "orc_ade_stamp": ([vp, vp], None),
            "orc_ca_mask_total_once": ([vp], None), "orc_ca_set_half": ([vp, ip], None), "orc_ca_age_relax": ([vp, ip], ip),
            "orc_ca_age_flags": ([vp, vp], None),
            "orc_dissolution_increments": ([ip, ip, ip, ip, ip, dp, ip, vp, ip, vp, ip, ip, vp, vp, vp], None),
            "orc_sphere_pack": ([ip, ip, ip, dp, dp, dp, C.c_uint64, C.c_char_p, ip, ip, ip, vp], ip),
            "orc_sym_eval": ([C.c_char_p, ip, vp, vp, C.POINTER(C.c_int)], ip),
            "orc_ade_set_symbolic": ([vp, C.c_char_p, C.c_char_p, ip, C.c_char_p], ip),
            "orc_gnn_eval": ([C.c_char_p, ip, vp, vp, C.POINTER(C.c_int)], ip),
            "orc_ade_set_graph_network": ([vp, C.c_char_p, C.c_char_p, ip], ip),
            "orc_srg_eval": ([C.c_char_p, ip, vp, vp, C.POINTER(C.c_int)], ip),
            "orc_ade_set_surrogate": ([vp, C.c_char_p, C.c_char_p, ip, vp, vp, dp, dp], ip),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed, walls="yz", grain=1, wall=1, pore=2):
    """The porosity-targeted sphere pack of the library's clb_geom_sphere_pack, restated in the
    oracle (the CPU baseline builds its input maps with it, without the product library)."""
    out = np.empty(nx * ny * nz, dtype=np.int8)
    if lib().orc_sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed, walls.encode(), grain, wall, pore, _p(out)):
        raise ValueError("bad sphere-pack arguments")
    return out


def sym_eval(path, X, n_rates_max=16):
    """The oracle's evaluation of a .sym rate-law file on the rows of X (its variables in file order)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0] * n_rates_max)
    nr = C.c_int()
    if lib().orc_sym_eval(os.fsencode(path), X.shape[0], _p(X), _p(out), C.byref(nr)) != 0:
        raise ValueError(f"cannot load {path}")
    return out[:X.shape[0] * nr.value].reshape(X.shape[0], nr.value)


def gnn_eval(path, X, n_out_max=17):
    """The oracle's evaluation of a .gnn graph network on the rows of X (concentrations in the
    file's species order): the species rates, then growth when the file has it."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0] * n_out_max)
    no = C.c_int()
    if lib().orc_gnn_eval(os.fsencode(path), X.shape[0], _p(X), _p(out), C.byref(no)) != 0:
        raise ValueError(f"cannot load {path}")
    return out[:X.shape[0] * no.value].reshape(X.shape[0], no.value)


def srg_eval(path, X, n_out_max=32):
    """The oracle's evaluation of a .srg surrogate network on the rows of X (its inputs), clamped to
    its training box: every output, output 0 the growth rate."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0] * n_out_max)
    no = C.c_int()
    if lib().orc_srg_eval(os.fsencode(path), X.shape[0], _p(X), _p(out), C.byref(no)) != 0:
        raise ValueError(f"cannot load {path}")
    return out[:X.shape[0] * no.value].reshape(X.shape[0], no.value)


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


def eq_nr(stoich, logK, comp, conc, tol=1e-10, max_it=200):
    """Newton-Raphson speciation of each row of conc (the oracle's restatement)."""
    S = np.ascontiguousarray(stoich, dtype=np.float64)
    lk = np.ascontiguousarray(logK, dtype=np.float64)
    cp = np.ascontiguousarray(comp, dtype=np.int32)
    conc = np.atleast_2d(np.asarray(conc, dtype=np.float64))
    out = np.empty_like(conc)
    conv = np.empty(conc.shape[0], dtype=np.int32)
    its = np.empty(conc.shape[0], dtype=np.int32)
    cv = C.c_int()
    for r in range(conc.shape[0]):
        ci = np.ascontiguousarray(conc[r])
        o = np.empty(S.shape[0])
        its[r] = lib().orc_eq_nr(S.shape[0], S.shape[1], _p(S), _p(lk), _p(cp), tol, max_it, _p(ci), _p(o), C.byref(cv))
        conv[r] = cv.value
        out[r] = o
    return out, conv.astype(bool), its


class OracleFlow:
    def __init__(self, mat, nx, ny, nz, tau, delta_p, solid_code=0, bounce_back_code=1, bio_codes=(),
                 perm_ratio=()):
        omega = 1.0 / tau
        dyn = np.full(256, DYN_BGK, dtype=np.int32)
        om = np.full(256, omega, dtype=np.float64)
        if bounce_back_code >= 0:
            dyn[bounce_back_code] = DYN_BB
        if solid_code >= 0:
            dyn[solid_code] = DYN_NONE
        for c, r in zip(bio_codes, perm_ratio):
            if r > 1e-14:
                dyn[c] = DYN_BGK
                om[c] = 1.0 / (r * (1.0 / omega - 0.5) + 0.5)
            else:
                dyn[c] = DYN_BB
        self.N = nx * ny * nz
        self.shape = (nx, ny, nz)
        self._mat = np.ascontiguousarray(mat, dtype=np.int8)
        self.h = lib().orc_flow_create(nx, ny, nz, _p(self._mat), _p(dyn), _p(om), delta_p)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_flow_destroy(self.h)
            self.h = None

    def step(self, n=1):
        lib().orc_flow_step(self.h, n)

    def solve(self, max_it, eps):
        return lib().orc_flow_solve(self.h, max_it, eps)

    @property
    def energy(self):
        return lib().orc_flow_energy(self.h)

    def velocity(self):
        u = np.empty(3 * self.N)
        lib().orc_flow_velocity(self.h, _p(u))
        return u.reshape(3, self.N)

    def populations(self):
        f = np.empty(19 * self.N)
        lib().orc_flow_populations(self.h, _p(f))
        return f.reshape(19, self.N)

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().orc_flow_set_populations(self.h, _p(f))

    def set_material(self, mat):
        self._mat = np.ascontiguousarray(mat, dtype=np.int8)
        lib().orc_flow_set_material(self.h, _p(self._mat))

    def set_dynamics(self, code, dyn, omega):
        lib().orc_flow_set_dynamics(self.h, int(code), int(dyn), float(omega))


class OracleAde:
    def __init__(self, mat, nx, ny, nz, species, u, solid_code=0, bounce_back_code=1, bio_codes=()):
        dyn = np.full(256, ADE_PORE, dtype=np.int32)
        react = np.ones(256, dtype=np.int32)
        for c in bio_codes:
            dyn[c] = ADE_BIO
        for c in (bounce_back_code, solid_code):
            if c >= 0:
                dyn[c] = ADE_BB
                react[c] = 0
        S = len(species)
        g = lambda k, d: np.array([s.get(k, d) for s in species], dtype=np.float64)
        gi = lambda k, d: np.array([s.get(k, d) for s in species], dtype=np.int32)
        wp = g("omega_pore", 1.0)
        wb = np.array([s.get("omega_biofilm", s["omega_pore"]) for s in species], dtype=np.float64)
        self._keep = [np.ascontiguousarray(mat, dtype=np.int8), dyn, react, wp, wb, gi("mobile", 1),
                      gi("left_type", 1), gi("right_type", 1), g("left_bc", 0.0), g("right_bc", 0.0),
                      g("c0", 0.0), np.ascontiguousarray(u, dtype=np.float64).reshape(-1)]
        k = self._keep
        self.N = nx * ny * nz
        self.S = S
        self.h = lib().orc_ade_create(nx, ny, nz, _p(k[0]), S, _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]),
                                      _p(k[5]), _p(k[6]), _p(k[7]), _p(k[8]), _p(k[9]), _p(k[10]), _p(k[11]))
        self.M = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ade_destroy(self.h)
            self.h = None

    def set_kinetics(self, law, params, dt):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._prm = p
        lib().orc_ade_set_kinetics(self.h, law, _p(p), p.size, dt)

    def set_biomass(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
        self.M = b.size // self.N
        lib().orc_ade_set_biomass(self.h, self.M, _p(b))

    def set_velocity(self, u):
        self._keep[11] = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        lib().orc_ade_set_velocity(self.h, _p(self._keep[11]))

    def set_speciation(self, stoich, logK, comp, tol=1e-10, max_it=200):
        S = np.ascontiguousarray(stoich, dtype=np.float64)
        self._spec = [S, np.ascontiguousarray(logK, dtype=np.float64), np.ascontiguousarray(comp, dtype=np.int32)]
        lib().orc_ade_set_speciation(self.h, S.shape[0], S.shape[1], _p(self._spec[0]), _p(self._spec[1]),
                                     _p(self._spec[2]), tol, max_it)

    def set_symbolic(self, path, names, microbe=-1, microbe_name=""):
        """A .sym rate law bound to the species `names` (microbe m's law, or abiotic for -1)."""
        rc = lib().orc_ade_set_symbolic(self.h, os.fsencode(path), "\n".join(names).encode(), int(microbe),
                                        microbe_name.encode())
        if rc != 0:
            raise ValueError(f"cannot bind {path}")

    def set_graph_network(self, path, names, microbe=-1):
        """A .gnn graph network bound to the species `names` (microbe m's law, or abiotic for -1)."""
        rc = lib().orc_ade_set_graph_network(self.h, os.fsencode(path), "\n".join(names).encode(), int(microbe))
        if rc != 0:
            raise ValueError(f"cannot bind {path} ({rc})")

    def set_surrogate(self, path, names, microbe, half_saturation, max_uptake_flux, biomass_molar_mass, decay):
        """Microbe `microbe` as a surrogate organism (.srg network, uptake parameters per species)."""
        self._srg = [np.ascontiguousarray(half_saturation, dtype=np.float64),
                     np.ascontiguousarray(max_uptake_flux, dtype=np.float64)]
        rc = lib().orc_ade_set_surrogate(self.h, os.fsencode(path), "\n".join(names).encode(), int(microbe),
                                         _p(self._srg[0]), _p(self._srg[1]), float(biomass_molar_mass), float(decay))
        if rc != 0:
            raise ValueError(f"cannot bind {path} ({rc})")

    def set_abiotic(self, law, params, surface_only=0):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._prm2 = p
        lib().orc_ade_set_abiotic(self.h, law, _p(p), p.size, int(surface_only))

    def set_precip(self, mineral, full, precip_code=0, dissolution=0, reopen=0.9, pore_code=2, dis_law=0,
                   dis_params=(), dis_surface_only=1):
        d = np.ascontiguousarray(dis_params if len(dis_params) else [0.0], dtype=np.float64)
        self._dprm = d
        lib().orc_ade_set_precip(self.h, int(mineral), float(full), int(precip_code), int(dissolution),
                                 float(reopen), int(pore_code), int(dis_law), _p(d), d.size, int(dis_surface_only))

    def set_thermo(self, species=(), nu=(), dG0=0.0, atp=0.0, dGatp=50.0, chi=1.0, cmin=1e-9, dGloss=0.0,
                   temperature=298.15, gas_constant=8.314462618e-3, conc_scale=1.0):
        """The thermodynamic gate of the biotic rates (one reaction block, energies in kJ/mol);
        no terms turns it off."""
        sp = np.ascontiguousarray(species if len(species) else [0], dtype=np.int32)
        nu_ = np.ascontiguousarray(nu if len(nu) else [0.0], dtype=np.float64)
        v = np.array([dG0, atp, dGatp, chi, cmin, dGloss, temperature, gas_constant, conc_scale], np.float64)
        self._thermo = (sp, nu_, v)
        lib().orc_ade_set_thermo(self.h, len(species), _p(sp), _p(nu_), _p(v))

    def thermo_factor(self, c):
        c = np.ascontiguousarray(c, dtype=np.float64)
        return lib().orc_thermo_factor(self.h, _p(c))

    def set_immobile(self, s, c):
        c = np.ascontiguousarray(c, dtype=np.float64).reshape(-1)
        lib().orc_ade_set_immobile(self.h, int(s), _p(c))

    def set_stamp(self, st):
        st = np.ascontiguousarray(st, dtype=np.uint8).reshape(-1)
        lib().orc_ade_set_stamp(self.h, _p(st))

    def stamp(self):
        out = np.empty(self.N, dtype=np.uint8)
        lib().orc_ade_stamp(self.h, _p(out))
        return out

    def geometry_update(self):
        a, b = C.c_int(), C.c_int()
        lib().orc_ade_geometry_update(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def material(self):
        m = np.empty(self.N, dtype=np.int8)
        lib().orc_ade_material(self.h, _p(m))
        return m

    def ca_setup(self, bmax, frac, seed, pore_codes=(2,), bb=1, solid=0, bio_codes=(3, 4), half=False):
        """half: the 'half' push (halfPushExcessBiomass3D) instead of 'fraction'."""
        pc = np.ascontiguousarray(pore_codes, dtype=np.int32)
        bc = np.ascontiguousarray(bio_codes[:self.M], dtype=np.int32)
        self._ca = (pc, bc)
        lib().orc_ca_setup(self.h, float(bmax), float(frac), int(seed), pc.size, _p(pc), int(bb), int(solid), _p(bc))
        lib().orc_ca_set_half(self.h, int(bool(half)))

    def ca_step(self):
        a, b = C.c_int(), C.c_int()
        rc = lib().orc_ca_step(self.h, C.byref(a), C.byref(b))
        return rc, a.value, bool(b.value)

    def refresh_dynamics(self):
        lib().orc_ade_refresh_dynamics(self.h)

    def ca_fields(self):
        t = np.empty(self.N)
        a = np.empty(self.N, dtype=np.int32)
        lib().orc_ca_fields(self.h, _p(t), _p(a))
        return t, a

    def biotic_increments(self, C, B):
        """run_kinetics on given densities C [S][N] and biomass B [M][N]: the clamped increments."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64).reshape(-1, self.N)
        dC, dB = np.empty_like(C), np.empty((B.shape[0], self.N))
        lib().orc_biotic_increments(self.h, _p(C), _p(B), _p(dC), _p(dB))
        return dC, dB

    def abiotic_increments(self, C):
        """run_abiotic_kinetics (or the surface-only pass) on given densities C [S][N]."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        dC = np.empty_like(C)
        lib().orc_abiotic_increments(self.h, _p(C), _p(dC))
        return dC

    def ca_mask_total_once(self):
        """updateLocalMaskNtotalLattices3D once on the current state."""
        lib().orc_ca_mask_total_once(self.h)

    def ca_age_relax(self, max_sweeps=1000):
        """updateAgeDistance3D until no age changes; returns the sweeps that changed something."""
        return lib().orc_ca_age_relax(self.h, int(max_sweeps))

    def ca_open_flags(self):
        d = np.empty(self.N, dtype=np.int32)
        lib().orc_ca_age_flags(self.h, _p(d))
        return d

    def step(self, n=1):
        lib().orc_ade_step(self.h, n)

    def concentration(self, s):
        c = np.empty(self.N)
        lib().orc_ade_density(self.h, s, _p(c))
        return c

    def populations(self, s):
        g = np.empty(7 * self.N)
        lib().orc_ade_populations(self.h, s, _p(g))
        return g.reshape(7, self.N)

    def biomass(self):
        b = np.empty(self.M * self.N)
        lib().orc_ade_biomass(self.h, _p(b))
        return b.reshape(self.M, self.N)


def dissolution_increments(shape, S, sM, dt, law, prm, surface_only, mat, solid, bb, stamp, C, dC):
    """The dissolution increments of one step for given fields (park per open face, gather by the
    open neighbours with the headroom clamp): C [S][N] densities, dC [S][N] pending increments;
    returns the increments after both passes."""
    nx, ny, nz = shape
    prm = np.ascontiguousarray(prm, dtype=np.float64)
    mat = np.ascontiguousarray(mat, dtype=np.int8)
    stamp = np.ascontiguousarray(stamp, dtype=np.uint8)
    C = np.ascontiguousarray(C, dtype=np.float64)
    out = np.array(dC, dtype=np.float64, copy=True, order="C")
    lib().orc_dissolution_increments(nx, ny, nz, S, sM, dt, law, _p(prm), int(surface_only), _p(mat), solid, bb,
                                     _p(stamp), _p(C), _p(out))
    return out

"""Regenerates tests/golden/geometry.json from the reference's own geometry generator
(complab3d_geometry.hh, compiled into oracle/_ref/libref_geometry.so by `make -C oracle ref`),
tests/golden/speciation.json from the reference's own equilibrium solver (EquilibriumChemistry,
compiled into oracle/_ref/libref_eqsolver.so with the reference's tests/palabos_stub.hh) and
tests/golden/dissolution.npz from the reference's own dissolution processors
(surfaceDissolutionKinetics3D + dissolutionGather3D of dissolutionVOP.hh, compiled into
oracle/_ref/libref_vop.so against oracle/palabos_shim.hh) on seeded fields, and
tests/golden/conversion.npz from the reference's node conversions (precipNodeConversion3D,
dissolNodeConversion3D, the same library), tests/golden/kinetics.npz from the reference's
kinetics processors (run_kinetics,
run_abiotic_kinetics of complab3d_processors_part1.hh and surfaceAbioticKinetics3D, compiled into
oracle/_ref/libref_kinetics.so with the FeS law of examples/15) and its thermodynamic gate
(complab3d_thermo.hh, alone and inside run_kinetics), tests/golden/automaton.npz from
the biofilm automaton's mask/total update and age relaxation
(updateLocalMaskNtotalLattices3D and updateAgeDistance3D of complab3d_processors_part2.hh, the
same library) on seeded maps.

Run from the repository root in a checkout that has the reference sources:
    make -C oracle ref && python tests/golden/make_golden.py
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_geometry.so")

CASES = [
    dict(kind="channel", nx=12, ny=9, nz=7, walls="y"),
    dict(kind="spheres", nx=24, ny=20, nz=16, radius=4.0, count=12, seed=7, walls="y"),
    dict(kind="spheres", nx=40, ny=32, nz=32, radius=6.0, count=20, seed=1, walls="yz"),
    dict(kind="cylinders", nx=30, ny=24, nz=5, radius=3.5, count=9, seed=3, walls="y"),
    dict(kind="random", nx=20, ny=16, nz=12, porosity=0.35, seed=11, walls="y"),
    dict(kind="random", nx=32, ny=32, nz=32, porosity=0.5, seed=2, walls="none"),
    dict(kind="fracture", nx=48, ny=40, nz=6, aperture=12.0, roughness=0.3, seed=1004, walls="none"),
    dict(kind="fracture", nx=30, ny=30, nz=4, aperture=6.0, roughness=2.0, seed=5, walls="y"),
    dict(kind="layered", nx=20, ny=24, nz=10, porosity=0.4, layers=4, seed=9, walls="z"),
]
DEFAULTS = dict(porosity=0.4, radius=6.0, aperture=6.0, roughness=2.0, count=20, layers=4, seed=1, walls="y")


def ref_generate(L, c):
    o = dict(DEFAULTS, **c)
    n = o["nx"] * o["ny"] * o["nz"]
    out = np.empty(n, dtype=np.int32)
    rc = L.ref_geom_generate(o["kind"].encode(), o["nx"], o["ny"], o["nz"], C.c_double(o["porosity"]),
                             C.c_double(o["radius"]), C.c_double(o["aperture"]), C.c_double(o["roughness"]),
                             o["count"], o["layers"], C.c_ulonglong(o["seed"]), o["walls"].encode(),
                             out.ctypes.data_as(C.c_void_p))
    assert rc == 0
    xs = out.reshape(o["nz"], o["ny"], o["nx"]).transpose(2, 1, 0).astype(np.int8)  # -> x slowest
    po, op, iso = C.c_double(), C.c_long(), C.c_long()
    cl, sp, pe = C.c_int(), C.c_int(), C.c_int()
    L.ref_geom_inspect(out.ctypes.data_as(C.c_void_p), o["nx"], o["ny"], o["nz"], C.byref(po), C.byref(op),
                       C.byref(iso), C.byref(cl), C.byref(sp), C.byref(pe))
    return o, np.ascontiguousarray(xs).ravel(), dict(porosity=po.value, open_voxels=op.value,
                                                      isolated_voxels=iso.value, clusters=cl.value,
                                                      spanning_clusters=sp.value, percolates=pe.value)


def speciation_cases():
    """Reference AA-PCF solutions (complab3d_processors_part4_eqsolver.hh, compiled into
    oracle/_ref/libref_eqsolver.so) of the carbonate example tableau and the 5x12 tableau."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "complab3d-gems_b200"))
    import workloads
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_eqsolver.so"))
    out = []
    for name, (S, logK, comp), n, lo, hi in [
        ("carbonate", workloads.carbonate_tableau(), 24, [-5, -9, -8, -6], [-2, -5, -4, -3]),
        ("tableau_5x12", workloads.tableau_5x12(), 48, [-7] * 5 + [-10] * 7, [-3] * 5 + [-5] * 7),
    ]:
        ns, nc = S.shape
        states = workloads.species_states(n, ns, np.array(lo), np.array(hi), seed=17)
        res, conv, its = [], [], []
        for c in states:
            o = np.zeros(ns)
            cv, it = C.c_int(), C.c_int()
            L.ref_eq_solve(ns, nc, np.ascontiguousarray(S).ctypes.data_as(C.c_void_p),
                           np.ascontiguousarray(logK).ctypes.data_as(C.c_void_p),
                           np.array(comp, dtype=np.int32).ctypes.data_as(C.c_void_p), C.c_double(1e-10), 200,
                           np.ascontiguousarray(c).ctypes.data_as(C.c_void_p), o.ctypes.data_as(C.c_void_p),
                           C.byref(cv), C.byref(it))
            res.append(o.tolist()); conv.append(cv.value); its.append(it.value)
        out.append(dict(name=name, stoich=S.tolist(), logK=logK.tolist(), component_species=comp, tol=1e-10,
                        inputs=states.tolist(), reference_outputs=res, converged=conv, iterations=its))
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "speciation.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {sum(len(c['inputs']) for c in out)} speciation cases")


def dissolution_cases():
    """Seeded small fields (open voxels, rock, walls; precipitated mineral voxels; some negative
    water; pending increments) through the reference's park + gather passes, both dissolution
    laws, with and without the surface-only rule."""
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_vop.so"))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rng = np.random.default_rng(2024)
    shape, S, sM = (10, 8, 7), 4, 3
    nx, ny, nz = shape
    N = nx * ny * nz
    rec = {}
    for case in range(6):
        mat = np.where(rng.random(N) < 0.2, 0, 2).astype(np.int8)
        mat[rng.random(N) < 0.05] = 1
        stamp = ((mat == 0) & (rng.random(N) < 0.6)).astype(np.uint8)
        Cf = rng.uniform(0.0, 1.0, (S, N))
        Cf[sM] = np.where(stamp == 1, rng.uniform(0.0, 2.0, N), 0.0)
        Cf[1] -= 0.3
        dC0 = np.where(rng.random((S, N)) < 0.3, rng.uniform(-0.05, 0.05, (S, N)), 0.0)
        law = 1 if case % 2 == 0 else 2
        prm = np.array([0.7, 0 if case < 4 else -1, 1.0, -2.0, 0.5, 0.0] if law == 1
                       else [0.3, -1.5, 1.0, 1.0, 0.0, 0.0], np.float64)
        dt = 1.0 if case < 3 else 0.25
        surf = int(case % 3 != 2)
        dC = dC0.copy()
        L.ref_dissolution_increments(nx, ny, nz, S, sM, C.c_double(dt), law, P(prm), len(prm), surf, P(mat), 0, 1,
                                     P(stamp), P(Cf), P(dC))
        for k, v in dict(mat=mat, stamp=stamp, C=Cf, dC0=dC0, prm=prm, dC=dC,
                         meta=np.array([law, surf, dt, S, sM])).items():
            rec[f"{case}_{k}"] = v
    rec["shape"] = np.array(shape)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "dissolution.npz"), **rec)
    print("wrote 6 dissolution cases")


def ca_cases():
    """Seeded small maps (pore, two biofilm codes, rock, walls) with biomass at and below the
    ceiling: the oracle's automaton set-up gives the stored totals, ages and open flags; the
    biomass then changes and the reference's updateLocalMaskNtotalLattices3D (one pass) and
    updateAgeDistance3D (3 sweeps, and to a fixed point or 1000 sweeps) give the expected mask,
    totals and ages."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_vop.so"))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rng = np.random.default_rng(31)
    shape = (9, 7, 6)
    nx, ny, nz = shape
    N = nx * ny * nz
    Bmax, frac = 100.0, 0.3
    codes, pores = np.array([3, 4], np.int32), np.array([2], np.int32)
    rec = {}
    for case in range(5):
        mat = np.where(rng.random(N) < 0.15, 0, 2).astype(np.int8)
        mat[rng.random(N) < 0.05] = 1
        mat[(mat == 2) & (rng.random(N) < 0.45)] = 3
        mat[(mat == 2) & (rng.random(N) < 0.15)] = 4
        bio = np.zeros((2, N))
        bio[0, mat == 3] = rng.uniform(0, Bmax, (mat == 3).sum())
        bio[1, mat == 4] = rng.uniform(0, Bmax, (mat == 4).sum())
        full = (mat >= 3) & (rng.random(N) < 0.5)
        bio[0, full & (mat == 3)] = Bmax
        bio[1, full & (mat == 4)] = Bmax
        O = oracle.OracleAde(mat, *shape, [dict(omega_pore=1.0, c0=0.1)], np.zeros(3 * N), bio_codes=(3, 4))
        O.set_biomass(bio)
        O.ca_setup(Bmax, frac, 7)
        total0, age0 = O.ca_fields()
        flags = O.ca_open_flags()
        bio2 = bio * rng.uniform(0.0, 1.0 if case < 3 else 1.6, bio.shape)
        f2 = (mat >= 3) & (rng.random(N) < 0.6)
        bio2[0, f2 & (mat == 3)] = Bmax
        bio2[1, f2 & (mat == 4)] = Bmax
        bio2[:, rng.random(N) < 0.1] = 0.0
        bio2 = np.ascontiguousarray(bio2)
        total, mask = total0.copy(), mat.astype(np.int32)
        L.ref_ca_mask_total(nx, ny, nz, 2, P(bio2), P(total), P(mask), 1, 0, P(codes), 1, P(pores),
                            C.c_double(frac), C.c_double(Bmax))
        ages = {}
        for k in (3, 1000):
            a = age0.astype(np.int32).copy()
            sw = L.ref_ca_age_relax(nx, ny, nz, P(a), P(flags), P(total), C.c_double(Bmax), k)
            ages[k] = (a, sw)
        for k, v in dict(mat=mat, bio=bio, bio2=bio2, total0=total0, age0=age0, flags=flags, total=total,
                         mask=mask, age3=ages[3][0], age_fix=ages[1000][0],
                         sweeps=np.array([ages[3][1], ages[1000][1]])).items():
            rec[f"{case}_{k}"] = v
    rec["shape"] = np.array(shape)
    rec["prm"] = np.array([Bmax, frac])
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "automaton.npz"), **rec)
    print("wrote 5 automaton cases")


def kinetics_cases():
    """Seeded small fields (rock, walls, pore, biofilm; concentrations with sub-threshold and
    negative entries) through the reference's run_kinetics with the library's decay, Monod and
    dual-Monod laws, and through its run_abiotic_kinetics / surfaceAbioticKinetics3D with the FeS
    precipitation law of examples/15. Some cases have rates that overdraw a voxel, where the
    reference's increment goes below -C."""
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_kinetics.so"))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rng = np.random.default_rng(77)
    shape = (10, 8, 7)
    nx, ny, nz = shape
    N = nx * ny * nz

    def conc(S, scale):
        c = rng.uniform(0, scale, (S, N))
        c[rng.random((S, N)) < 0.05] = 1e-13
        c[rng.random((S, N)) < 0.05] *= -0.1
        return c

    rec = {}
    biotic = ((1, [1e-3, 0.5, 2.0], 0, 1.0, 1.0), (2, [0.3, 0.02, 0.1, 0.5, 0.1, 1e-3], 0, 1.0, 1.0),
              (3, [0.5, 0.2, 0.4, 0.01], 2, 1.0, 1.0), (3, [5.0, 0.2, 0.4, 0.01], 2, 0.5, 0.3))
    for case, (law, prm, M, dt, scale) in enumerate(biotic):
        S = 3
        mat = np.where(rng.random(N) < 0.2, 0, 2).astype(np.int8)
        mat[rng.random(N) < 0.05] = 1
        mat[(mat == 2) & (rng.random(N) < 0.3)] = 3
        Cf = conc(S, scale)
        B = rng.uniform(0, 2, (M, N))
        B[:, rng.random(N) < 0.1] = 0.0
        prm = np.array(prm, np.float64)
        dC, dB = np.zeros((S, N)), np.zeros((max(M, 1), N))
        L.ref_biotic_increments(nx, ny, nz, S, M, C.c_double(dt), law, P(prm), len(prm), P(mat), 0, 1, P(Cf),
                                P(B if M else dB), P(dC), P(dB))
        for k, v in dict(mat=mat, C=Cf, B=B, prm=prm, dC=dC, dB=dB[:M], meta=np.array([law, M, dt])).items():
            rec[f"b{case}_{k}"] = v
    case = 0
    for surf in (0, 1):
        for dt, scale in ((1.0, 0.9), (1.0, 2.0), (0.25, 1.0)):
            S = 4
            mat = np.where(rng.random(N) < 0.25, 0, 2).astype(np.int8)
            mat[rng.random(N) < 0.05] = 1
            Cf = conc(S, scale)
            dC = np.zeros((S, N))
            L.ref_abiotic_increments(nx, ny, nz, S, C.c_double(dt), surf, P(mat), 0, 1, P(Cf), P(dC))
            for k, v in dict(mat=mat, C=Cf, dC=dC, meta=np.array([surf, dt])).items():
                rec[f"a{case}_{k}"] = v
            case += 1
    # the thermodynamic gate: factors of two reaction blocks on seeded concentration vectors, and
    # run_kinetics gated by it (dual Monod, one microbe)
    gates = (([0, 1, 2, 3], [-1.0, -1.0, 1.0, 1.0], [-33.12, 0.25, 50.0, 1.0, 1e-9, 0.0, 277.15, 8.314e-3, 1e-3]),
             ([0, 2], [-1.0, 2.0], [-20.0, 0.5, 45.0, 2.0, 1e-7, 1.5, 298.15, 8.314462618e-3, 1.0]))
    for case, (sp, nu, v) in enumerate(gates):
        sp, nu, v = np.array(sp, np.int32), np.array(nu, np.float64), np.array(v, np.float64)
        S = 4
        L.ref_set_thermo(len(sp), P(sp), P(nu), P(v), 1)
        L.ref_thermo_factor.restype = C.c_double
        cs = 10 ** rng.uniform(-7, 1, (600, S))
        cs[rng.random((600, S)) < 0.08] = 0.0
        F = np.array([L.ref_thermo_factor(S, P(np.ascontiguousarray(c))) for c in cs])
        mat = np.where(rng.random(N) < 0.2, 0, 2).astype(np.int8)
        mat[(mat == 2) & (rng.random(N) < 0.4)] = 3
        Cf = 10 ** rng.uniform(-5, 0.5, (S, N))
        B = rng.uniform(0, 2, (1, N))
        prm = np.array([0.5, 0.2, 0.4, 0.01], np.float64)
        dC, dB = np.zeros((S, N)), np.zeros((1, N))
        L.ref_biotic_increments(nx, ny, nz, S, 1, C.c_double(1.0), 3, P(prm), len(prm), P(mat), 0, 1, P(Cf), P(B),
                                P(dC), P(dB))
        L.ref_set_thermo(0, P(sp), P(nu), P(v), 1)
        for k, val in dict(sp=sp, nu=nu, v=v, cs=cs, F=F, mat=mat, C=Cf, B=B, prm=prm, dC=dC, dB=dB).items():
            rec[f"g{case}_{k}"] = val
    rec["shape"] = np.array(shape)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "kinetics.npz"), **rec)
    print("wrote 4 biotic, 6 abiotic and 2 gated kinetics cases")


def conversion_cases():
    """Seeded small maps with mineral fields at, above and below the sealing density, and stamped
    (previously sealed) voxels above and below the reopening density, through the reference's
    precipNodeConversion3D and, with dissolution on, dissolNodeConversion3D; the precipitate
    code is the solid code or a code of its own."""
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_vop.so"))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rng = np.random.default_rng(8)
    shape, S, sM, full, reopen = (10, 8, 7), 3, 2, 2.0, 0.9
    nx, ny, nz = shape
    N = nx * ny * nz
    rec = {}
    for case in range(6):
        pcode = 0 if case < 4 else 5
        dis = int(case % 2 == 0)
        mat = np.where(rng.random(N) < 0.2, 0, 2).astype(np.int8)
        mat[rng.random(N) < 0.05] = 1
        mat[(mat == 2) & (rng.random(N) < 0.3)] = 3
        if pcode == 5:
            mat[(mat == 0) & (rng.random(N) < 0.3)] = 5
        stamp = ((mat == pcode) & (rng.random(N) < 0.5)).astype(np.uint8)
        Cf = rng.uniform(0, 1, (S, N))
        Cf[sM] = rng.uniform(0, 2.5, N)
        Cf[sM, stamp == 1] = rng.uniform(1.5, 2.1, int((stamp == 1).sum()))
        Cf[sM, rng.random(N) < 0.03] = full  # exactly at the sealing density
        m, st = mat.copy(), stamp.copy()
        L.ref_node_conversion(nx, ny, nz, S, sM, C.c_double(full), C.c_double(reopen), pcode, 2, 0, 1, dis,
                              P(Cf), P(m), P(st))
        for k, v in dict(mat=mat, stamp=stamp, C=Cf, mat_out=m, stamp_out=st,
                         meta=np.array([pcode, dis])).items():
            rec[f"{case}_{k}"] = v
    rec["shape"] = np.array(shape)
    rec["prm"] = np.array([S, sM, full, reopen])
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "conversion.npz"), **rec)
    print("wrote 6 node conversion cases")


def main():
    conversion_cases()
    kinetics_cases()
    ca_cases()
    dissolution_cases()
    speciation_cases()
    L = C.CDLL(REF)
    out = []
    for c in CASES:
        o, arr, ins = ref_generate(L, c)
        rec = dict(options=o, sha256=hashlib.sha256(arr.tobytes()).hexdigest(), inspection=ins)
        if arr.size <= 1000:
            rec["voxels"] = arr.tolist()
        out.append(rec)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "geometry.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} geometry cases")


if __name__ == "__main__":
    main()

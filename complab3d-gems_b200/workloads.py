"""Seeded synthetic workloads of the reactive-transport step (material maps + parameters).

Material numbers follow the reference convention (config/geometry/README.md): 0 solid,
1 bounce-back wall, 2 pore, 3.. biofilm of microbe 0... A grain of a sphere pack is an
impermeable no-slip obstacle, i.e. the reference's bounce-back material (code 1). Every map gets
the two ghost x-planes the reference adds when it reads a geometry (readGeometry duplicates the
first and last slice, complab_functions.hh:178-207), so nx below always counts them.

Relaxation from diffusivity uses the D3Q7 lattice sound speed cs2 = 1/4:
tau = D / cs2 + 1/2 (complab.cpp:1221-1253 in lattice units).
"""
from __future__ import annotations

import numpy as np

CS2_ADE = 0.25

# constants of the library's C ABI used in the workload descriptions (include/clb.h), kept here so
# that building a workload does not load the library
DIRICHLET, NEUMANN = 0, 1
LAW_DECAY, LAW_MONOD, LAW_DUAL_MONOD = 1, 2, 3


def _library_sphere_pack(*args, **kw):
    import clb
    return clb.sphere_pack(*args, **kw)


def add_ghost_planes(inner, nx_inner, ny, nz):
    inner = np.asarray(inner, dtype=np.int8).reshape(nx_inner, ny, nz)
    full = np.empty((nx_inner + 2, ny, nz), dtype=np.int8)
    full[1:-1] = inner
    full[0] = inner[0]
    full[-1] = inner[-1]
    return full.reshape(-1)


def omega_from_d(d):
    return 1.0 / (d / CS2_ADE + 0.5)


def sphere_pack_domain(nx_inner, ny, nz, porosity, rmin, rmax, seed, walls="yz", gen=None):
    """`gen`: the sphere-pack generator (default: the library's clb_geom_sphere_pack; the CPU
    baseline passes the oracle's restatement of it, which gives the same voxels)."""
    gen = gen or _library_sphere_pack
    inner = gen(nx_inner, ny, nz, porosity, rmin, rmax, seed, walls, grain=1, wall=1, pore=2)
    return add_ghost_planes(inner, nx_inner, ny, nz), (nx_inner + 2, ny, nz)


def pack64x32x32_decay(scale=1, gen=None):
    """64x32x32 sphere pack (r = 4, porosity 0.40, walls on the four side faces), tau 0.8,
    dP 1e-4, one solute D_pore 0.1 / D_biofilm 0.05, C = 1 Dirichlet inlet, Neumann outlet,
    first-order decay k = 1e-3 per step, clamped. `scale` < 1 shrinks the box for quick tests."""
    nxi, ny, nz = max(8, int(64 * scale)), max(6, int(32 * scale)), max(6, int(32 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.40, 4.0, 4.0, seed=1001, gen=gen)
    species = [dict(omega_pore=omega_from_d(0.1), omega_biofilm=omega_from_d(0.05), mobile=1,
                    left_type=DIRICHLET, right_type=NEUMANN, left_bc=1.0, c0=0.0)]
    return dict(name="sphere-pack 64x32x32 flow + 1 decaying solute", mat=mat, shape=shape, tau=0.8,
                delta_p=1e-4, eps=1e-6, species=species, law=LAW_DECAY, params=[1e-3], dt=1.0,
                ade_steps=2000)


def pack256x128x128(scale=1, gen=None):
    """256x128x128 overlapping-sphere pack (porosity 0.35, r ~ U[3, 8]), flow only, tau 0.7,
    Peclet rescale (Pe 10, L 8), residual 1e-7."""
    nxi, ny, nz = max(8, int(256 * scale)), max(8, int(128 * scale)), max(8, int(128 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.35, 3.0, 8.0, seed=1002, gen=gen)
    return dict(name="overlapping-sphere pack 256x128x128 flow", mat=mat, shape=shape, tau=0.7, delta_p=1e-4,
                eps=1e-7, peclet=10.0, char_length=8.0, tau_ade_fixed=0.8)


def percolating_pores(mat, shape, open_codes=(2,)):
    """Mask of the open voxels (materials in open_codes) of the interior planes x = 1..nx-2 that
    face-connected open paths inside those planes join to both x = 1 and x = nx-2."""
    from scipy import ndimage

    m = np.isin(mat.reshape(shape), open_codes)
    m[0] = m[-1] = False
    lab, _ = ndimage.label(m)
    keep = np.intersect1d(np.unique(lab[1][lab[1] > 0]), np.unique(lab[-2][lab[-2] > 0]))
    return np.isin(lab, keep).ravel()


def pack256cube_8species(scale=1, seed=1003, gen=None):
    """256^3 sphere pack (porosity 0.40), 8 species with D_pore ~ U[0.02, 0.2] and
    D_biofilm = D_pore / 2, two microbes (materials 3 and 4) seeded on as many voxels as 2 % of the
    pore voxels, drawn from the percolating pore cluster of the interior planes; dual-Monod
    kinetics mu_max 1e-4, Ks 0.1, Y 0.4, decay 1e-6; the biofilm automaton ('fraction' push, max
    density 100, biofilm threshold 0.1 of it) every iteration; the flow (tau 0.8, pressure drop
    1e-4, FP32) solved to 1e-6 first and re-solved every 500 iterations; 10,000 iterations.

    Seeds stay out of pockets the percolating cluster does not reach: the automaton pushes only
    between voxels of x = 1..nx-2 (the reference's bdryGap of 1), so a colony in a pocket with no
    open face neighbour there (a pore at x = 1 walled in by grains except toward the inlet plane)
    cannot shed its excess, or fills the pocket and leaves the age wavefront without a fixed
    point; either ends the reference's run (complab.cpp:3030-3046) as it ends ours."""
    nxi, ny, nz = max(8, int(256 * scale)), max(8, int(256 * scale)), max(8, int(256 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.40, 3.0, 8.0, seed=seed, gen=gen)
    rng = np.random.default_rng(seed)
    pore = np.flatnonzero(mat == 2)
    joined = np.flatnonzero(percolating_pores(mat, shape))
    seeded = rng.choice(joined, size=max(2, min(joined.size, int(0.02 * pore.size))), replace=False)
    seeded.sort()
    half = seeded.size // 2
    mat = mat.copy()
    mat[seeded[:half]] = 3
    mat[seeded[half:]] = 4
    N = mat.size
    bio = np.zeros((2, N))
    bio[0, mat == 3] = 50.0
    bio[1, mat == 4] = 50.0
    d = rng.uniform(0.02, 0.2, size=8)
    species = []
    for k in range(8):
        species.append(dict(omega_pore=omega_from_d(d[k]), omega_biofilm=omega_from_d(0.5 * d[k]), mobile=1,
                            left_type=DIRICHLET if k < 3 else NEUMANN, right_type=NEUMANN,
                            left_bc=1.0 if k < 3 else 0.0, c0=0.1 if k < 3 else 0.0))
    return dict(name="sphere-pack 256^3, 8 species, 2 biofilm microbes", mat=mat, shape=shape, tau=0.8,
                delta_p=1e-4, eps=1e-6, species=species, law=LAW_DUAL_MONOD,
                params=[1e-4, 0.1, 0.4, 1e-6], dt=1.0, biomass=bio, bio_codes=(3, 4), perm_ratio=(0.1, 0.1),
                bmax=100.0, biofilm_fraction=0.1, ca_seed=seed, resolve_every=500, iterations=10000,
                flow_max_iterations=100000)


# Flow iterations per transport iteration of the 256^3 coupled configuration: the re-solves'
# collide-and-stream calls over the configuration's 10,000 iterations, as measured on one B200
# (7,106 flow iterations: the first in-loop re-solve fills the tracer's window, the later ones
# find the flow settled; bench.py's headline reports the run's own figure). The CPU baseline weights
# its flow and transport samples by it so that both arms time the same mix of work.
FLOW_PER_TRANSPORT_CONFIG3 = 0.711


def fracture192_carbonate(gen, scale=1.0, seed=1004):
    """Precipitation with equilibrium chemistry: a 192^3 rough fracture (aperture 12, roughness 0.3;
    `gen(nx_inner, ny, nz)` returns the generator's map, 0 rock and 2 pore), the 5-component
    12-species tableau (tableau_5x12) solved per voxel, species fed at the inlet and initially
    present at log-uniform levels in [1e-6, 1e-4] (H+ dominant so every component total is
    positive), two components supersaturated with an immobile mineral (k 2e-6, log10 Ksp -6) that
    seals a voxel at density 1e-3 (the deposit starts uniform in [0, 1e-3)), flow tau 0.8 at
    pressure drop 1e-4 re-solved every 200 steps."""
    S, logK, comp = tableau_5x12(seed)
    ns = S.shape[0]
    nxi, ny, nz = (max(8, int(192 * scale)),) * 3
    mat = add_ghost_planes(gen(nxi, ny, nz), nxi, ny, nz)
    shape = (nxi + 2, ny, nz)
    rng = np.random.default_rng(seed)
    sp = [dict(omega_pore=1 / 0.9, left_type=DIRICHLET, right_type=NEUMANN, left_bc=float(10 ** rng.uniform(-5, -3.5)),
               c0=float(10 ** rng.uniform(-6, -4))) for _ in range(ns)]
    sp[0]["c0"], sp[0]["left_bc"] = 3e-3, 2e-3
    for s in (1, 2):
        sp[s]["c0"], sp[s]["left_bc"] = 2e-3, 2e-3
    sp.append(dict(omega_pore=1.0, mobile=0, left_type=NEUMANN, right_type=NEUMANN, c0=0.0))
    nu = [0.0] * (ns + 1)
    nu[1], nu[2] = 1.0, 1.0
    full = 1e-3
    m0 = np.random.default_rng(seed + 1).uniform(0.0, full, mat.size) * (mat == 2)
    return dict(name="rough fracture 192^3, 5 components x 12 species, mineral", mat=mat, shape=shape, S=S,
                logK=logK, comp=comp, species=sp, mineral=[2e-6, -6.0, ns] + nu, mineral_species=ns, full=full,
                deposit=m0, tau=0.8, delta_p=1e-4, resolve_every=200)


def ensemble_uneven_packs(n_domains=96, seed=1005, scale=1.0):
    """Ensemble sweep: n_domains independent sphere packs of uneven sizes (inner nx in
    {32, 48, 64, 96}, ny = nz in {24, 32, 48}, drawn from the seeded stream), porosity U[0.3, 0.5],
    grain radius U[2, 4], flow tau U[0.6, 1.0] at pressure drop 1e-4, three species with D_pore
    U[0.05, 0.2] (biofilm half of it), Dirichlet inlet / Neumann outlet, Monod decay with rate
    constants log-uniform in [1e-6, 1e-3] and half-saturation 0.1. FP32. `scale` < 1 shrinks the
    sizes (tests)."""
    rng = np.random.default_rng(seed)
    doms = []
    for d in range(n_domains):
        nxi = int(rng.choice([32, 48, 64, 96]))
        nyz = int(rng.choice([24, 32, 48]))
        nxi, nyz = max(8, int(nxi * scale)), max(6, int(nyz * scale))
        phi = float(rng.uniform(0.3, 0.5))
        mat, shape = sphere_pack_domain(nxi, nyz, nyz, phi, 2.0, 4.0, seed=seed * 1000 + d)
        tau = float(rng.uniform(0.6, 1.0))
        species = []
        for s in range(3):
            dp = float(rng.uniform(0.05, 0.2))
            species.append(dict(omega_pore=omega_from_d(dp), omega_biofilm=omega_from_d(0.5 * dp), mobile=1,
                                left_type=DIRICHLET, right_type=NEUMANN, left_bc=1.0, c0=0.0))
        k = 10.0 ** rng.uniform(-6, -3, size=3)
        doms.append(dict(mat=mat, shape=shape, tau=tau, delta_p=1e-4, species=species, law=LAW_MONOD,
                         params=list(k) + [0.1] * 3, dt=1.0))
    return dict(name=f"ensemble of {n_domains} uneven sphere packs, D3Q19 + 3 x D3Q7 each", domains=doms)


def carbonate_tableau():
    """The two-component carbonate tableau of the reference's equilibrium example
    (examples/04_equilibrium/CompLaB.xml): HCO3 and H are components; CO3 = HCO3 - H
    (log K -10.33), H2CO3 = HCO3 + H (log K 6.35)."""
    S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], dtype=np.float64)
    logK = np.array([0.0, 0.0, -10.33, 6.35])
    return S, logK, [0, 1]


def tableau_5x12(seed=1004):
    """A 5-component, 12-species carbonate-like tableau: species 0..4 are the components
    (component 0 plays H+), species 5..11 complexes of one or two components with an H+
    coefficient in {-1, 0, 1}; log K drawn uniformly from [-12, 2] with a seeded generator."""
    rng = np.random.default_rng(seed)
    S = np.zeros((12, 5))
    S[:5, :5] = np.eye(5)
    logK = np.zeros(12)
    for k in range(5, 12):
        p = rng.integers(1, 5)
        S[k, p] = 1.0
        if rng.random() < 0.5:
            q = rng.integers(1, 5)
            if q != p:
                S[k, q] = 1.0
        S[k, 0] = float(rng.integers(-1, 2))
        logK[k] = rng.uniform(-12.0, 2.0)
    return S, logK, [0, 1, 2, 3, 4]


def species_states(n, ns, lo, hi, seed):
    """n species states with log10 c uniform in [lo, hi] per species."""
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(lo, hi, size=(n, ns))

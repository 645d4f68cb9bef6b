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

import clb

CS2_ADE = 0.25


def add_ghost_planes(inner, nx_inner, ny, nz):
    inner = np.asarray(inner, dtype=np.int8).reshape(nx_inner, ny, nz)
    full = np.empty((nx_inner + 2, ny, nz), dtype=np.int8)
    full[1:-1] = inner
    full[0] = inner[0]
    full[-1] = inner[-1]
    return full.reshape(-1)


def omega_from_d(d):
    return 1.0 / (d / CS2_ADE + 0.5)


def sphere_pack_domain(nx_inner, ny, nz, porosity, rmin, rmax, seed, walls="yz"):
    inner = clb.sphere_pack(nx_inner, ny, nz, porosity, rmin, rmax, seed, walls, grain=1, wall=1, pore=2)
    return add_ghost_planes(inner, nx_inner, ny, nz), (nx_inner + 2, ny, nz)


def config1(scale=1):
    """64x32x32 sphere pack (r = 4, porosity 0.40, walls on the four side faces), tau 0.8,
    dP 1e-4, one solute D_pore 0.1 / D_biofilm 0.05, C = 1 Dirichlet inlet, Neumann outlet,
    first-order decay k = 1e-3 per step, clamped. `scale` < 1 shrinks the box for quick tests."""
    nxi, ny, nz = max(8, int(64 * scale)), max(6, int(32 * scale)), max(6, int(32 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.40, 4.0, 4.0, seed=1001)
    species = [dict(omega_pore=omega_from_d(0.1), omega_biofilm=omega_from_d(0.05), mobile=1,
                    left_type=clb.DIRICHLET, right_type=clb.NEUMANN, left_bc=1.0, c0=0.0)]
    return dict(name="sphere-pack 64x32x32 flow + 1 decaying solute", mat=mat, shape=shape, tau=0.8,
                delta_p=1e-4, eps=1e-6, species=species, law=clb.LAW_DECAY, params=[1e-3], dt=1.0,
                ade_steps=2000)


def config2(scale=1):
    """256x128x128 overlapping-sphere pack (porosity 0.35, r ~ U[3, 8]), flow only, tau 0.7,
    Peclet rescale (Pe 10, L 8), residual 1e-7."""
    nxi, ny, nz = max(8, int(256 * scale)), max(8, int(128 * scale)), max(8, int(128 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.35, 3.0, 8.0, seed=1002)
    return dict(name="overlapping-sphere pack 256x128x128 flow", mat=mat, shape=shape, tau=0.7, delta_p=1e-4,
                eps=1e-7, peclet=10.0, char_length=8.0, tau_ade_fixed=0.8)


def config3(scale=1, seed=1003):
    """256^3 sphere pack (porosity 0.40), 8 species with D_pore ~ U[0.02, 0.2] and
    D_biofilm = D_pore / 2, two microbes (materials 3 and 4) seeded on 2 % of pore voxels,
    dual-Monod kinetics mu_max 1e-4, Ks 0.1, Y 0.4, decay 1e-6."""
    nxi, ny, nz = max(8, int(256 * scale)), max(8, int(256 * scale)), max(8, int(256 * scale))
    mat, shape = sphere_pack_domain(nxi, ny, nz, 0.40, 3.0, 8.0, seed=seed)
    rng = np.random.default_rng(seed)
    pore = np.flatnonzero(mat == 2)
    seeded = rng.choice(pore, size=max(2, int(0.02 * pore.size)), replace=False)
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
                            left_type=clb.DIRICHLET if k < 3 else clb.NEUMANN, right_type=clb.NEUMANN,
                            left_bc=1.0 if k < 3 else 0.0, c0=0.1 if k < 3 else 0.0))
    return dict(name="sphere-pack 256^3, 8 species, 2 biofilm microbes", mat=mat, shape=shape, tau=0.8,
                delta_p=1e-4, eps=1e-6, species=species, law=clb.LAW_DUAL_MONOD,
                params=[1e-4, 0.1, 0.4, 1e-6], dt=1.0, biomass=bio, bio_codes=(3, 4), perm_ratio=(0.1, 0.1),
                bmax=100.0)

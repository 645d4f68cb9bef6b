"""clb_reduce_noalloc (reductions from the library's fixed per-device buffer, no allocation)
against clb_reduce on the same live fields, two calls in a row.

Both entry points run the same fixed-order reduction tree (warp shuffles, then warps and blocks in
a fixed order, no atomics), so their results are the same bits, call after call; only the scratch
they use differs. This file is named to be collected last, so the entry point is also exercised
after every other GPU test has used the device."""
import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

SPECIES = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=1.0, c0=0.0),
    dict(omega_pore=1 / 0.62, omega_biofilm=1 / 0.56, left_type=1, right_type=0, right_bc=0.4, c0=0.2),
    dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.8),
]


def make_domain(clb, prec):
    shape = (18, 11, 10)
    mat = mixed_geometry(*shape, seed=11)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=prec, bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
    D.ade_init(SPECIES)
    rng = np.random.default_rng(7)
    u = np.zeros((3, D.N))
    u[0] = rng.uniform(0.0, 0.02, D.N)
    D.set_velocity(u)
    b = np.zeros((2, D.N))
    b[0, mat == 3] = 40.0
    b[1, mat == 4] = 25.0
    D.set_biomass(b)
    D.set_kinetics(2, [1e-2, 3e-2, 1e-3, 0.1, 0.2, 0.5], 1.0)
    return D


def assert_same(a, b):
    for key in ("total", "content", "biomass", "min", "max"):
        assert a[key].tobytes() == b[key].tobytes(), key
    for key in ("open_voxels", "nonfinite", "ade_iterations"):
        assert a[key] == b[key], key


@pytest.mark.parametrize("prec", ["F64", "F32", "F16S"])
def test_noalloc_reduce_matches_reduce_twice_in_a_row(clb, prec):
    D = make_domain(clb, getattr(clb, prec))
    D.ade_step(37)
    ref = D.reduce()
    first = D.reduce_noalloc()
    second = D.reduce_noalloc()
    assert ref["open_voxels"] > 0 and ref["total"][0] > 0
    assert_same(first, ref)
    assert_same(second, ref)
    # the buffer carries nothing over: after more steps the result follows the new fields
    D.ade_step(5)
    ref = D.reduce()
    assert_same(D.reduce_noalloc(), ref)
    assert_same(D.reduce_noalloc(), ref)

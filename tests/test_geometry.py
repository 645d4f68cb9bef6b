"""Geometry generators and inspection against the reference's own generator.

The golden file was produced by complab3d_geometry.hh itself (tests/golden/make_golden.py);
these tests run the product's host code through the C ABI (no GPU needed)."""
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "geometry.json")))


@pytest.mark.parametrize("case", GOLD, ids=[f"{c['options']['kind']}-{i}" for i, c in enumerate(GOLD)])
def test_generator_bit_exact(clb, case):
    o = case["options"]
    arr = clb.geom_generate(o["kind"], o["nx"], o["ny"], o["nz"], porosity=o["porosity"], radius=o["radius"],
                            aperture=o["aperture"], roughness=o["roughness"], count=o["count"],
                            layers=o["layers"], seed=o["seed"], walls=o["walls"])
    if "voxels" in case:
        assert arr.tolist() == case["voxels"]
    assert hashlib.sha256(arr.tobytes()).hexdigest() == case["sha256"]


@pytest.mark.parametrize("case", GOLD, ids=[f"{c['options']['kind']}-{i}" for i, c in enumerate(GOLD)])
def test_inspection_matches_reference(clb, case):
    o = case["options"]
    arr = clb.geom_generate(o["kind"], o["nx"], o["ny"], o["nz"], porosity=o["porosity"], radius=o["radius"],
                            aperture=o["aperture"], roughness=o["roughness"], count=o["count"],
                            layers=o["layers"], seed=o["seed"], walls=o["walls"])
    r = clb.inspect(arr, o["nx"], o["ny"], o["nz"])
    ref = case["inspection"]
    assert r["porosity"] == pytest.approx(ref["porosity"], abs=0)
    for k in ("open_voxels", "isolated_voxels", "clusters", "spanning_clusters", "percolates"):
        assert r[k] == ref[k], k


def test_unknown_kind_is_an_error(clb):
    with pytest.raises(clb.ClbError):
        clb.geom_generate("voronoi", 4, 4, 4)


def test_read_dat_duplicates_ghost_planes(clb, tmp_path):
    nxi, ny, nz = 5, 3, 4
    rng = np.random.default_rng(0)
    inner = rng.integers(0, 4, size=(nxi, ny, nz)).astype(np.int8)
    p = tmp_path / "g.dat"
    p.write_text("\n".join(str(v) for v in inner.ravel()) + "\n")
    full = clb.read_dat(str(p), nxi, ny, nz).reshape(nxi + 2, ny, nz)
    assert np.array_equal(full[1:-1], inner)
    assert np.array_equal(full[0], inner[0]) and np.array_equal(full[-1], inner[-1])


def test_read_dat_short_file_is_an_error(clb, tmp_path):
    p = tmp_path / "g.dat"
    p.write_text("2 2 2\n")
    with pytest.raises(clb.ClbError):
        clb.read_dat(str(p), 2, 2, 2)


@pytest.mark.parametrize("phi,rmin,rmax", [(0.40, 4, 4), (0.35, 3, 8)])
def test_sphere_pack_hits_porosity_and_is_seeded(clb, phi, rmin, rmax):
    n = (40, 24, 24)
    a = clb.sphere_pack(*n, phi, rmin, rmax, 77, "yz")
    b = clb.sphere_pack(*n, phi, rmin, rmax, 77, "yz")
    c = clb.sphere_pack(*n, phi, rmin, rmax, 78, "yz")
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    por = np.mean(a == 2)
    assert phi - 0.02 < por <= phi
    g = a.reshape(n)
    assert np.all(g[:, 0, :] == 1) and np.all(g[:, :, -1] == 1)
    assert clb.inspect(a, *n)["percolates"] == 1


def test_oracle_sphere_pack_equals_the_library(clb, oracle):
    """The oracle's restatement of the sphere pack (the CPU baseline's input maps) is the
    library's generator voxel for voxel."""
    for args in ((40, 24, 20, 0.40, 4.0, 4.0, 1001, "yz"), (30, 17, 19, 0.35, 3.0, 8.0, 1002, "y"),
                 (25, 25, 25, 0.6, 2.0, 5.5, 7, "all")):
        np.testing.assert_array_equal(clb.sphere_pack(*args), oracle.sphere_pack(*args))

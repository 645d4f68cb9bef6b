"""clb_write_vti on a domain: the files hold the interior planes of what clb_get_field returns."""
import os

import numpy as np
import pytest

from helpers import mixed_geometry
from test_vti import read_vti

pytestmark = pytest.mark.gpu


def interior(a, shape, comps=1):
    nx, ny, nz = shape
    a = np.asarray(a).reshape(comps, nx, ny, nz)[:, 1:-1]
    return a.transpose(3, 2, 1, 0).reshape(-1)


def test_domain_fields_to_vti(clb, tmp_path):
    shape = (14, 9, 8)
    mat = mixed_geometry(*shape, seed=5)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F32, ade_precision=clb.F64, bio_codes=(3, 4),
                   perm_ratio=(0.3, 0.3))
    D.flow_init(3e-4)
    D.flow_step(50)
    D.ade_init([dict(omega_pore=1 / 0.9, left_type=clb.DIRICHLET, right_type=clb.NEUMANN, left_bc=1.0, c0=0.1)])
    D.couple_velocity()
    D.ade_step(20)
    p = lambda n: os.path.join(tmp_path, n)
    D.write_vti(clb.FIELD_FLOW_VELOCITY, p("ns_0000050.vti"))
    D.write_vti(clb.FIELD_MATERIAL, p("geom.vti"))
    D.write_vti(clb.FIELD_CONCENTRATION, p("c0_0000020.vti"), index=0)
    u = D.velocity().reshape(3, -1)
    dims, arr = read_vti(p("ns_0000050.vti"))
    assert dims == (shape[0] - 2, shape[1], shape[2])
    np.testing.assert_array_equal(arr["velocity"][0], interior(u.astype(np.float32), shape, 3))
    norm = np.sqrt((u ** 2).sum(0)).astype(np.float32)
    np.testing.assert_allclose(arr["velocityNorm"][0], interior(norm, shape), rtol=1e-6, atol=0)
    _, arr = read_vti(p("geom.vti"))
    np.testing.assert_array_equal(arr["tag"][0], interior(D.material().astype(np.float32), shape))
    _, arr = read_vti(p("c0_0000020.vti"))
    assert arr["Density"][2] == "Float64"
    np.testing.assert_array_equal(arr["Density"][0], interior(D.concentration(0), shape))
    with pytest.raises(clb.ClbError):
        D.write_vti(clb.FIELD_CA_AGE, p("x.vti"))

"""The oracle pinned to the reference's closed-form duct answers (golden vectors of
ABC_sweep_package/tools/analytic_channel.py ade_1d, tests/golden/channel.json): at Pe = 0 the
steady cross-section means of A - B, A + C and B + C of the A + B -> C duct are its straight
lines to round-off, and each combination equals the unreacting tracer fed with its boundary
values."""
import numpy as np

import channel_case as cc


def test_oracle_pe0_straight_lines(oracle):
    u = cc.velocity(0.0)
    O = oracle.OracleAde(cc.material(), cc.NX, cc.NY, cc.NZ, cc.species(), u)
    O.set_abiotic(4, cc.ABIOTIC, 0)
    O.step(300)
    c = [O.concentration(s) for s in range(6)]
    for k, (name, field) in enumerate(cc.combinations(c).items()):
        np.testing.assert_allclose(field, c[3 + k], rtol=0, atol=1e-13, err_msg=name)
    O.step(15700)
    c = [O.concentration(s) for s in range(6)]
    for name, field in cc.combinations(c).items():
        err = np.max(np.abs(cc.cross_section_mean(field) - cc.golden(0.0, name)))
        assert err < 1e-11, (name, err)

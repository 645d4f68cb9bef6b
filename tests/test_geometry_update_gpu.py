"""Precipitation sealing, dissolution and reopening on the GPU against the FP64 oracle.

Scenarios follow the reference's examples 13 (A + B -> P(s) at the grain surface, voxels seal at
max_precipRho) and 15 (the same plus first-order acid dissolution of the sealed precipitate with
reopening below reopen_fraction x full), a saturation-index (Omega) mineral law, and the flow
re-solve around sealed voxels. Populations of every node, the material map and the mineral field
are compared after each update interval; FP64 parity is 1e-12 absolute."""
import numpy as np
import pytest

from helpers import mixed_geometry

pytestmark = pytest.mark.gpu

BIO = dict(bio_codes=(3, 4), perm_ratio=(0.3, 0.3))
ATOL = 1e-12


def flow_field(oracle, mat, shape, steps=300):
    O = oracle.OracleFlow(mat, *shape, 0.8, 3e-4, **BIO)
    O.step(steps)
    return O.velocity()


def pair(clb, oracle, mat, shape, species, u, prec=None):
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64 if prec is None else prec, **BIO)
    D.ade_init(species)
    D.set_velocity(u)
    O = oracle.OracleAde(mat, *shape, species, u, bio_codes=(3, 4))
    return D, O


def compare(D, O, species, atol=ATOL):
    np.testing.assert_array_equal(D.material(), O.material())
    for s, sp in enumerate(species):
        if sp.get("mobile", 1):
            np.testing.assert_allclose(D.ade_populations(s), O.populations(s), rtol=0, atol=atol, err_msg=f"species {s}")
        else:
            np.testing.assert_allclose(D.concentration(s), O.concentration(s), rtol=1e-12, atol=atol,
                                       err_msg=f"species {s}")


A_B_P = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=0, right_type=1, left_bc=1.0, c0=0.5),
    dict(omega_pore=1 / 0.7, omega_biofilm=1 / 0.65, left_type=1, right_type=0, right_bc=1.0, c0=0.4),
    dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0),
]


@pytest.mark.parametrize("surface_only", [1, 0])
def test_precipitation_seals_like_the_oracle(clb, oracle, surface_only):
    shape = (22, 11, 10)
    mat = mixed_geometry(*shape, seed=21)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, A_B_P, u)
    D.set_abiotic_kinetics(clb.LAW_PRECIP, [0.8, 0, 1, 2], surface_only)
    O.set_abiotic(4, [0.8, 0, 1, 2], surface_only)
    D.precip_setup(2, 0.12)
    O.set_precip(2, 0.12, precip_code=0)
    total_sealed = 0
    for rnd in range(4):
        D.ade_step(25)
        O.step(25)
        a = D.geometry_update()
        b = O.geometry_update()
        assert a == b, (rnd, a, b)
        total_sealed += a[0]
        compare(D, O, A_B_P)
    assert total_sealed > 0


A_B_H_P = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=0, right_type=1, left_bc=1.0, c0=0.5),
    dict(omega_pore=1 / 0.7, omega_biofilm=1 / 0.65, left_type=1, right_type=0, right_bc=1.0, c0=0.4),
    dict(omega_pore=1 / 0.8, omega_biofilm=1 / 0.75, left_type=0, right_type=1, left_bc=0.6, c0=0.2),
    dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0),
]


def test_precipitation_dissolution_cycle_like_the_oracle(clb, oracle):
    """Example 15: FeS precipitates from Fe + HS, acid dissolves the sealed precipitate back into
    Fe and HS (parked per open face, gathered by the water), and voxels reopen below 0.9 full."""
    shape = (22, 11, 10)
    mat = mixed_geometry(*shape, seed=22)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, A_B_H_P, u)
    kp, kd = 0.1, 2.0
    sigma = [1.0, 1.0, -1.0, 0.0]
    D.set_abiotic_kinetics(clb.LAW_PRECIP, [kp, 0, 1, 3], 1)
    O.set_abiotic(4, [kp, 0, 1, 3], 1)
    D.precip_setup(3, 0.1, dissolution=1, reopen_fraction=0.9, dissolution_law=clb.DISSOL_FIRST_ORDER,
                   dissolution_params=[kd, 2] + sigma)
    O.set_precip(3, 0.1, precip_code=0, dissolution=1, reopen=0.9, pore_code=2, dis_law=1,
                 dis_params=[kd, 2] + sigma)
    sealed = reopened = 0
    for rnd in range(8):
        D.ade_step(15)
        O.step(15)
        a = D.geometry_update()
        b = O.geometry_update()
        assert a == b, (rnd, a, b)
        sealed += a[0]
        reopened += a[1]
        compare(D, O, A_B_H_P)
    print("sealed", sealed, "reopened", reopened)
    assert sealed > 0 and reopened > 0


CA_CO3_M = [
    dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=0, right_type=1, left_bc=0.4, c0=0.1),
    dict(omega_pore=1 / 0.75, omega_biofilm=1 / 0.7, left_type=0, right_type=1, left_bc=0.3, c0=0.05),
    dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.02),
]


def test_saturation_index_mineral_law_like_the_oracle(clb, oracle):
    """R_M = k (Omega - 1), Omega = Ca CO3 / Ksp: precipitation where supersaturated, dissolution
    (clamped at the mineral present) where undersaturated, then sealing, then dissolution of the
    sealed mineral by the same saturation law from its water."""
    shape = (20, 10, 9)
    mat = mixed_geometry(*shape, seed=23)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, CA_CO3_M, u)
    prm = [2e-3, np.log10(0.01), 2, 1.0, 1.0, 0.0]
    D.set_abiotic_kinetics(clb.LAW_MINERAL, prm, 0)
    O.set_abiotic(5, prm, 0)
    dis = [5e-3, np.log10(0.01), 1.0, 1.0, 0.0]
    D.precip_setup(2, 0.06, dissolution=1, reopen_fraction=0.9, dissolution_law=clb.DISSOL_MINERAL,
                   dissolution_params=dis)
    O.set_precip(2, 0.06, precip_code=0, dissolution=1, reopen=0.9, pore_code=2, dis_law=2, dis_params=dis)
    sealed = 0
    for rnd in range(5):
        D.ade_step(20)
        O.step(20)
        a = D.geometry_update()
        b = O.geometry_update()
        assert a == b, (rnd, a, b)
        sealed += a[0]
        compare(D, O, CA_CO3_M)
    assert sealed > 0


def test_sealed_flow_resolve_like_the_oracle(clb, oracle):
    """seal_flow: sealed voxels become bounce-back on the flow lattice and the flow is re-solved
    (here a fixed number of steps), then coupled into the species again."""
    shape = (20, 10, 9)
    mat = mixed_geometry(*shape, seed=24)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64, ade_precision=clb.F64, **BIO)
    D.flow_init(3e-4)
    D.flow_step(200)
    OF = oracle.OracleFlow(mat, *shape, 0.8, 3e-4, **BIO)
    OF.step(200)
    D.ade_init(A_B_P)
    D.couple_velocity()
    u = OF.velocity()
    O = oracle.OracleAde(mat, *shape, A_B_P, u, bio_codes=(3, 4))
    D.set_abiotic_kinetics(clb.LAW_PRECIP, [0.8, 0, 1, 2], 1)
    O.set_abiotic(4, [0.8, 0, 1, 2], 1)
    D.precip_setup(2, 0.12, seal_flow=1, flow_max_iterations=60, flow_eps=0.0)
    O.set_precip(2, 0.12, precip_code=0)
    OF.set_dynamics(127, 0, 0.0)  # bounce-back
    for rnd in range(3):
        D.ade_step(30)
        O.step(30)
        a = D.geometry_update(allow_unconverged=True)
        b = O.geometry_update()
        assert a == b
        if a[0] or a[1]:
            fm = mat.copy()
            fm[(O.material() == 0) & (mat != 0)] = 127  # sealed voxels: bounce-back on the flow lattice
            OF.set_material(fm)
            OF.step(60)
            O.set_velocity(OF.velocity())
        np.testing.assert_allclose(D.flow_populations(), OF.populations(), rtol=0, atol=ATOL)
        np.testing.assert_allclose(D.velocity(), OF.velocity(), rtol=0, atol=ATOL)


def test_closed_box_mass_balance_with_sealing(clb):
    """Closed faces, no flow: A + B -> P conserves A's content plus the precipitate, and so does
    sealing (a sealed voxel keeps its populations)."""
    shape = (16, 10, 9)
    mat = mixed_geometry(*shape, seed=25)
    sp = [dict(omega_pore=1 / 0.9, omega_biofilm=1 / 0.8, left_type=2, right_type=2, c0=0.5),
          dict(omega_pore=1 / 0.8, omega_biofilm=1 / 0.7, left_type=2, right_type=2, c0=0.4),
          dict(omega_pore=1.0, mobile=0, left_type=1, right_type=1, c0=0.0)]
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, **BIO)
    D.ade_init(sp)
    D.set_abiotic_kinetics(clb.LAW_PRECIP, [0.3, 0, 1, 2], 0)
    D.precip_setup(2, 0.15)

    def balance():
        r = D.reduce()
        return r["content"][0] + D.concentration(2).sum(), r["content"][1] + D.concentration(2).sum()

    b0 = balance()
    sealed = 0
    for _ in range(5):
        D.ade_step(20)
        sealed += D.geometry_update()[0]
    b1 = balance()
    assert sealed > 0
    for x0, x1 in zip(b0, b1):
        assert abs(x1 - x0) <= 1e-11 * abs(x0), (x0, x1)


def test_reduced_precision_with_dissolution(clb, oracle):
    shape = (22, 11, 10)
    mat = mixed_geometry(*shape, seed=22)
    u = flow_field(oracle, mat, shape)
    D, O = pair(clb, oracle, mat, shape, A_B_H_P, u, prec=clb.F32)
    sigma = [1.0, 1.0, -1.0, 0.0]
    D.set_abiotic_kinetics(clb.LAW_PRECIP, [0.1, 0, 1, 3], 1)
    O.set_abiotic(4, [0.1, 0, 1, 3], 1)
    D.precip_setup(3, 0.1, dissolution=1, dissolution_law=clb.DISSOL_FIRST_ORDER, dissolution_params=[2.0, 2] + sigma)
    O.set_precip(3, 0.1, precip_code=0, dissolution=1, reopen=0.9, pore_code=2, dis_law=1, dis_params=[2.0, 2] + sigma)
    D.ade_step(40)
    O.step(40)
    for s in range(3):
        c, co = D.concentration(s), O.concentration(s)
        err = np.linalg.norm(c - co) / np.linalg.norm(co)
        assert err < 1e-4, (s, err)


def test_precip_setup_errors(clb):
    shape = (10, 6, 6)
    mat = mixed_geometry(*shape, seed=26)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64, **BIO)
    D.ade_init(A_B_P)
    with pytest.raises(clb.ClbError):
        D.precip_setup(0, 0.1)          # a mobile species cannot be the mineral
    with pytest.raises(clb.ClbError):
        D.precip_setup(2, 0.0)          # full density must be positive
    with pytest.raises(clb.ClbError):
        D.precip_setup(2, 0.1, precip_code=2)  # sealed voxels must bounce back
    with pytest.raises(clb.ClbError):
        D.set_abiotic_kinetics(clb.LAW_PRECIP, [1.0, 0, 7, 2])

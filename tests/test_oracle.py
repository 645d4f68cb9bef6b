"""Invariants that pin the FP64 oracle (the reference's only pinned facts for the LBM path:
mass conservation in a closed box, D3Q7 deposit weights summing to one, the steady linear
profile of pure diffusion between two Dirichlet planes, Poiseuille symmetry)."""
import numpy as np
import pytest


def duct(nx, ny, nz):
    m = np.full((nx, ny, nz), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    return m


def test_closed_box_conserves_content_to_roundoff(oracle):
    nx, ny, nz = 20, 10, 9
    m = duct(nx, ny, nz)
    m[8:12, 3:6, 3:6] = 1  # an obstacle held by bounce-back
    F = oracle.OracleFlow(m.ravel(), nx, ny, nz, tau=0.8, delta_p=2e-4)
    F.step(300)
    u = F.velocity()
    sp = [dict(omega_pore=1 / 0.9, left_type=2, right_type=2, c0=0.37)]
    A = oracle.OracleAde(m.ravel(), nx, ny, nz, sp, u)
    c0 = A.populations(0).sum()
    A.step(500)
    assert abs(A.populations(0).sum() - c0) < 1e-11 * abs(c0) * 1e3


def test_poiseuille_profile_is_symmetric_and_positive(oracle):
    nx, ny, nz = 24, 11, 11
    F = oracle.OracleFlow(duct(nx, ny, nz).ravel(), nx, ny, nz, tau=0.8, delta_p=1e-4)
    it = F.solve(30000, 1e-7)
    assert it < 30000
    u = F.velocity().reshape(3, nx, ny, nz)
    prof = u[0, nx // 2, ny // 2, 1:-1]
    assert np.all(prof > 0)
    np.testing.assert_allclose(prof, prof[::-1], rtol=1e-9)
    assert np.max(np.abs(u[1:, 1:-1])) < 1e-3 * np.max(u[0])


def test_pure_diffusion_steady_profile_is_linear(oracle):
    nx, ny, nz = 22, 5, 5
    m = np.full((nx, ny, nz), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    sp = [dict(omega_pore=1.0, left_type=0, right_type=0, left_bc=1.0, right_bc=0.0, c0=0.0)]
    A = oracle.OracleAde(m.ravel(), nx, ny, nz, sp, np.zeros(3 * m.size))
    A.step(30000)
    c = A.concentration(0).reshape(nx, ny, nz)[:, 2, 2]
    slope = np.diff(c[1:-1])
    assert np.all(slope < 0)
    np.testing.assert_allclose(slope, slope.mean(), rtol=1e-6)


def test_decay_deposit_removes_exactly_dc(oracle):
    # one step of decay in a uniform closed box removes k*C*dt per open voxel
    nx, ny, nz = 8, 5, 5
    m = duct(nx, ny, nz)
    sp = [dict(omega_pore=1.2, left_type=2, right_type=2, c0=0.5)]
    A = oracle.OracleAde(m.ravel(), nx, ny, nz, sp, np.zeros(3 * m.size))
    A.set_kinetics(1, [1e-2], 1.0)
    before = A.populations(0).sum()
    A.step(1)
    n_react = np.sum(m[1:-1] == 2)
    assert A.populations(0).sum() - before == pytest.approx(-1e-2 * 0.5 * n_react, rel=1e-12)


def test_clamp_never_drives_concentration_negative(oracle):
    nx, ny, nz = 8, 5, 5
    m = duct(nx, ny, nz)
    sp = [dict(omega_pore=1.2, left_type=2, right_type=2, c0=0.5)]
    A = oracle.OracleAde(m.ravel(), nx, ny, nz, sp, np.zeros(3 * m.size))
    A.set_kinetics(1, [5.0], 1.0)  # R dt = -2.5 C: the clamp binds
    A.step(1)
    c = A.concentration(0).reshape(nx, ny, nz)
    assert np.all(c[1:-1][m[1:-1] == 2] >= -1e-15)

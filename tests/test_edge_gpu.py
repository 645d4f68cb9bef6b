"""Edge cases of the compacted layout and the steps on the GPU against the FP64 oracle: thin and
ragged domains (one voxel thick, nz not a multiple of 32), a node count just past one 256-node
tile, and a domain with no fluid node at all."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SP = [dict(omega_pore=1 / 0.9, left_type=0, right_type=1, left_bc=1.0, c0=0.1),
      dict(omega_pore=1 / 0.7, left_type=1, right_type=2, c0=0.4)]


def random_map(shape, seed, p_wall=0.25):
    rng = np.random.default_rng(seed)
    m = np.where(rng.random(shape) < p_wall, 1, 2).astype(np.int8)
    m[0] = m[1]   # ghost planes duplicate their neighbours
    m[-1] = m[-2]
    return m.ravel()


SHAPES = [((9, 1, 5), 0.25), ((6, 3, 1), 0.25), ((11, 2, 37), 0.3), ((5, 7, 33), 0.2), ((4, 8, 9), 0.0)]


@pytest.mark.parametrize("shape,p_wall", SHAPES, ids=[str(s) for s, _ in SHAPES])
@pytest.mark.parametrize("steps", [1, 9])
def test_flow_populations_match_oracle(clb, oracle, shape, p_wall, steps):
    mat = random_map(shape, sum(shape), p_wall)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64)
    D.flow_init(3e-4)
    D.flow_step(steps)
    O = oracle.OracleFlow(mat, *shape, 0.8, 3e-4)
    O.step(steps)
    fg, fo = D.flow_populations(), O.populations()
    assert np.max(np.abs(fg - fo)) <= 1e-11 * np.max(np.abs(fo))
    D.close()


@pytest.mark.parametrize("shape,p_wall", SHAPES, ids=[str(s) for s, _ in SHAPES])
def test_transport_matches_oracle(clb, oracle, shape, p_wall):
    mat = random_map(shape, 3 * sum(shape), p_wall)
    N = mat.size
    rng = np.random.default_rng(4)
    u = np.zeros((3, N))
    u[0] = rng.uniform(0.0, 0.02, N)
    D = clb.Domain(mat, *shape, 0.8, ade_precision=clb.F64)
    D.ade_init(SP)
    D.set_velocity(u)
    O = oracle.OracleAde(mat, *shape, SP, u)
    D.ade_step(9)
    O.step(9)
    for s in range(len(SP)):
        np.testing.assert_allclose(D.ade_populations(s), O.populations(s), rtol=0, atol=1e-12)
    D.close()


def test_domain_without_fluid_steps_as_a_no_op(clb):
    shape = (6, 5, 4)
    mat = np.full(int(np.prod(shape)), 1, np.int8)  # every voxel a bounce-back wall
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F32, ade_precision=clb.F32)
    D.flow_init(1e-4)
    D.flow_step(4)
    assert np.all(D.velocity() == 0.0)
    st = D.flow_stats()
    assert st["active_nodes"] == 0
    D.ade_init(SP)
    D.couple_velocity()
    D.ade_step(3)
    r = D.reduce()
    assert r["open_voxels"] == 0 and r["nonfinite"] == 0
    D.close()

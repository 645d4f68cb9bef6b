"""D3Q19 flow lattice on the GPU (through the C ABI) against the FP64 oracle.

Tolerances: FP64 storage must match to round-off (relative max 1e-11 on every population);
FP32 storage within 1e-5 relative L2 of the velocity; FP16-shifted within 3e-2 (its
populations carry 11 significant bits)."""
import numpy as np
import pytest

from helpers import mixed_geometry, rel_l2

pytestmark = pytest.mark.gpu

BIO = dict(bio_codes=(3, 4), perm_ratio=(0.3, 0.0))


# kernel variants of the two AA half-steps: (even step through bulk-copied tiles, odd step
# pipelined through shared memory)
VARIANTS = {"tma": (1, 0), "plain": (0, 0), "pipe": (1, 1)}


def make_pair(clb, oracle, mat, shape, tau, dp, prec, even_tma=1, odd_pipe=0, **bio):
    nx, ny, nz = shape
    D = clb.Domain(mat, nx, ny, nz, tau, flow_precision=prec, **bio)
    D.tune("flow_even_tma", even_tma)
    D.tune("flow_odd_pipe", odd_pipe)
    D.flow_init(dp)
    O = oracle.OracleFlow(mat, nx, ny, nz, tau, dp, bio_codes=bio.get("bio_codes", ()),
                          perm_ratio=bio.get("perm_ratio", ()))
    return D, O


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("shape", [(18, 11, 9), (12, 7, 45), (40, 21, 33)])
@pytest.mark.parametrize("walls", [True, False])
@pytest.mark.parametrize("steps", [1, 2, 37, 200])
def test_f64_populations_match_oracle(clb, oracle, shape, walls, steps, variant):
    mat = mixed_geometry(*shape, walls=walls)
    tma, pipe = VARIANTS[variant]
    D, O = make_pair(clb, oracle, mat, shape, 0.8, 3e-4, clb.F64, even_tma=tma, odd_pipe=pipe, **BIO)
    D.flow_step(steps)
    O.step(steps)
    fg, fo = D.flow_populations(), O.populations()
    scale = np.max(np.abs(fo))
    assert np.max(np.abs(fg - fo)) <= 1e-11 * scale
    np.testing.assert_allclose(D.velocity(), O.velocity(), rtol=0, atol=1e-12 * np.max(np.abs(O.velocity())))


def test_f64_solve_matches_oracle_iterations(clb, oracle):
    shape = (22, 12, 12)
    mat = mixed_geometry(*shape, solid_block=False, biofilm=False)
    D, O = make_pair(clb, oracle, mat, shape, 0.8, 1e-4, clb.F64)
    it_g, conv = D.flow_solve(40000, 1e-6)
    it_o = O.solve(40000, 1e-6)
    assert conv
    assert abs(it_g - it_o) <= 1
    assert rel_l2(D.velocity(), O.velocity()) < 1e-9
    st = D.flow_stats(8.0)
    assert st["permeability"] > 0


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("prec,tol", [("F32", 1e-5), ("F16S", 3e-2)])
def test_reduced_precision_velocity_error(clb, oracle, prec, tol, variant):
    shape = (26, 14, 14)
    mat = mixed_geometry(*shape, seed=9)
    tma, pipe = VARIANTS[variant]
    # FP16 storage has no pipelined odd step: the knob set before initialisation falls back
    D, O = make_pair(clb, oracle, mat, shape, 0.8, 1e-4, getattr(clb, prec), even_tma=tma, odd_pipe=pipe, **BIO)
    D.flow_step(400)
    O.step(400)
    err = rel_l2(D.velocity(), O.velocity())
    print(f"{prec} velocity rel L2 after 400 steps: {err:.3e}")
    assert err < tol


def test_set_populations_round_trip(clb, oracle):
    shape = (12, 7, 6)
    mat = mixed_geometry(*shape)
    D, O = make_pair(clb, oracle, mat, shape, 0.7, 1e-4, clb.F64)
    D.flow_step(3)  # odd parity: the scatter must invert the gather
    f = D.flow_populations()
    rng = np.random.default_rng(1)
    g = f + 1e-5 * rng.standard_normal(f.shape)
    D.set_flow_populations(g)
    # wall nodes keep only the slots their fluid neighbours use; every fluid node keeps all
    fluid = mat != 1
    np.testing.assert_array_equal(D.flow_populations()[:, fluid], g[:, fluid])
    O.set_populations(g)
    D.flow_step(5)
    O.step(5)
    assert np.max(np.abs(D.flow_populations()[:, fluid] - O.populations()[:, fluid])) < 1e-13
    np.testing.assert_allclose(D.velocity(), O.velocity(), rtol=0, atol=1e-15)


def test_flow_step_before_init_is_an_error(clb):
    D = clb.Domain(np.full(4 * 4 * 4, 2, np.int8), 4, 4, 4, 0.8)
    with pytest.raises(clb.ClbError) as e:
        D.flow_step(1)
    assert e.value.status == 7


def test_autotune_leaves_state_unchanged(clb, oracle):
    shape = (30, 16, 20)
    mat = mixed_geometry(*shape, seed=11)
    D, O = make_pair(clb, oracle, mat, shape, 0.8, 2e-4, clb.F64, **BIO)
    D.flow_step(7)
    O.step(7)
    rep = D.autotune(4)
    assert "->" in rep and "tma=" in rep
    D.flow_step(5)
    O.step(5)
    fluid = mat != 1
    assert np.max(np.abs(D.flow_populations()[:, fluid] - O.populations()[:, fluid])) < 1e-13
    D.tune("flow_min_blocks", 2)
    D.tune("flow_odd_pipe", 1)
    with pytest.raises(clb.ClbError):
        D.tune("flow_min_blocks", 5)
    with pytest.raises(clb.ClbError):
        D.tune("no_such_knob", 1)


def test_pipelined_odd_step_f32_matches_plain_bit_for_bit(clb):
    """The pipelined odd step does the same arithmetic as the plain one: identical populations."""
    shape = (34, 19, 23)
    mat = mixed_geometry(*shape, seed=21)
    out = []
    for pipe in (0, 1):
        D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F32, **BIO)
        D.tune("flow_odd_pipe", pipe)
        D.flow_init(2e-4)
        D.flow_step(61)
        out.append(D.flow_populations())
    np.testing.assert_array_equal(out[0], out[1])


def test_pipelined_odd_step_refused_for_fp16_storage(clb):
    shape = (10, 6, 6)
    D = clb.Domain(mixed_geometry(*shape), *shape, 0.8, flow_precision=clb.F16S)
    D.flow_init(1e-4)
    with pytest.raises(clb.ClbError):
        D.tune("flow_odd_pipe", 1)


def test_velocity_read_as_float32_equals_float64_rounded(clb):
    shape = (16, 9, 8)
    D = clb.Domain(mixed_geometry(*shape, seed=3), *shape, 0.8, flow_precision=clb.F32, **BIO)
    D.flow_init(2e-4)
    D.flow_step(30)
    u64, u32 = D.velocity(), D.velocity(np.float32)
    assert u32.dtype == np.float32
    np.testing.assert_array_equal(u32, u64.astype(np.float32))
    with pytest.raises(ValueError):
        D.velocity(np.int32)


def test_flow_stats_match_the_reference_formulas_on_the_oracle_field(clb, oracle):
    """Mean |u| and max u_x over x = 1..nx-2, the outlet-plane Darcy velocity (x = nx-2) and the
    permeability k = u_darcy nu L / dP (complab.cpp:1136-1160), from the GPU against the same
    reductions of the oracle's velocity field."""
    shape = (24, 12, 12)
    nx, ny, nz = shape
    mat = mixed_geometry(*shape, seed=13, biofilm=False)
    D, O = make_pair(clb, oracle, mat, shape, 0.8, 2e-4, clb.F64)
    D.flow_step(300)
    O.step(300)
    L = 8.0
    st = D.flow_stats(L)
    u = O.velocity().reshape(3, nx, ny, nz)
    inner = u[:, 1:nx - 1]
    nu = (0.8 - 0.5) / 3.0
    darcy = u[0, nx - 2].mean()
    np.testing.assert_allclose(st["pore_mean_u"], np.sqrt((inner ** 2).sum(0)).mean(), rtol=1e-10)
    np.testing.assert_allclose(st["pore_max_ux"], inner[0].max(), rtol=1e-10)
    np.testing.assert_allclose(st["darcy_outlet_ux"], darcy, rtol=1e-10)
    np.testing.assert_allclose(st["permeability"], darcy * nu * L / 2e-4, rtol=1e-10)


def test_peclet_rescale_reaches_the_target_velocity(clb):
    """The Péclet rescale (complab.cpp:1156-1179): the pressure drop is scaled so that the outlet
    Darcy velocity gives Pe = u L / D with D the fixed ADE diffusivity; after the one re-solve the
    achieved Péclet number is within 2 % (Stokes flow is linear in the pressure drop)."""
    shape = (30, 14, 14)
    mat = mixed_geometry(*shape, seed=17, solid_block=False, biofilm=False)
    D = clb.Domain(mat, *shape, 0.8, flow_precision=clb.F64)
    D.flow_init(1e-4)
    pe, L, tau_ade = 1.0, 8.0, 0.8
    dp, it, conv = D.flow_solve_peclet(pe, L, tau_ade, 60000, 1e-8)
    assert conv and dp != 1e-4
    st = D.flow_stats(L)
    d_fixed = 0.25 * (tau_ade - 0.5)
    nu = (0.8 - 0.5) / 3.0
    u_darcy = st["permeability"] * dp / (nu * L)
    assert abs(u_darcy * L / d_fixed - pe) / pe < 0.02

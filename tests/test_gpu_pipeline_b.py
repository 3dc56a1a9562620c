"""Pipeline B on the device (through the C-ABI) against the reference's own
outputs: the b_ref_* fixtures of oracle/_ref/mac_ref_b, i.e. the per-step init
and Algorithms_RungeKutta_all of test/Jet3.cpp:642-726 (stage topology, forces
with viscosity 1e-3, force projection with Dirichlet air pressures,
extrapolation of speed and acceleration, RK4 over grid and particles) from the
depth world after 10 steps.

The init is bit-exact. Steps carry the projection solves (relative residual
1e-13 here): pressure within 1e-9 and speeds within 1e-10 relative L2 after one
step, topology and the particle set identical.
"""
import pytest

from compare import compare_particles, compare_topology, field_errors

pytestmark = pytest.mark.gpu


def _b_input(golden):
    s = golden("d_ref_s10")
    s.params.viscosity = 1e-3
    s.params.pipeline = 1
    return s


def _ctx(state):
    from mac_b200.gpu import Context
    return Context(state.params, max_bricks=4096, max_particles=1 << 21, rtol=1e-13, max_iters=3000)


def test_pipeline_b_init_bit_exact(golden):
    s = _b_input(golden)
    ref = golden("b_ref_i10")
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.topology()
        ctx.extrapolate()
        got = ctx.download()
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert all(v == 0.0 for v in e.values()), e
    assert got.params.dt == ref.params.dt


def test_pipeline_b_steps(golden):
    s = _b_input(golden)
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.step()
        got = ctx.download()
        ref = golden("b_ref_s11")
        compare_topology(got, ref)
        e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
        assert e["p"] <= 1e-9 and max(e["u0x"], e["u0y"], e["u0z"]) <= 1e-10, e
        compare_particles(got, ref, atol=1e-12)
        assert abs(got.params.t - ref.params.t) <= 1e-15
        for _ in range(4):
            ctx.step()
        got = ctx.download()
    ref = golden("b_ref_s15")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= 1e-8 and max(e["u0x"], e["u0y"], e["u0z"]) <= 1e-9, e
    compare_particles(got, ref, atol=1e-10)


def test_pipeline_b_needs_the_depth_composition(golden):
    from mac_b200.gpu import Context, MacError
    s = golden("c1_ref_s30")
    s.params.pipeline = 1
    with pytest.raises(MacError):
        Context(s.params, max_bricks=1024, max_particles=1 << 20)

"""The 32x32x64 jet (h = 0.05, inflow radius 4 at w = 1, CFL 0.5, LayerMax 4)
run for 100 steps on the device from the reference's first init, the loop of
test/TestJetDEau_Basic.cpp:434-441.

Before every device step the device state is downloaded and handed to the
oracle for one step (its solve: FP64 Jacobi-CG to 1e-14, the Umfpack
stand-in); the device's own next step from the same state must match it:
topology (cells, layers, materials, flags), dt and time bit for bit, pressure
within 1e-9 and velocities within 1e-10 (relative L2), particles within 1e-10.
Both MG-PCG forms run, each to a relative residual of 1e-13.
"""
import pytest

from compare import compare_particles, compare_topology, field_errors

pytestmark = pytest.mark.gpu

STEPS = 100
P_TOL = 1e-9
U_TOL = 1e-10


@pytest.mark.parametrize("solver", ["mgpcg64", "mixed"])
def test_c1_100_steps_each_checked_against_the_oracle(golden, run_oracle, solver):
    from mac_b200.gpu import Context
    from mac_b200.world import first_init
    setup = golden("c1_setup")
    worst = {"p": 0.0, "u": 0.0}
    with Context(setup.params, max_bricks=2048, max_particles=1 << 20, solver=solver, rtol=1e-13,
                 max_iters=3000) as ctx:
        first_init(ctx, setup)
        for k in range(STEPS):
            state = ctx.download()
            want, _ = run_oracle("step", state, 1, 1e-14)
            ctx.step()
            got = ctx.download()
            compare_topology(got, want)
            assert got.params.dt == want.params.dt, k
            assert abs(got.params.t - want.params.t) <= 1e-15, k
            e = field_errors(got, want, ("p", "u0x", "u0y", "u0z"))
            u = max(e["u0x"], e["u0y"], e["u0z"])
            assert e["p"] <= P_TOL and u <= U_TOL, (k, e)
            compare_particles(got, want, atol=1e-10)
            worst["p"] = max(worst["p"], e["p"])
            worst["u"] = max(worst["u"], u)
        assert got.fluid_cells() > 1000
    print(f"{solver}: {STEPS} steps, worst pressure {worst['p']:.2e}, worst velocity {worst['u']:.2e}")

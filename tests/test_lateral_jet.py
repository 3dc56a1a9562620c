"""The lateral jet (384x192x192, h = 0.01, circular side-wall inflow of radius
16 cells at 3 m/s aimed 15 degrees up, gravity -9.81 z, CFL 0.5): 1000 steps on
the device from the first init, with the state at steps 100 and 1000 handed to
the oracle for one step, compared with the device's own next step from the same
state (topology and particles bit-exact or within 1e-12, pressure within 1e-9,
velocities within 1e-10; the solves run to 1e-13 against the oracle's 1e-14).
"""
import numpy as np
import pytest

from compare import compare_particles, compare_topology, field_errors


def _world():
    from mac_b200.state import lateral_jet_world
    return lateral_jet_world()


def test_lateral_world_shape():
    from mac_b200.state import INFLOW, SOLID
    s = _world()
    ex = s.exists.astype(bool)
    ck = s.cell_keys()[ex]
    t = s.type[ex]
    inflow = t == INFLOW
    assert 780 <= inflow.sum() <= 830  # pi 16^2
    assert np.all(ck[inflow][:, 0] == 0)
    assert np.all(s.flags[ex][inflow] & 7 == 7)
    u = s.f64["u0x"][ex][inflow]
    w = s.f64["u0z"][ex][inflow]
    assert np.allclose(u, 3.0 * np.cos(np.deg2rad(15.0))) and np.allclose(w, 3.0 * np.sin(np.deg2rad(15.0)))
    assert np.all(t[(ck[:, 2] == -1)] == SOLID)


@pytest.mark.gpu
def test_lateral_jet_1000_steps_checked_against_the_oracle(run_oracle):
    from mac_b200.gpu import Context
    from mac_b200.world import first_init
    s = _world()
    kw = dict(max_bricks=60000, max_particles=8_000_000, rtol=1e-13, max_iters=3000)
    checked = 0
    with Context(s.params, **kw) as ctx:
        first_init(ctx, s)
        done = 0
        for stop in (100, 1000):
            while done < stop:
                ctx.step()
                done += 1
            state = ctx.download()
            assert state.fluid_cells() > 0
            want, _ = run_oracle("step", state, 1, 1e-14)
            with Context(state.params, **kw) as c2:
                c2.upload(state)
                c2.step()
                got = c2.download()
            compare_topology(got, want)
            e = field_errors(got, want, ("p", "u0x", "u0y", "u0z"))
            assert e["p"] <= 1e-9 and max(e["u0x"], e["u0y"], e["u0z"]) <= 1e-10, (stop, e)
            compare_particles(got, want, atol=1e-12)
            checked += 1
            print(f"step {stop}: {state.fluid_cells()} fluid cells, {state.nparticles} particles, errors {e}")
    assert checked == 2

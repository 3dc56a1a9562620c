"""Device parity (through the C-ABI) for the viscous and depth compositions
and pipeline B on the seeded worlds of test_oracle_live_reference.py, against
the oracle from the same input states: the viscous forces, the depth first
init and topology and pipeline B's per-step init bit for bit; whole steps
within the fixture tests' tolerances (pressure 1e-9, velocities 1e-10
relative L2, the solves at a relative residual of 1e-13).
"""
import copy
import dataclasses

import pytest

from compare import compare_particles, compare_topology, field_errors, max_abs_diff
from test_oracle_live_reference import DEPTH_WORLDS, NU, SPIN_UP, VISC_WORLDS, WORLDS

pytestmark = pytest.mark.gpu

P_TOL = 1e-9
U_TOL = 1e-10


def _ctx(state):
    from mac_b200.gpu import Context
    return Context(state.params, max_bricks=4096, max_particles=1 << 21, rtol=1e-13, max_iters=3000)


def _exact(a, b, fields):
    d = max_abs_diff(a, b, fields, existing_only=False)
    assert all(v == 0.0 for v in d.values()), d


def _step_close(got, want, atol=1e-12):
    compare_topology(got, want)
    e = field_errors(got, want, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    compare_particles(got, want, atol=atol)


@pytest.fixture(scope="module")
def states(tmp_path_factory):
    """The oracle's spun-up states: each viscous world after SPIN_UP steps (and
    its per-step topology), each depth world after six steps."""
    import oracle
    from mac_b200.state import State, jet_world
    oracle.build()
    d = tmp_path_factory.mktemp("compositions")
    out = {}
    for name in VISC_WORLDS:
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        jet_world(**WORLDS[name]).write(t("setup"))
        oracle.run_oracle("firstinit", t("setup"), t("s0"))
        oracle.run_oracle("step", t("s0"), t("s8"), SPIN_UP)
        oracle.run_oracle("topology", t("s8"), t("t8"))
        out[name] = {k: State.read(t(k)) for k in ("s8", "t8")}
        for s in out[name].values():
            s.params.viscosity = NU
    for name, (kw, (dmax, dint, drem), cube) in DEPTH_WORLDS.items():
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        s = jet_world(**kw)
        pr = s.params
        pr.depth_mode, pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube = 1, dmax, dint, drem, cube
        s.write(t("setup"))
        oracle.run_oracle("firstinit", t("setup"), t("s0"))
        oracle.run_oracle("step", t("s0"), t("s6"), 6)
        out[name] = {"setup": s, **{k: State.read(t(k)) for k in ("s0", "s6")}}
    return out


@pytest.mark.parametrize("world", VISC_WORLDS)
def test_viscous_forces_and_step(states, run_oracle, world):
    t8, s8 = states[world]["t8"], states[world]["s8"]
    want, _ = run_oracle("vforces", t8)
    with _ctx(t8) as ctx:
        ctx.upload(t8)
        ctx.forces(0)
        got = ctx.download()
    compare_topology(got, want)
    _exact(got, want, ("ax", "ay", "az", "u0x", "u0y", "u0z"))
    want, _ = run_oracle("vstep", s8)
    with _ctx(s8) as ctx:
        ctx.upload(s8)
        ctx.step()
        got = ctx.download()
    _step_close(got, want)


@pytest.mark.parametrize("world", list(DEPTH_WORLDS))
def test_depth_init_topology_and_step(states, run_oracle, world):
    from mac_b200.world import first_init
    r = states[world]
    with _ctx(r["setup"]) as ctx:
        first_init(ctx, r["setup"])
        got = ctx.download()
    compare_topology(got, r["s0"])
    _exact(got, r["s0"], ("u0x", "u0y", "u0z", "p"))
    assert compare_particles(got, r["s0"]) == 0.0
    want, _ = run_oracle("topology", r["s6"])
    with _ctx(r["s6"]) as ctx:
        ctx.upload(r["s6"])
        ctx.topology()
        got = ctx.download()
    compare_topology(got, want)
    assert compare_particles(got, want) == 0.0
    assert got.params.dt == want.params.dt
    want, _ = run_oracle("step", r["s6"])
    with _ctx(r["s6"]) as ctx:
        ctx.upload(r["s6"])
        ctx.step()
        got = ctx.download()
    _step_close(got, want)


def test_pipeline_b_init_and_step(states, run_oracle):
    s = copy.copy(states[next(iter(DEPTH_WORLDS))]["s6"])
    s.params = dataclasses.replace(s.params, viscosity=NU, pipeline=1)
    want, _ = run_oracle("binit", s)
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.topology()
        ctx.extrapolate()
        got = ctx.download()
    compare_topology(got, want)
    assert compare_particles(got, want) == 0.0
    _exact(got, want, ("u0x", "u0y", "u0z", "p"))
    assert got.params.dt == want.params.dt
    want, _ = run_oracle("bstep", s)
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.step()
        got = ctx.download()
    _step_close(got, want)

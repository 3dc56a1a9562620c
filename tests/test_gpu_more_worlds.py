"""Device parity (through the C-ABI) on the seeded jets of
test_oracle_live_reference.py (other boxes, inflows, pools and LayerMax
values than the committed fixtures' world), against the oracle from the same
input states: the first init, the per-step topology, the force and
extrapolation stencils and both particle moves bit for bit; a whole step
within the tolerances of the fixture tests (pressure 1e-9, velocities 1e-10
relative L2, the solve at a relative residual of 1e-13).
"""
import pytest

from compare import compare_particles, compare_topology, field_errors, max_abs_diff
from test_oracle_live_reference import SPIN_UP, WORLDS

pytestmark = pytest.mark.gpu

P_TOL = 1e-9
U_TOL = 1e-10
ALL = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")


def _ctx(state):
    from mac_b200.gpu import Context
    return Context(state.params, max_bricks=4096, max_particles=1 << 21, rtol=1e-13, max_iters=2000)


def _exact(a, b, fields=ALL):
    d = max_abs_diff(a, b, fields, existing_only=False)
    assert all(v == 0.0 for v in d.values()), d


@pytest.fixture(scope="module")
def oracle_runs(tmp_path_factory):
    """Per world: the set-up state, the oracle's first init and its state after
    SPIN_UP steps, and that state after the oracle's per-step topology."""
    import oracle
    from mac_b200.state import State, jet_world
    oracle.build()
    d = tmp_path_factory.mktemp("worlds")
    runs = {}
    for name, kw in WORLDS.items():
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        jet_world(**kw).write(t("setup"))
        oracle.run_oracle("firstinit", t("setup"), t("s0"))
        oracle.run_oracle("step", t("s0"), t("s8"), SPIN_UP)
        oracle.run_oracle("topology", t("s8"), t("t8"))
        runs[name] = {k: State.read(t(k)) for k in ("setup", "s0", "s8", "t8")}
    return runs


@pytest.mark.parametrize("world", list(WORLDS))
def test_first_init_and_topology_bit_exact(oracle_runs, world):
    from mac_b200.world import first_init
    r = oracle_runs[world]
    with _ctx(r["setup"]) as ctx:
        first_init(ctx, r["setup"])
        got = ctx.download()
    compare_topology(got, r["s0"])
    _exact(got, r["s0"], ("u0x", "u0y", "u0z", "p"))
    assert compare_particles(got, r["s0"]) == 0.0
    with _ctx(r["s8"]) as ctx:
        ctx.upload(r["s8"])
        ctx.topology()
        got = ctx.download()
    compare_topology(got, r["t8"])
    _exact(got, r["t8"])
    assert compare_particles(got, r["t8"]) == 0.0
    assert got.params.dt == r["t8"].params.dt


@pytest.mark.parametrize("world", list(WORLDS))
def test_stencils_and_moves_bit_exact(oracle_runs, run_oracle, world):
    t8 = oracle_runs[world]["t8"]
    for stage, call, fields in (("forces", lambda c: c.forces(0), ("ax", "ay", "az", "u0x", "u0y", "u0z")),
                                ("extrapolate", lambda c: c.extrapolate(), ("u0x", "u0y", "u0z"))):
        want, _ = run_oracle(stage, t8)
        with _ctx(t8) as ctx:
            ctx.upload(t8)
            call(ctx)
            got = ctx.download()
        compare_topology(got, want)
        _exact(got, want, fields)
    for stage, sym in (("move", 1), ("movelin", 0)):
        want, _ = run_oracle(stage, t8)
        t8.params.interp_symmetric = sym
        with _ctx(t8) as ctx:
            ctx.upload(t8)
            ctx.move()
            got = ctx.download()
        t8.params.interp_symmetric = 1
        assert compare_particles(got, want) == 0.0


@pytest.mark.parametrize("world", list(WORLDS))
def test_step_within_tolerance(oracle_runs, run_oracle, world):
    s8 = oracle_runs[world]["s8"]
    want, _ = run_oracle("step", s8)
    with _ctx(s8) as ctx:
        ctx.upload(s8)
        ctx.step()
        got = ctx.download()
    compare_topology(got, want)
    e = field_errors(got, want, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    compare_particles(got, want, atol=1e-12)

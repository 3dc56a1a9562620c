"""The oracle against the reference's own code run here (oracle/_ref, compiled
from the reference's headers by oracle/Makefile), on seeded jet worlds other
than the committed fixtures' one: other box shapes, inflow radii and speeds,
pool depths, LayerMax values and particle seeds.

From the same input state the oracle must agree bit for bit on the set-up
passes, the first init, the per-step topology, the force and extrapolation
stencils and both particle moves, and within solver rounding on the
projection and a full step (both solve to a relative residual of 1e-14).
Skipped where the reference runners are not built.
"""
import os

import pytest

from compare import compare_particles, compare_topology, field_errors, max_abs_diff

ALL = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")

# (box nx, ny, nz, h, inflow radius, inflow speed, pool depth, LayerMax, seed)
WORLDS = {
    "box24x20x40_pool6": dict(nx=24, ny=20, nz=40, h=0.05, r_inflow=3.0, w_inflow=1.5, pool_depth=6,
                              layer_max=3, seed=7),
    "box16x32x48_lm6": dict(nx=16, ny=32, nz=48, h=0.04, r_inflow=5.0, w_inflow=2.0, pool_depth=0,
                            layer_max=6, seed=11),
    "box28x28x24_pool10": dict(nx=28, ny=28, nz=24, h=0.05, r_inflow=4.0, w_inflow=0.8, pool_depth=10,
                               layer_max=4, seed=3),
}
SPIN_UP = 8  # reference steps from the first init before the per-stage checks


def _exact(a, b, fields=ALL):
    d = max_abs_diff(a, b, fields, existing_only=False)
    assert all(v == 0.0 for v in d.values()), d


@pytest.fixture(scope="module")
def ref_runs(tmp_path_factory):
    """Per world: the set-up state and the reference's outputs from it."""
    import oracle
    from mac_b200.state import State, jet_world
    oracle.build()
    if not oracle.have_ref():
        pytest.skip("reference runners (oracle/_ref) not built")
    d = tmp_path_factory.mktemp("live")
    runs = {}
    for name, kw in WORLDS.items():
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        s = jet_world(**kw)
        s.write(t("setup"))
        oracle.run_ref("setup", t("setup"), t("rsetup"))
        oracle.run_ref("firstinit", t("setup"), t("s0"))
        oracle.run_ref("step", t("s0"), t("s8"), SPIN_UP)
        oracle.run_ref("topology", t("s8"), t("t8"))
        for st in ("forces", "extrapolate", "move", "movelin", "project"):
            oracle.run_ref(st, t("t8"), t("t8_" + st))
        oracle.run_ref("step", t("s8"), t("s9"), 1)
        runs[name] = {k: State.read(t(k)) for k in
                      ("setup", "rsetup", "s0", "s8", "t8", "t8_forces", "t8_extrapolate", "t8_move",
                       "t8_movelin", "t8_project", "s9")}
    return runs


@pytest.mark.parametrize("world", list(WORLDS))
def test_setup_and_first_init_bit_exact(ref_runs, run_oracle, world):
    from mac_b200.world import setup_passes
    r = ref_runs[world]
    got = setup_passes(r["setup"])
    compare_topology(got, r["rsetup"])
    _exact(got, r["rsetup"])
    got, _ = run_oracle("firstinit", r["setup"])
    compare_topology(got, r["s0"])
    _exact(got, r["s0"])
    assert compare_particles(got, r["s0"]) == 0.0


@pytest.mark.parametrize("world", list(WORLDS))
def test_topology_bit_exact(ref_runs, run_oracle, world):
    r = ref_runs[world]
    got, st = run_oracle("topology", r["s8"])
    compare_topology(got, r["t8"])
    _exact(got, r["t8"])
    assert compare_particles(got, r["t8"]) == 0.0
    assert got.params.dt == r["t8"].params.dt
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("world", list(WORLDS))
@pytest.mark.parametrize("stage", ["forces", "extrapolate", "move", "movelin"])
def test_stages_bit_exact(ref_runs, run_oracle, world, stage):
    r = ref_runs[world]
    got, st = run_oracle(stage, r["t8"])
    ref = r["t8_" + stage]
    compare_topology(got, ref)
    _exact(got, ref)
    assert compare_particles(got, ref) == 0.0
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("world", list(WORLDS))
def test_projection_and_step_within_rounding(ref_runs, run_oracle, world):
    r = ref_runs[world]
    got, st = run_oracle("project", r["t8"])
    compare_topology(got, r["t8_project"])
    e = field_errors(got, r["t8_project"], ALL)
    assert max(e.values()) <= 1e-12, e
    assert st["relres"] <= 1e-14
    got, _ = run_oracle("step", r["s8"])
    compare_topology(got, r["s9"])
    e = field_errors(got, r["s9"], ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, r["s9"], atol=1e-14)

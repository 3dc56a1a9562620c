"""The oracle against the reference's own code run here (oracle/_ref, compiled
from the reference's headers by oracle/Makefile), on seeded jet worlds other
than the committed fixtures' one: other box shapes, inflow radii and speeds,
pool depths, LayerMax values and particle seeds.

From the same input state the oracle must agree bit for bit on the set-up
passes, the first init, the per-step topology, the force and extrapolation
stencils and both particle moves, and within solver rounding on the
projection and a full step (both solve to a relative residual of 1e-14). The
same holds for the viscous composition on two of the worlds (viscosity 2e-3),
and for the depth composition on two pool worlds with other Policy_Depth
rules, one of which also runs pipeline B's init and step, and for a small
lateral jet (side-wall inflow aimed 15 degrees up). Skipped where the
reference runners are not built.
"""
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


# ---------------------------------------------------------------- viscous
VISC_WORLDS = ("box24x20x40_pool6", "box28x28x24_pool10")
NU = 2e-3


@pytest.fixture(scope="module")
def ref_visc(ref_runs, tmp_path_factory):
    """The viscous composition (Algorithms_Viscosity, Algorithms_Solve_Pressure_Dirichlet
    with Policy_Dirichlet_Boundary) from the spun-up states of two worlds."""
    import oracle
    from mac_b200.state import State
    d = tmp_path_factory.mktemp("livev")
    out = {}
    for name in VISC_WORLDS:
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        r = ref_runs[name]
        for k in ("t8", "s8"):
            s = r[k]  # viscosity set for the written copy only
            s.params.viscosity = NU
            s.write(t(k + "v"))
            s.params.viscosity = 0.0
        for st in ("vforces", "vproject", "vode"):
            oracle.run_ref(st, t("t8v"), t("t8v_" + st))
        oracle.run_ref("vstep", t("s8v"), t("s9v"), 1)
        out[name] = {k: State.read(t(k)) for k in ("t8v", "s8v", "t8v_vforces", "t8v_vproject", "t8v_vode", "s9v")}
    return out


@pytest.mark.parametrize("world", VISC_WORLDS)
def test_viscous_forces_bit_exact(ref_visc, run_oracle, world):
    r = ref_visc[world]
    got, st = run_oracle("vforces", r["t8v"])
    compare_topology(got, r["t8v_vforces"])
    _exact(got, r["t8v_vforces"])
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("world", VISC_WORLDS)
@pytest.mark.parametrize("stage", ["vproject", "vode"])
def test_viscous_solver_stages_within_rounding(ref_visc, run_oracle, world, stage):
    r = ref_visc[world]
    got, st = run_oracle(stage, r["t8v"])
    compare_topology(got, r["t8v_" + stage])
    e = field_errors(got, r["t8v_" + stage], ALL)
    assert max(e.values()) <= 1e-12, e
    assert st["relres"] <= 1e-14


@pytest.mark.parametrize("world", VISC_WORLDS)
def test_viscous_step_within_rounding(ref_visc, run_oracle, world):
    r = ref_visc[world]
    got, _ = run_oracle("vstep", r["s8v"])
    compare_topology(got, r["s9v"])
    e = field_errors(got, r["s9v"], ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, r["s9v"], atol=1e-14)


# ------------------------------------------------------------------ depth
# (world keywords, Policy_Depth (max, interior, remove), cube refill n)
DEPTH_WORLDS = {
    "depth20x28x36_pool14": (dict(nx=20, ny=28, nz=36, h=0.05, r_inflow=3.0, w_inflow=1.2, pool_depth=14,
                                  layer_max=4, seed=5), (5, 2, 4), 1),
    "depth24x24x28_pool16": (dict(nx=24, ny=24, nz=28, h=0.05, r_inflow=4.0, w_inflow=1.0, pool_depth=16,
                                  layer_max=3, seed=9), (6, 4, 4), 1),
}


@pytest.fixture(scope="module")
def ref_depth(tmp_path_factory):
    import oracle
    from mac_b200.state import State, jet_world
    oracle.build()
    if not oracle.have_ref():
        pytest.skip("reference runners (oracle/_ref) not built")
    d = tmp_path_factory.mktemp("lived")
    runs = {}
    for name, (kw, (dmax, dint, drem), cube) in DEPTH_WORLDS.items():
        t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
        s = jet_world(**kw)
        pr = s.params
        pr.depth_mode, pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube = 1, dmax, dint, drem, cube
        s.write(t("setup"))
        oracle.run_ref("firstinit", t("setup"), t("s0"))
        oracle.run_ref("step", t("s0"), t("s6"), 6)
        oracle.run_ref("topology", t("s6"), t("t6"))
        oracle.run_ref("step", t("s6"), t("s7"), 1)
        runs[name] = {k: State.read(t(k)) for k in ("setup", "s0", "s6", "t6", "s7")}
    # pipeline B (three speed buffers, force-mode projection) from the first world
    name = next(iter(DEPTH_WORLDS))
    t = lambda n: str(d / f"{name}_{n}.state")  # noqa: E731
    s = runs[name]["s6"]
    s.params.viscosity = NU
    s.write(t("bs6"))
    s.params.viscosity = 0.0
    oracle.run_ref("binit", t("bs6"), t("bi6"))
    oracle.run_ref("bstep", t("bs6"), t("bs7"), 1)
    runs[name].update({k: State.read(t(k)) for k in ("bs6", "bi6", "bs7")})
    return runs


@pytest.mark.parametrize("world", list(DEPTH_WORLDS))
def test_depth_first_init_and_topology_bit_exact(ref_depth, run_oracle, world):
    from mac_b200.state import INTERIOR
    r = ref_depth[world]
    got, _ = run_oracle("firstinit", r["setup"])
    compare_topology(got, r["s0"])
    _exact(got, r["s0"], ("u0x", "u0y", "u0z", "p"))
    assert compare_particles(got, r["s0"]) == 0.0
    got, _ = run_oracle("topology", r["s6"])
    compare_topology(got, r["t6"])
    assert compare_particles(got, r["t6"]) == 0.0
    assert got.params.dt == r["t6"].params.dt
    ex = r["t6"].exists.astype(bool)
    assert (ex & (r["t6"].type == INTERIOR)).sum() > 0  # the depth rules are exercised


@pytest.mark.parametrize("world", list(DEPTH_WORLDS))
def test_depth_step_within_rounding(ref_depth, run_oracle, world):
    r = ref_depth[world]
    got, _ = run_oracle("step", r["s6"])
    compare_topology(got, r["s7"])
    e = field_errors(got, r["s7"], ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, r["s7"], atol=1e-14)


def test_pipeline_b_init_and_step(ref_depth, run_oracle):
    r = ref_depth[next(iter(DEPTH_WORLDS))]
    got, _ = run_oracle("binit", r["bs6"])
    compare_topology(got, r["bi6"])
    assert compare_particles(got, r["bi6"]) == 0.0
    _exact(got, r["bi6"], ("u0x", "u0y", "u0z", "p"))
    got, _ = run_oracle("bstep", r["bs6"])
    compare_topology(got, r["bs7"])
    e = field_errors(got, r["bs7"], ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, r["bs7"], atol=1e-13)


# ---------------------------------------------------------------- lateral
# a small lateral jet (side-wall inflow aimed 15 degrees up, as the 384x192x192
# configuration), run through the same checks
LATERAL = dict(nx=32, ny=20, nz=20, h=0.05, r_inflow=4.0, speed=2.0, angle_deg=15.0)


@pytest.fixture(scope="module")
def ref_lateral(tmp_path_factory):
    import oracle
    from mac_b200.state import State, lateral_jet_world
    oracle.build()
    if not oracle.have_ref():
        pytest.skip("reference runners (oracle/_ref) not built")
    d = tmp_path_factory.mktemp("livel")
    t = lambda n: str(d / f"lateral_{n}.state")  # noqa: E731
    lateral_jet_world(**LATERAL).write(t("setup"))
    oracle.run_ref("firstinit", t("setup"), t("s0"))
    oracle.run_ref("step", t("s0"), t("s8"), SPIN_UP)
    oracle.run_ref("topology", t("s8"), t("t8"))
    for st in ("forces", "extrapolate", "move"):
        oracle.run_ref(st, t("t8"), t("t8_" + st))
    oracle.run_ref("step", t("s8"), t("s9"), 1)
    return {k: State.read(t(k)) for k in ("setup", "s0", "s8", "t8", "t8_forces", "t8_extrapolate", "t8_move", "s9")}


def test_lateral_jet_bit_exact_and_step(ref_lateral, run_oracle):
    from mac_b200.state import INFLOW
    r = ref_lateral
    got, _ = run_oracle("firstinit", r["setup"])
    compare_topology(got, r["s0"])
    _exact(got, r["s0"])
    assert compare_particles(got, r["s0"]) == 0.0
    got, _ = run_oracle("topology", r["s8"])
    compare_topology(got, r["t8"])
    _exact(got, r["t8"])
    assert compare_particles(got, r["t8"]) == 0.0
    for stage in ("forces", "extrapolate", "move"):
        got, st = run_oracle(stage, r["t8"])
        compare_topology(got, r["t8_" + stage])
        _exact(got, r["t8_" + stage])
        assert compare_particles(got, r["t8_" + stage]) == 0.0
        assert st["invalid_reads"] == 0
    got, _ = run_oracle("step", r["s8"])
    compare_topology(got, r["s9"])
    e = field_errors(got, r["s9"], ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, r["s9"], atol=1e-14)
    # the side-wall inflow is there and has produced fluid
    ex = r["s8"].exists.astype(bool)
    assert (r["s8"].type[ex] == INFLOW).sum() > 40 and r["s8"].nparticles > 1000

"""Parity of the CUDA path (through the C-ABI) with the oracle and with the
reference's own outputs (committed fixtures), stage by stage, from the same
input state.

Tolerances: integer work (cells, layers, materials, flags, particle keys) is
bit-exact; the stencil, extrapolation and particle kernels are bit-exact too
(FP64, reference operation order, no FMA contraction). Quantities behind the
iterative pressure solve are compared by relative L2 error: pressure <= 1e-9,
velocities <= 1e-10 (the solve runs to a relative residual of 1e-13 here).
"""
import numpy as np
import pytest

from compare import compare_particles, compare_topology, field_errors, max_abs_diff

pytestmark = pytest.mark.gpu

P_TOL = 1e-9
U_TOL = 1e-10


def _ctx(state, **kw):
    from mac_b200.gpu import Context
    kw.setdefault("rtol", 1e-13)
    kw.setdefault("max_iters", 2000)
    return Context(state.params, max_bricks=kw.pop("max_bricks", 2048), max_particles=kw.pop("max_particles", 1 << 20),
                   **kw)


def _exact(a, b, fields):
    d = max_abs_diff(a, b, fields, existing_only=False)
    assert all(v == 0.0 for v in d.values()), d


def test_topology_matches_reference(golden, run_oracle):
    s30 = golden("c1_ref_s30")
    ref = golden("c1_ref_t30")
    with _ctx(s30) as ctx:
        ctx.upload(s30)
        ctx.topology()
        got = ctx.download()
    orc, _ = run_oracle("topology", s30)
    for want in (ref, orc):
        compare_topology(got, want)
        _exact(got, want, ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p"))
        assert compare_particles(got, want) == 0.0
        assert got.params.dt == want.params.dt
        assert got.params.step == want.params.step


def test_forces_bit_exact(golden):
    t30 = golden("c1_ref_t30")
    ref = golden("c1_ref_t30_forces")
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        ctx.forces(0)
        got = ctx.download()
    compare_topology(got, ref)
    _exact(got, ref, ("ax", "ay", "az", "u0x", "u0y", "u0z"))


def test_extrapolate_bit_exact(golden):
    t30 = golden("c1_ref_t30")
    ref = golden("c1_ref_t30_extrapolate")
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        ctx.extrapolate()
        got = ctx.download()
    compare_topology(got, ref)
    _exact(got, ref, ("u0x", "u0y", "u0z"))


@pytest.mark.parametrize("name,sym", [("move", 1), ("movelin", 0)])
def test_move_particles_bit_exact(golden, name, sym):
    t30 = golden("c1_ref_t30")
    t30.params.interp_symmetric = sym
    ref = golden("c1_ref_t30_" + name)
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        ctx.move()
        got = ctx.download()
    assert compare_particles(got, ref) == 0.0


@pytest.mark.parametrize("solver", ["mgpcg64", "mixed", "cg64"])
def test_projection_tolerance(golden, run_oracle, solver):
    t30 = golden("c1_ref_t30")
    ref = golden("c1_ref_t30_project")
    with _ctx(t30, solver=solver) as ctx:
        ctx.upload(t30)
        ctx.project(0)
        st = ctx.stats()
        got = ctx.download()
    orc, _ = run_oracle("project", t30)
    for want in (ref, orc):
        compare_topology(got, want)
        e = field_errors(got, want, ("p", "u0x", "u0y", "u0z"))
        assert e["p"] <= P_TOL, e
        assert max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    assert st["relres"] <= 1e-13
    assert st["max_div"] < 1e-8


def test_rk2tvd_tolerance(golden):
    t30 = golden("c1_ref_t30")
    ref = golden("c1_ref_t30_ode")
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        ctx.rk2tvd()
        got = ctx.download()
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az"))
    assert e["p"] <= P_TOL, e
    assert max(e[k] for k in ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z")) <= U_TOL, e
    assert max(e[k] for k in ("ax", "ay", "az")) <= 1e-8, e


def test_full_step(golden):
    s30 = golden("c1_ref_s30")
    ref = golden("c1_ref_s31")
    with _ctx(s30) as ctx:
        ctx.upload(s30)
        ctx.step()
        got = ctx.download()
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    compare_particles(got, ref, atol=1e-12)
    assert abs(got.params.t - ref.params.t) <= 1e-15


def test_first_init_matches_reference(golden):
    from mac_b200.world import first_init
    setup = golden("c1_setup")
    ref = golden("c1_ref_s0")
    with _ctx(setup) as ctx:
        first_init(ctx, setup)
        got = ctx.download()
    compare_topology(got, ref)
    _exact(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert compare_particles(got, ref) == 0.0


def test_composable_projection_in_a_host_rk2tvd(golden):
    """Algorithms_RungeKutta_RK2_TVD (src/Algorithms_RungeKutta_RK2_TVD.h:20-66)
    with its speed-buffer loops on the host and the projections at the
    composable interface on the device (mac_pressure_init, then
    mac_pressure_divergence_projection per stage, then mac_pressure_end), the
    fields moved with mac_upload_field / mac_download_field: matches the
    reference's own RK2-TVD output."""
    t30 = golden("c1_ref_t30")
    ref = golden("c1_ref_t30_ode")
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        dt = t30.params.dt
        flags = ctx.download().flags.reshape(-1)
        ctx.pressure_init()
        ctx.forces(0)  # acc = 0, gravity + convection on speed 0
        acc = {a: ctx.download_field("a" + a) for a in "xyz"}
        u0 = {a: ctx.download_field("u0" + a) for a in "xyz"}
        for a in "xyz":  # stage 1 (forced): u1 = u0 + acc dt
            ctx.upload_field("u1" + a, u0[a] + acc[a] * dt)
        ctx.divergence_projection(1)
        ctx.forces(1)
        acc = {a: ctx.download_field("a" + a) for a in "xyz"}
        u1 = {a: ctx.download_field("u1" + a) for a in "xyz"}
        for i, a in enumerate("xyz"):  # stage 2 (non-forced: const faces keep u0)
            new = 0.5 * u0[a] + 0.5 * u1[a] + 0.5 * acc[a] * dt
            const = (flags & (1 << i)) != 0
            ctx.upload_field("u0" + a, np.where(const, u0[a], new))
        ctx.divergence_projection(0)
        ctx.pressure_end()
        got = ctx.download()
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z", "u1x", "u1y", "u1z"))
    assert e["p"] <= P_TOL, e
    assert max(e[k] for k in ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z")) <= U_TOL, e


def test_divergence_projection_needs_an_init(golden):
    from mac_b200.gpu import MacError
    t30 = golden("c1_ref_t30")
    with _ctx(t30) as ctx:
        ctx.upload(t30)
        with pytest.raises(MacError):
            ctx.divergence_projection(0)


def test_stage_buffers_can_be_left_out_of_the_transfers(golden):
    """NULL speed-1 and acceleration pointers in mac_host_state: the step
    writes both before reading them on every existing cell, so a world
    uploaded without them steps to the same topology, speed 0, pressure and
    particles, bit for bit on the existing cells, as one uploaded whole."""
    from mac_b200.gpu import HostState
    s30 = golden("c1_ref_s30")
    with _ctx(s30) as ctx:
        ctx.upload(s30)
        ctx.step()
        want = ctx.download()
    lean = HostState(s30.nbricks + 64, s30.nparticles + 4096, stage_buffers=False).fill(s30)
    with _ctx(s30) as ctx:
        ctx.upload(None, lean)
        ctx.step()
        ctx.download(lean, to_state=False)
        got = lean.to_state(s30.params)
    compare_topology(got, want)
    d = max_abs_diff(got, want, ("u0x", "u0y", "u0z", "p"), existing_only=True)
    assert all(v == 0.0 for v in d.values()), d
    assert compare_particles(got, want) == 0.0


STEP_FIELDS = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")


def _steps(state, n, solver, dependent_launch=True, concurrent_binning=True):
    with _ctx(state, solver=solver, rtol=1e-8) as ctx:
        ctx.set_dependent_launch(dependent_launch)
        ctx.set_concurrent_binning(concurrent_binning)
        ctx.upload(state)
        for _ in range(n):
            ctx.step()
        return ctx.download(), ctx.stats()["total_iterations"]


@pytest.mark.parametrize("solver", ["mixed", "mgpcg64", "cg64"])
def test_steps_are_reproducible(golden, solver):
    """Three steps from the same state give the same world bit for bit on
    every run: the domain bricks are put in coordinate order before the
    solve, so the CG's partial sums add in the same order whatever order the
    bricks were created or appended in (new bricks take pool slots in the
    order the topology's atomics hand them out)."""
    s30 = golden("c1_ref_s30")
    a, ia = _steps(s30, 3, solver)
    b, ib = _steps(s30, 3, solver)
    assert ia == ib
    compare_topology(a, b)
    d = max_abs_diff(a, b, STEP_FIELDS, existing_only=True)
    assert all(v == 0.0 for v in d.values()), d
    assert compare_particles(a, b) == 0.0


@pytest.mark.parametrize("dependent_launch,concurrent_binning", [(False, True), (True, False), (False, False)])
def test_launch_forms_change_no_bit(golden, dependent_launch, concurrent_binning):
    """The CG loop's kernels launched with programmatic stream serialisation
    and the particle binning on a second stream during RK2-TVD (the defaults)
    give the same world, particles included, as plain stream order and the
    binning inside the move."""
    s30 = golden("c1_ref_s30")
    a, ia = _steps(s30, 3, "mixed")
    b, ib = _steps(s30, 3, "mixed", dependent_launch, concurrent_binning)
    assert ia == ib
    compare_topology(a, b)
    d = max_abs_diff(a, b, STEP_FIELDS, existing_only=True)
    assert all(v == 0.0 for v in d.values()), d
    assert compare_particles(a, b) == 0.0

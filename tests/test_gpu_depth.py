"""Parity of the depth composition on the device (through the C-ABI) with the
reference's own outputs (the d_ref_* fixtures of oracle/_ref/mac_ref_depth:
a 24x24x32 jet over a 12-cell pool, Policy_Depth(4, 3, 3), cube(1) refill) and,
on a deeper pool that needs several relaxation launches, with the oracle.

Integer work is bit-exact: existence, material (interior included), layer,
depth and the particle set after removal and refill; quantities behind the
pressure solve are within the tolerances of the pipeline-A parity tests.
"""
import os
import sys

import numpy as np
import pytest

from compare import compare_particles, compare_topology, field_errors

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

P_TOL = 1e-9
U_TOL = 1e-10


def _ctx(state, **kw):
    from mac_b200.gpu import Context
    kw.setdefault("rtol", 1e-13)
    kw.setdefault("max_iters", 3000)
    return Context(state.params, max_bricks=kw.pop("max_bricks", 4096),
                   max_particles=kw.pop("max_particles", 1 << 21), **kw)


def test_depth_first_init_bit_exact(golden):
    from make_golden import depth_world
    from mac_b200.world import first_init
    s = depth_world()
    ref = golden("d_ref_s0")
    with _ctx(s) as ctx:
        first_init(ctx, s)
        got = ctx.download()
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert all(v == 0.0 for v in e.values()), e


def test_depth_topology_bit_exact(golden):
    from mac_b200.state import INTERIOR
    s10 = golden("d_ref_s10")
    ref = golden("d_ref_t10")
    with _ctx(s10) as ctx:
        ctx.upload(s10)
        ctx.topology()
        got = ctx.download()
        st = ctx.stats()
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    assert got.params.dt == ref.params.dt
    ex = ref.exists.astype(bool)
    assert st["fluid_cells"] == ref.fluid_cells()
    assert (ex & (ref.type == INTERIOR)).sum() > 1000


def test_depth_steps(golden):
    s10 = golden("d_ref_s10")
    with _ctx(s10) as ctx:
        ctx.upload(s10)
        ctx.step()
        got = ctx.download()
        ref = golden("d_ref_s11")
        compare_topology(got, ref)
        e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
        assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
        compare_particles(got, ref, atol=1e-12)
        for _ in range(9):
            ctx.step()
        got = ctx.download()
    ref = golden("d_ref_s20")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= 1e-8 and max(e["u0x"], e["u0y"], e["u0z"]) <= 1e-9, e
    compare_particles(got, ref, atol=1e-10)


def test_deep_pool_depth_against_the_oracle(run_oracle):
    """64x64x48 box over a 36-cell pool: depths up to 18, so the inward BFS
    crosses several bricks and the relaxation needs several launches."""
    from mac_b200.state import INTERIOR, jet_world
    from mac_b200.world import first_init
    s = jet_world(nx=64, ny=64, nz=48, pool_depth=36, h=0.02)
    pr = s.params
    pr.depth_mode, pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube = 1, 7, 3, 5, 1
    with _ctx(s, max_bricks=8192, max_particles=1 << 22) as ctx:
        first_init(ctx, s)
        s0 = ctx.download()
        ctx.topology()
        got = ctx.download()
    want0, _ = run_oracle("firstinit", s)
    compare_topology(s0, want0)
    assert compare_particles(s0, want0) == 0.0
    want, _ = run_oracle("topology", s0)
    compare_topology(got, want)
    assert compare_particles(got, want) == 0.0
    ex = got.exists.astype(bool)
    assert got.depth[ex].max() >= 16
    assert (ex & (got.type == INTERIOR)).sum() > 50000
    assert got.nparticles < s0.nparticles  # deep interior particles were removed

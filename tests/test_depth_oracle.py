"""The oracle's depth composition pinned to the reference's own outputs.

The reference world built with the Interior cell type and Policy_Depth
(oracle/_ref/mac_ref_depth, the topology of test/Jet3.cpp:519-549) produced
the d_ref_* fixtures from a 24x24x32 jet over a 12-cell pool with
Policy_Depth(4, 3, 3) and the cube(1) refill. The restatement must reproduce:

* the first init and the per-step topology bit for bit: existence, material
  (Interior cells included), layer, depth, and the particle set after the
  removal of particles in interior cells deeper than the removal depth
  (src/Algorithms_Layer_Initial_With_Particle_Depth.h:26-47) and the cube
  refill of inflow and shallow interior cells
  (src/Algorithms_Create_Fluid_Particle_Depth.h:21-43);
* whole steps within solver rounding.
"""
import os
import sys

import numpy as np
import pytest

from compare import compare_particles, compare_topology, field_errors

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import depth_world  # noqa: E402

from mac_b200.state import INTERIOR  # noqa: E402


def _exact_fields(got, ref, fields):
    e = field_errors(got, ref, fields)
    assert all(v == 0.0 for v in e.values()), e


def test_depth_world_has_interior_cells_and_removal(golden):
    s0, s10 = golden("d_ref_s0"), golden("d_ref_s10")
    for s in (s0, s10):
        ex = s.exists.astype(bool)
        assert (ex & (s.type == INTERIOR)).sum() > 1000
        assert s.depth[ex].max() > s.params.depth_remove
    # particles in interior cells deeper than the removal depth are gone: fewer
    # particles than 8 per fluid cell of the initial pool
    assert s10.nparticles < s0.nparticles
    assert s0.params.depth_mode == 1 and s0.params.refill_cube == 1


def test_depth_first_init_bit_exact(golden, run_oracle):
    got, _ = run_oracle("firstinit", depth_world())
    ref = golden("d_ref_s0")
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    _exact_fields(got, ref, ("u0x", "u0y", "u0z", "p"))


def test_depth_topology_bit_exact(golden, run_oracle):
    got, _ = run_oracle("topology", golden("d_ref_s10"))
    ref = golden("d_ref_t10")
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    assert got.params.dt == ref.params.dt


def test_depth_steps_track_reference(golden, run_oracle):
    got, _ = run_oracle("step", golden("d_ref_s10"))
    ref = golden("d_ref_s11")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, ref, atol=1e-14)
    got, _ = run_oracle("step", golden("d_ref_s10"), n=10)
    ref = golden("d_ref_s20")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-10, e
    compare_particles(got, ref, atol=1e-11)


@pytest.mark.parametrize("planted", ["interior", "remove"])
def test_planted_depth_mistakes_are_caught(golden, run_oracle, planted):
    """The comparison sees a wrong Policy_Depth: the oracle run with a shifted
    interior or removal depth differs from the reference's topology."""
    s = golden("d_ref_s10")
    if planted == "interior":
        s.params.depth_interior += 1
    else:
        s.params.depth_remove += 1
    got, _ = run_oracle("topology", s)
    ref = golden("d_ref_t10")
    with pytest.raises(AssertionError):
        compare_topology(got, ref)
        assert compare_particles(got, ref) == 0.0
    assert not np.array_equal(got.pos.shape, ref.pos.shape) or planted == "interior"


# ------------------------------------------------------------ pipeline B
def _b_input(golden):
    s = golden("d_ref_s10")
    s.params.viscosity = 1e-3
    return s


def test_pipeline_b_init_bit_exact(golden, run_oracle):
    """The per-step init of test/Jet3.cpp:546 (depth topology, dt, extrapolation)."""
    got, _ = run_oracle("binit", _b_input(golden))
    ref = golden("b_ref_i10")
    compare_topology(got, ref)
    assert compare_particles(got, ref) == 0.0
    _exact_fields(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert got.params.dt == ref.params.dt


def test_pipeline_b_steps_track_reference(golden, run_oracle):
    """Algorithms_RungeKutta_all over grid and particles
    (src/Algorithms_RungeKutta_all.h:35-156) with the stage topology, the force
    projection and the extrapolation of the acceleration: one and five steps."""
    for n, name in ((1, "b_ref_s11"), (5, "b_ref_s15")):
        got, _ = run_oracle("bstep", _b_input(golden), n=n)
        ref = golden(name)
        compare_topology(got, ref)
        e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
        assert max(e.values()) <= 1e-12, (n, e)
        compare_particles(got, ref, atol=1e-13)
        assert got.params.t == ref.params.t

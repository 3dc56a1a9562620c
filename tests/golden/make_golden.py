"""Generates the committed golden fixtures from the reference's own code.

Run here, where the reference sources exist (oracle/Makefile builds
oracle/_ref/mac_ref from them). The outputs are compressed states of the
32x32x64 vertical-jet world (h = 0.05, inflow radius 4 at w = 1, LayerMax 4,
CFL 0.5) produced by the unmodified reference algorithms:

  c1_setup.npz         world as built (walls, inflow), before any pass
  c1_ref_setup.npz     after Solid_To_Const + Speed_Constant_Mirror
  c1_ref_s0.npz        after the reference's first init
  c1_ref_s30.npz       after 30 steps
  c1_ref_t30.npz       c1_ref_s30 after the per-step init (topology + dt)
  c1_ref_t30_<stage>.npz  c1_ref_t30 after one stage: forces, ode, project,
                       extrapolate, move, movelin
  c1_ref_s31.npz       one full step from c1_ref_s30
  c1_ref_s60.npz       after 60 steps from c1_ref_s0
  c1_ref_t30_csc.bin   the CSC system the reference assembled for the projection
                       of c1_ref_t30 (n, nnz, offset, indice, value, b, x)

Viscous fixtures (viscosity 1e-3 in the state header; the reference's
Algorithms_Viscosity and Algorithms_Solve_Pressure_Dirichlet with
Policy_Dirichlet_Boundary, composed as test/Lateral_jet_3.cpp does):

  c1_ref_t30v_<stage>.npz  c1_ref_t30 with viscosity after vforces, vproject, vode
  c1_ref_s31v.npz      one viscous step from c1_ref_s30 (with viscosity)
  c1_ref_s40v.npz      ten viscous steps from c1_ref_s30

Depth-composition fixtures (oracle/_ref/mac_ref_depth: the Interior cell type,
Policy_Depth(4, 3, 3) as test/Lateral_jet_3.cpp:494 and the reference's
Policy_Add_Particle_Cube(1) refill) of a 24x24x32 jet over a 12-cell pool
(``depth_world()``):

  d_ref_s0.npz         after the first init
  d_ref_s10.npz        after 10 steps
  d_ref_t10.npz        d_ref_s10 after the per-step init (depth topology + dt)
  d_ref_s11.npz        one step from d_ref_s10
  d_ref_s20.npz        ten steps from d_ref_s10

Pipeline-B fixtures (oracle/_ref/mac_ref_b: Algorithms_RungeKutta_all over the
depth world, test/Jet3.cpp:546-675, viscosity 1e-3), from d_ref_s10:

  b_ref_i10.npz        after the pipeline-B per-step init (depth topology, dt,
                       extrapolation)
  b_ref_s11.npz        one pipeline-B step
  b_ref_s15.npz        five pipeline-B steps

Usage: python tests/golden/make_golden.py [--viscous-only | --depth-only | --b-only]
"""
from __future__ import annotations

import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from mac_b200.state import State, jet_world  # noqa: E402
import oracle  # noqa: E402

STAGES = ["forces", "ode", "project", "extrapolate", "move", "movelin"]
VSTAGES = ["vforces", "vproject", "vode"]
VISCOSITY = 1e-3


def viscous(t, out):
    for name in ("t30", "s30"):
        s = State.load_npz(out("c1_ref_" + name))
        s.params.viscosity = VISCOSITY
        s.write(t(name + "v"))
    for st in VSTAGES:
        oracle.run_ref(st, t("t30v"), t("t30v_" + st))
        State.read(t("t30v_" + st)).save_npz(out("c1_ref_t30v_" + st))
    oracle.run_ref("vstep", t("s30v"), t("s31v"), 1)
    State.read(t("s31v")).save_npz(out("c1_ref_s31v"))
    oracle.run_ref("vstep", t("s30v"), t("s40v"), 10)
    State.read(t("s40v")).save_npz(out("c1_ref_s40v"))


def depth_world() -> State:
    """The depth fixtures' input: jet_world(24, 24, 32) over a 12-cell pool."""
    s = jet_world(nx=24, ny=24, nz=32, pool_depth=12)
    pr = s.params
    pr.depth_mode, pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube = 1, 4, 3, 3, 1
    return s


def depth(t, out):
    depth_world().write(t("dsetup"))
    oracle.run_ref("firstinit", t("dsetup"), t("ds0"))
    oracle.run_ref("step", t("ds0"), t("ds10"), 10)
    oracle.run_ref("topology", t("ds10"), t("dt10"))
    oracle.run_ref("step", t("ds10"), t("ds11"), 1)
    oracle.run_ref("step", t("ds10"), t("ds20"), 10)
    for name in ("s0", "s10", "t10", "s11", "s20"):
        State.read(t("d" + name)).save_npz(out("d_ref_" + name))


def pipeline_b(t, out):
    s = State.load_npz(out("d_ref_s10"))
    s.params.viscosity = VISCOSITY
    s.write(t("bs10"))
    oracle.run_ref("binit", t("bs10"), t("bi10"))
    oracle.run_ref("bstep", t("bs10"), t("bs11"), 1)
    oracle.run_ref("bstep", t("bs10"), t("bs15"), 5)
    for name in ("i10", "s11", "s15"):
        State.read(t("b" + name)).save_npz(out("b_ref_" + name))


def main():
    oracle.build()
    if not oracle.have_ref():
        raise SystemExit("oracle/_ref/mac_ref is not built (reference sources missing)")
    tmp = tempfile.mkdtemp()
    t = lambda n: os.path.join(tmp, n + ".state")
    out = lambda n: os.path.join(HERE, n + ".npz")
    if "--viscous-only" in sys.argv:
        viscous(t, out)
        print("viscous fixtures written to", HERE)
        return
    if "--depth-only" in sys.argv:
        depth(t, out)
        print("depth fixtures written to", HERE)
        return
    if "--b-only" in sys.argv:
        pipeline_b(t, out)
        print("pipeline-B fixtures written to", HERE)
        return
    s = jet_world()
    s.write(t("setup"))
    s.save_npz(out("c1_setup"))
    oracle.run_ref("setup", t("setup"), t("rsetup"))
    State.read(t("rsetup")).save_npz(out("c1_ref_setup"))
    oracle.run_ref("firstinit", t("setup"), t("s0"))
    State.read(t("s0")).save_npz(out("c1_ref_s0"))
    oracle.run_ref("step", t("s0"), t("s30"), 30)
    State.read(t("s30")).save_npz(out("c1_ref_s30"))
    oracle.run_ref("step", t("s30"), t("s31"), 1)
    State.read(t("s31")).save_npz(out("c1_ref_s31"))
    oracle.run_ref("step", t("s30"), t("s60"), 30)
    State.read(t("s60")).save_npz(out("c1_ref_s60"))
    oracle.run_ref("topology", t("s30"), t("t30"))
    State.read(t("t30")).save_npz(out("c1_ref_t30"))
    for st in STAGES:
        oracle.run_ref(st, t("t30"), t("t30_" + st))
        State.read(t("t30_" + st)).save_npz(out("c1_ref_t30_" + st))
    oracle.run_ref("csc", t("t30"), t("junk"), os.path.join(HERE, "c1_ref_t30_csc.bin"))
    viscous(t, out)
    depth(t, out)
    pipeline_b(t, out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""The C++ drop-in layer (include/mac_gpu/Mac_GPU.h) inside the reference's own
world: oracle/_ref/mac_ref_gpu composes the unmodified reference headers and
swaps in (a) Policy_Solve_Linear_GPU as the solver policy of the reference's
Algorithms_Solve_Pressure, (b) Algorithms_Step_GPU + Algorithms_To_Host_GPU for
the pipeline-A step, (c) Algorithms_Solve_Pressure_GPU as the projection the
reference's own RK2-TVD and Algorithms_Do_Pressure call through
Init_Iteration / Divergence_Projection / End_Iteration. oracle/_ref/mac_ref_b_gpu is the depth world of
test/Jet3.cpp (interior cells, depth chunk, three speed buffers) whose
Algorithms_Step_GPU runs pipeline B: the session carries the interior material
and the depths across. Results are compared with the reference's own outputs
(committed fixtures) at the tolerances of the device parity tests.

The binary is built from the reference sources by oracle/Makefile (target
ref_gpu) on a machine that has them; where it is absent the tests skip.
"""
import os
import subprocess

import pytest

from compare import compare_particles, compare_topology, field_errors

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "oracle", "_ref", "mac_ref_gpu")
P_TOL = 1e-9
U_TOL = 1e-10


BIN_B = os.path.join(HERE, "..", "oracle", "_ref", "mac_ref_b_gpu")


def _run(cmd, state, tmp_path, n=None, rtol="1e-13", binary=BIN):
    from mac_b200.state import State
    if not os.path.exists(binary):
        pytest.skip(f"{os.path.basename(binary)} is not built (needs the reference sources)")
    src, dst = str(tmp_path / "in.state"), str(tmp_path / "out.state")
    state.write(src)
    args = [binary, cmd, src, dst] + ([str(n)] if n is not None else [])
    out = subprocess.run(args, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, MAC_REF_RTOL=rtol))
    assert out.returncode == 0, out.stderr + out.stdout
    assert "mac_gpu:" not in out.stdout, out.stdout
    return State.read(dst)


def test_reference_projection_with_device_solver_policy(golden, tmp_path):
    got = _run("gpuproject", golden("c1_ref_t30"), tmp_path, rtol="1e-14")
    ref = golden("c1_ref_t30_project")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e


def test_reference_rk2tvd_with_device_projection(golden, tmp_path):
    """The reference's own Algorithms_RungeKutta_RK2_TVD (host loops over the
    speed buffers, Init_Iteration / Divergence_Projection / End_Iteration
    through Policy::) composed with Algorithms_Solve_Pressure_GPU."""
    got = _run("gpuode", golden("c1_ref_t30"), tmp_path, rtol="1e-14")
    ref = golden("c1_ref_t30_ode")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z", "u1x", "u1y", "u1z"))
    assert e["p"] <= P_TOL, e
    assert max(e[k] for k in ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z")) <= U_TOL, e


def test_reference_do_pressure_with_device_projection(golden, tmp_path):
    got = _run("gpudopressure", golden("c1_ref_t30"), tmp_path, rtol="1e-14")
    ref = golden("c1_ref_t30_project")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e


def test_reference_world_steps_on_device(golden, tmp_path):
    got = _run("gpustep", golden("c1_ref_s30"), tmp_path, n=1)
    ref = golden("c1_ref_s31")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    compare_particles(got, ref, atol=1e-12)
    assert abs(got.params.t - ref.params.t) <= 1e-15
    assert got.params.step == ref.params.step


def test_reference_depth_world_runs_pipeline_b_on_device(golden, tmp_path):
    s = golden("d_ref_s10")
    s.params.viscosity = 1e-3
    got = _run("gpustep", s, tmp_path, n=1, binary=BIN_B)
    ref = golden("b_ref_s11")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("p", "u0x", "u0y", "u0z"))
    assert e["p"] <= P_TOL and max(e["u0x"], e["u0y"], e["u0z"]) <= U_TOL, e
    compare_particles(got, ref, atol=1e-12)
    assert abs(got.params.t - ref.params.t) <= 1e-15

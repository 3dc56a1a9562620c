"""The oracle (C restatement) against the reference's own outputs.

The fixtures under tests/golden were produced by the unmodified reference
algorithms compiled from their headers (tests/golden/make_golden.py). From the
same input state the oracle must agree bit for bit on everything that does
not go through the linear solve, and within solver rounding on the rest (both
solve to a relative residual of 1e-14).
"""
import numpy as np
import pytest

from compare import compare_particles, compare_topology, field_errors, max_abs_diff

ALL = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")


def _exact(a, b, fields=ALL):
    d = max_abs_diff(a, b, fields, existing_only=False)
    assert all(v == 0.0 for v in d.values()), d


def test_topology_bit_exact(golden, run_oracle):
    got, st = run_oracle("topology", golden("c1_ref_s30"))
    ref = golden("c1_ref_t30")
    compare_topology(got, ref)
    _exact(got, ref)
    assert compare_particles(got, ref) == 0.0
    assert got.params.dt == ref.params.dt
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("stage,fields", [("forces", ("ax", "ay", "az")),
                                          ("extrapolate", ("u0x", "u0y", "u0z"))])
def test_stencil_stages_bit_exact(golden, run_oracle, stage, fields):
    got, st = run_oracle(stage, golden("c1_ref_t30"))
    ref = golden("c1_ref_t30_" + stage)
    compare_topology(got, ref)
    _exact(got, ref)
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("stage,sym", [("move", 1), ("movelin", 0)])
def test_particle_moves_bit_exact(golden, run_oracle, stage, sym):
    s = golden("c1_ref_t30")
    got, st = run_oracle(stage, s)
    ref = golden("c1_ref_t30_" + stage)
    assert compare_particles(got, ref) == 0.0
    assert st["invalid_reads"] == 0


@pytest.mark.parametrize("stage", ["project", "ode"])
def test_solver_stages_within_rounding(golden, run_oracle, stage):
    got, st = run_oracle(stage, golden("c1_ref_t30"))
    ref = golden("c1_ref_t30_" + stage)
    compare_topology(got, ref)
    e = field_errors(got, ref, ALL)
    assert max(e.values()) <= 1e-12, e
    assert st["relres"] <= 1e-14
    assert st["max_div"] <= 1e-10


def test_full_step(golden, run_oracle):
    got, _ = run_oracle("step", golden("c1_ref_s30"))
    ref = golden("c1_ref_s31")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, ref, atol=1e-14)


def test_first_init_bit_exact(golden, run_oracle):
    got, _ = run_oracle("firstinit", golden("c1_setup"))
    ref = golden("c1_ref_s0")
    compare_topology(got, ref)
    _exact(got, ref)
    assert compare_particles(got, ref) == 0.0


def test_thirty_steps_track_reference(golden, run_oracle):
    """Thirty consecutive steps from the first init: the topology stays
    identical and the fields within solver rounding of the reference run."""
    got, _ = run_oracle("step", golden("c1_ref_s0"), n=30)
    ref = golden("c1_ref_s30")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-9, e
    assert got.nparticles == ref.nparticles


def test_setup_passes_match_reference(golden):
    from mac_b200.world import setup_passes
    got = setup_passes(golden("c1_setup"))
    ref = golden("c1_ref_setup")
    compare_topology(got, ref)
    _exact(got, ref)


def test_cg_stand_in_matches_direct_solve():
    """Pins the Umfpack stand-in: the CSC system the reference assembled, solved
    by a sparse direct LU, against the CG solution the reference stored."""
    import os

    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    from conftest import GOLDEN
    raw = open(os.path.join(GOLDEN, "c1_ref_t30_csc.bin"), "rb").read()
    off = 0
    checked = 0
    while off < len(raw):
        n, nnz = np.frombuffer(raw, dtype="<i8", count=2, offset=off)
        off += 16
        ptr = np.frombuffer(raw, dtype="<i4", count=n + 1, offset=off); off += 4 * (n + 1)
        ind = np.frombuffer(raw, dtype="<i4", count=nnz, offset=off); off += 4 * nnz
        val = np.frombuffer(raw, dtype="<f8", count=nnz, offset=off); off += 8 * nnz
        b = np.frombuffer(raw, dtype="<f8", count=n, offset=off); off += 8 * n
        x = np.frombuffer(raw, dtype="<f8", count=n, offset=off); off += 8 * n
        A = sp.csc_matrix((val, ind, ptr), shape=(n, n))
        assert abs(A - A.T).max() == 0.0  # the assembled operator is symmetric
        xd = spla.spsolve(A, b)
        err = np.linalg.norm(x - xd) / np.linalg.norm(xd)
        assert err <= 1e-10, err
        checked += 1
    assert checked >= 1


# ------------------------------------------------- viscosity (Dirichlet pressure)
def _viscous(golden, name, nu=1e-3):
    s = golden(name)
    s.params.viscosity = nu
    return s


def test_viscous_forces_bit_exact(golden, run_oracle):
    """Algorithms<Gravity, Convection, Viscosity> (src/Algorithms_Viscosity.h:24-30)."""
    got, st = run_oracle("vforces", _viscous(golden, "c1_ref_t30"))
    ref = golden("c1_ref_t30v_vforces")
    compare_topology(got, ref)
    _exact(got, ref)
    assert st["invalid_reads"] == 0
    plain = golden("c1_ref_t30_forces")
    assert max_abs_diff(got, plain, ("ax", "ay", "az"))["az"] > 1e-3  # the viscous term is there


@pytest.mark.parametrize("stage", ["vproject", "vode"])
def test_viscous_solver_stages_within_rounding(golden, run_oracle, stage):
    """Algorithms_Solve_Pressure_Dirichlet with Policy_Dirichlet_Boundary
    (src/Algorithms_Solve_Pressure_Dirichlet.h:171-233, src/Policy_Dirichlet_Boundary.h:27-109)."""
    got, st = run_oracle(stage, _viscous(golden, "c1_ref_t30"))
    ref = golden("c1_ref_t30v_" + stage)
    compare_topology(got, ref)
    e = field_errors(got, ref, ALL)
    assert max(e.values()) <= 1e-12, e
    assert st["relres"] <= 1e-14


def test_viscous_steps_track_reference(golden, run_oracle):
    got, _ = run_oracle("vstep", _viscous(golden, "c1_ref_s30"))
    ref = golden("c1_ref_s31v")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-12, e
    compare_particles(got, ref, atol=1e-14)
    got, _ = run_oracle("vstep", _viscous(golden, "c1_ref_s30"), n=10)
    ref = golden("c1_ref_s40v")
    compare_topology(got, ref)
    e = field_errors(got, ref, ("u0x", "u0y", "u0z", "p"))
    assert max(e.values()) <= 1e-10, e

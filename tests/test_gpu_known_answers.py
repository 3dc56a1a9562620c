"""Known answers of the reference's own tests on the device path (through the
C-ABI), on the small worlds test_known_answers.py builds for the oracle:

* upwind convection -1.25 at the corner of a diagonal speed step
  (test/old/TestPolicy_Upwind_1_Order.h:214-215), through the force kernel
  with gravity 0;
* RK4 particle moves 0.1 / 0.01 in a uniform unit field
  (test/old/TestAlgorithms_Move_Particles.h:159-567);
* the projection of a five-cell plus, 1.25 / 0.2499999999999998890 / 0.75
  (test/old/TestAlgorithms_Solve_Pressure.h:449-470), with every solver form.
"""
import numpy as np
import pytest

from mac_b200.state import FLUID, Params
from test_known_answers import _at, _cells

pytestmark = pytest.mark.gpu


def _ctx(state, **kw):
    from mac_b200.gpu import Context
    kw.setdefault("rtol", 1e-13)
    kw.setdefault("max_iters", 500)
    return Context(state.params, max_bricks=256, max_particles=1024, **kw)


def test_upwind_diagonal_on_device():
    cells = {(x, y, z): (FLUID, 0, (0.0, 0.0, 0.0)) for x in range(3) for y in range(3) for z in (-1, 0, 1)}
    cells[(1, 1, 0)] = (FLUID, 0, (1.0, 1.0, 0.0))
    s = _cells(cells, Params(h=(1.0, 1.0, 1.0), gravity=0.0))
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.forces(0)
        got = ctx.download()
    assert abs(_at(got, (1, 1, 0), "ax") - (-1.25)) < 1e-12
    assert abs(_at(got, (1, 1, 0), "ay") - (-1.25)) < 1e-12


@pytest.mark.parametrize("sym", [0, 1])
@pytest.mark.parametrize("h,dt,want", [(1.0, 0.1, 0.1), (0.1, 0.01, 0.01)])
def test_particle_moves_on_device(sym, h, dt, want):
    cells = {(x, y, z): (FLUID, 0, (1.0, 1.0, 1.0))
             for x in range(-2, 3) for y in range(-2, 3) for z in range(-2, 3)}
    s = _cells(cells, Params(h=(h, h, h), gravity=0.0, dt=dt, interp_symmetric=sym))
    s.pos = np.zeros((1, 3))
    with _ctx(s) as ctx:
        ctx.upload(s)
        ctx.move()
        got = ctx.download()
    assert np.allclose(got.pos[0], [want, want, want], rtol=0, atol=1e-10), got.pos[0]


@pytest.mark.parametrize("solver", ["mgpcg64", "mixed", "cg64"])
def test_projection_plus_on_device(solver):
    plus = {(0, 0): (2.0, 2.0), (1, 0): (1.0, 1.0), (-1, 0): (1.0, 1.0), (0, 1): (1.0, 1.0), (0, -1): (1.0, 1.0)}
    cells = {}
    for x in range(-2, 3):
        for y in range(-2, 3):
            u = plus.get((x, y))
            cells[(x, y, 0)] = (FLUID if u else 0, 4, (u[0], u[1], 0.0) if u else (0.0, 0.0, 0.0))
            cells[(x, y, -1)] = (2, 0, (0.0, 0.0, 0.0))
            cells[(x, y, 1)] = (2, 4, (0.0, 0.0, 0.0))
    s = _cells(cells, Params(h=(1.0, 1.0, 1.0), gravity=0.0))
    with _ctx(s, solver=solver) as ctx:
        ctx.upload(s)
        ctx.project(0)
        got = ctx.download()
    want = {(0, 0): (1.25, 1.25), (1, 0): (1.25, 0.24999999999999988898), (0, 1): (0.24999999999999988898, 1.25),
            (-1, 0): (0.75, 0.75), (0, -1): (0.75, 0.75)}
    for (x, y), (wx, wy) in want.items():
        assert abs(_at(got, (x, y, 0), "u0x") - wx) < 1e-10, (solver, x, y)
        assert abs(_at(got, (x, y, 0), "u0y") - wy) < 1e-10, (solver, x, y)
    assert abs(_at(got, (0, 0, 0), "p") - 1.0) < 1e-10

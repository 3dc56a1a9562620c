"""Standalone pressure solve on the 128^3 pool + 12 spheres world (solid box,
air above, face speeds uniform in [-1, 1]): the device projection with the
plain FP64 MG-PCG and with the mixed form (FP32 multigrid inside FP64 CG),
each with one and with two Jacobi sweeps around the finest level's coarse
correction,
against the oracle's FP64 projection (CG to a relative residual of 1e-14) of
the same world.

Tolerances: solved to 1e-12 both forms must give pressure within 1e-9 and
velocities within 1e-10 (relative L2); at the config's own 1e-10 the errors
are reported and bounded by 1e-8 / 1e-9.
"""
import numpy as np
import pytest

from compare import field_errors

N = 128


@pytest.fixture(scope="module")
def pool_world():
    from mac_b200.state import pool_spheres_world
    from mac_b200.world import setup_passes
    return setup_passes(pool_spheres_world(N))


def test_world_shape(pool_world):
    from mac_b200.state import AIR, FLUID, SOLID
    s = pool_world
    ex = s.exists.astype(bool)
    ck = s.cell_keys()[ex]
    t = s.type[ex]
    # the set-up passes create +e_i neighbours beyond the far shell (as grid[key] does)
    assert ck.min() == -1 and ck.max() == N + 2
    inner = (ck.min(axis=1) >= 0) & (ck.max(axis=1) < N)
    shell = ~inner & (ck.max(axis=1) <= N)
    assert np.all(t[shell] == SOLID) and np.all(t[inner] != SOLID)
    assert np.all(t[~inner & ~shell] == AIR)
    nf = int((t == FLUID).sum())
    assert 0.8e6 <= nf <= 1.0e6, nf
    assert int((t[inner] == AIR).sum()) + nf == N ** 3
    # the faces between the shell and the open cells are const (Neumann)
    fl = s.flags[ex]
    assert np.all(fl[(ck[:, 0] == 0) & inner] & 1)
    assert np.all(fl[(ck[:, 2] == N) & (ck[:, 0] >= 0) & (ck[:, 0] < N) & (ck[:, 1] >= 0) & (ck[:, 1] < N)] & 4)


@pytest.fixture(scope="module")
def oracle_projection(pool_world, tmp_path_factory):
    import oracle
    from mac_b200.state import State
    d = tmp_path_factory.mktemp("pool")
    pool_world.write(str(d / "in.state"))
    stats = oracle.run_oracle("project", str(d / "in.state"), str(d / "out.state"), 1, 1e-14)
    assert stats["relres"] <= 1e-14
    return State.read(str(d / "out.state"))


@pytest.mark.gpu
@pytest.mark.parametrize("sweeps", [1, 2])
@pytest.mark.parametrize("solver", ["mgpcg64", "mixed"])
@pytest.mark.parametrize("rtol,p_tol,u_tol", [(1e-12, 1e-9, 1e-10), (1e-10, 1e-8, 1e-9)])
def test_pool_projection_against_oracle(pool_world, oracle_projection, solver, rtol, p_tol, u_tol, sweeps):
    from mac_b200.gpu import Context
    with Context(pool_world.params, max_bricks=8192, max_particles=1024, solver=solver, rtol=rtol,
                 max_iters=500) as ctx:
        ctx.set_multigrid(sweeps)
        ctx.upload(pool_world)
        ctx.project(0)
        st = ctx.stats()
        got = ctx.download()
    e = field_errors(got, oracle_projection, ("p", "u0x", "u0y", "u0z"))
    print(f"{solver} sweeps {sweeps} rtol {rtol:g}: iterations {st['iterations']}, relres {st['relres']:.2e}, errors {e}")
    assert st["relres"] <= rtol
    assert e["p"] <= p_tol, e
    assert max(e["u0x"], e["u0y"], e["u0z"]) <= u_tol, e

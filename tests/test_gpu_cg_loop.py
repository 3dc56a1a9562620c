"""Where the pressure solve's CG loop stops, on a 64^3 pool + spheres world.

The multigrid forms apply each iteration's update x += alpha p, r -= alpha q
and its convergence test inside the next V-cycle's first kernel, read the
done flag one iteration late and, near convergence, test right after that
kernel; the Jacobi-CG form keeps one host read per iteration. In every form a
cap of k iterations stops the solve after exactly k updates of x, more
iterations bring the iterate closer to the converged one, and a right-hand
side of zero takes no iteration and leaves the pressure at zero.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 64


@pytest.fixture(scope="module")
def pool64():
    from mac_b200.state import pool_spheres_world
    from mac_b200.world import setup_passes
    return setup_passes(pool_spheres_world(N, r_range=(6.0 * N / 128, 20.0 * N / 128)))


def _ctx(s, solver, rtol, max_iters, sweeps=2, prefetch=False):
    from mac_b200.gpu import Context
    c = Context(s.params, max_bricks=int(s.nbricks * 1.2) + 64, max_particles=1024, solver=solver, rtol=rtol,
                max_iters=max_iters)
    c.set_multigrid(sweeps, prefetch)
    return c


@pytest.mark.parametrize("solver,sweeps,prefetch", [("mixed", 2, False), ("mgpcg64", 2, False), ("cg64", 2, False),
                                                    ("mixed", 1, False), ("mgpcg64", 1, False), ("mixed", 2, True),
                                                    ("mixed", 1, True)])
@pytest.mark.parametrize("cap", [1, 2, 5])
def test_iteration_cap_is_exact(pool64, solver, sweeps, prefetch, cap):
    with _ctx(pool64, solver, 1e-14, cap, sweeps, prefetch) as ctx:
        ctx.upload(pool64)
        ctx.project(0, allow_not_converged=True)
        st = ctx.stats()
    assert st["iterations"] == cap
    assert st["relres"] > 1e-14


@pytest.mark.parametrize("solver,sweeps", [("mixed", 2), ("mgpcg64", 2), ("mixed", 1)])
def test_capped_solves_approach_the_converged_one(pool64, solver, sweeps):
    """More iterations bring the pressure closer to the converged solve's (the
    capped solves' iterates are the loop's own, not ones a late stop skipped)."""
    ps = []
    for cap in (3, 6, 9, 200):
        with _ctx(pool64, solver, 1e-12, cap, sweeps) as ctx:
            ctx.upload(pool64)
            ctx.project(0, allow_not_converged=True)
            got = ctx.download()
        ex = got.exists.astype(bool)
        ps.append(got.f64["p"][ex].copy())
    ref = ps[-1]
    err = [float(np.linalg.norm(p - ref) / np.linalg.norm(ref)) for p in ps[:-1]]
    assert err[0] > err[1] > err[2], err
    assert err[2] < 1e-3, err


@pytest.mark.parametrize("solver", ["mixed", "mgpcg64", "cg64"])
def test_zero_rhs_takes_no_iteration(pool64, solver):
    z = copy.copy(pool64)
    z.f64 = {k: (np.zeros_like(v) if k.startswith("u") else v) for k, v in pool64.f64.items()}
    with _ctx(z, solver, 1e-10, 100) as ctx:
        ctx.upload(z)
        ctx.project(0)
        st = ctx.stats()
        got = ctx.download()
    assert st["iterations"] == 0
    ex = got.exists.astype(bool)
    assert np.all(got.f64["p"][ex] == 0.0)


@pytest.mark.parametrize("solver,sweeps", [("mixed", 1), ("mixed", 2), ("mgpcg64", 2)])
def test_prefetching_first_kernel_matches_one_block_per_brick(pool64, solver, sweeps):
    """The V-cycle's first kernel run as resident blocks prefetching bricks
    with asynchronous bulk copies computes what the one-block-per-brick kernel
    computes (only the r.r partials are summed in another grouping): the same
    iteration count within one and the same pressure within 1e-10."""
    out = []
    for prefetch in (True, False):
        with _ctx(pool64, solver, 1e-10, 500, sweeps) as ctx:
            ctx.set_multigrid(sweeps, prefetch)
            ctx.upload(pool64)
            ctx.project(0)
            st = ctx.stats()
            got = ctx.download()
        ex = got.exists.astype(bool)
        out.append((st["iterations"], got.f64["p"][ex].copy()))
    (i1, p1), (i0, p0) = out
    assert abs(i1 - i0) <= 1, (i1, i0)
    assert np.linalg.norm(p1 - p0) / np.linalg.norm(p0) <= 1e-10


def test_smoother_settings(pool64):
    """mac_set_smoother: weights whose two-sweep damping leaves (-1, 1) on
    (0, 2] are refused; other weights and coarse scales change the iteration
    count, not the answer (pressure within 1e-9 of the default settings' at a
    relative residual of 1e-12)."""
    from mac_b200.gpu import MacError
    out = []
    for w1, w2, scale in ((0.5711, 1.8216, 0.6), (0.9, 0.9, 0.6), (0.548, 1.025, 0.7)):
        with _ctx(pool64, "mixed", 1e-12, 500) as ctx:
            ctx.set_smoother(w1, w2, 0.9, scale)
            ctx.upload(pool64)
            ctx.project(0)
            got = ctx.download()
            out.append((ctx.stats()["iterations"], got.f64["p"][got.exists.astype(bool)].copy()))
    for its, p in out[1:]:
        assert np.linalg.norm(p - out[0][1]) / np.linalg.norm(out[0][1]) <= 1e-9
    with _ctx(pool64, "mixed", 1e-12, 500) as ctx:
        for bad in ((1.2, 1.2, 0.9, 0.6), (0.9, 0.9, 1.0, 0.6), (0.9, 0.9, 0.9, 1.5), (0.0, 0.9, 0.9, 0.6),
                    (0.3, 4.0, 0.9, 0.6)):
            with pytest.raises(MacError):
                ctx.set_smoother(*bad)


@pytest.mark.parametrize("max_cells", [64, 1 << 30])
def test_coarse_block_split(pool64, max_cells):
    """Dense multigrid levels moved between the device-wide sweeps and the
    one-block coarse solve (every dense level but the coarsest device-wide,
    or all in the block): the same solve to within the tolerance, with about
    the same number of iterations."""
    out = []
    for mc in (1024, max_cells):
        with _ctx(pool64, "mixed", 1e-12, 500) as ctx:
            ctx.set_coarse_block(mc)
            ctx.upload(pool64)
            ctx.project(0)
            got = ctx.download()
            out.append((ctx.stats()["iterations"], got.f64["p"][got.exists.astype(bool)].copy()))
    assert abs(out[1][0] - out[0][0]) <= 2, (out[0][0], out[1][0])
    assert np.linalg.norm(out[1][1] - out[0][1]) / np.linalg.norm(out[0][1]) <= 1e-9

"""The learned preconditioner inside the projection (flexible CG, solver
"learned"): a network trained on the device for a few hundred steps on CG
pairs from random 32^3 masks is used on a held-out 64^3 pool + spheres world.

Checks: the solve reaches the requested relative residual and the pressure
matches the oracle's FP64 projection (relative L2 <= 1e-9 at rtol 1e-12); a
network that makes no progress stalls and the MG-PCG fall-back still converges.
"""
import numpy as np
import pytest

from compare import field_errors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world():
    from mac_b200.state import pool_spheres_world
    from mac_b200.world import setup_passes
    return setup_passes(pool_spheres_world(64, r_range=(3.0, 10.0), seed=5, vel_seed=6))


@pytest.fixture(scope="module")
def oracle_p(world, tmp_path_factory):
    import oracle
    from mac_b200.state import State
    d = tmp_path_factory.mktemp("learned")
    world.write(str(d / "in.state"))
    oracle.run_oracle("project", str(d / "in.state"), str(d / "out.state"), 1, 1e-14)
    return State.read(str(d / "out.state"))


@pytest.fixture(scope="module")
def trained():
    from mac_b200.unet import UNet
    net = UNet(0, seed=3)
    net.set_loss("energy")
    net.make_dataset(nmasks=64, size=32, nsnap=8, niter=800, seed=11)
    losses = net.train(300, batch=8, lr=1e-3, seed=5)
    assert losses[-20:].mean() < 0.5 * losses[:20].mean(), (losses[:20].mean(), losses[-20:].mean())
    yield net
    net.close()


def _solve(world, solver, rtol, net=None):
    from mac_b200.gpu import Context
    with Context(world.params, max_bricks=2048, max_particles=1024, solver=solver, rtol=rtol, max_iters=2000) as ctx:
        if net is not None:
            ctx.set_preconditioner(net)
        ctx.upload(world)
        ctx.project(0)
        st = ctx.stats()
        return st, ctx.download()


def test_learned_solve_converges_to_the_oracle(world, oracle_p, trained):
    st, got = _solve(world, "learned", 1e-12, trained)
    e = field_errors(got, oracle_p, ("p", "u0x", "u0y", "u0z"))
    print("learned:", st["iterations"], "iterations,", st["learned_iterations"], "with the network,",
          st["fallbacks"], "fall-backs; errors", e)
    assert st["relres"] <= 1e-12
    assert e["p"] <= 1e-9 and max(e["u0x"], e["u0y"], e["u0z"]) <= 1e-10, e


def test_stalled_network_falls_back(world, oracle_p):
    from mac_b200.unet import UNet
    with UNet(0) as net:
        net.set_params(np.zeros(net.nparams, np.float32), 1.0)  # z = 0 before smoothing
        from mac_b200.gpu import Context
        with Context(world.params, max_bricks=2048, max_particles=1024, solver="learned", rtol=1e-12,
                     max_iters=2000) as ctx:
            ctx.set_preconditioner(net)
            ctx.set_learned_smoothing(0.0)  # so z = 0: no progress at all
            ctx.upload(world)
            ctx.project(0)
            st = ctx.stats()
            got = ctx.download()
    assert st["relres"] <= 1e-12
    assert st["fallbacks"] >= 1
    e = field_errors(got, oracle_p, ("p",))
    assert e["p"] <= 1e-9, e

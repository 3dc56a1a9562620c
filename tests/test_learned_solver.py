"""The learned preconditioner inside the projection (flexible CG, solver
"learned") with the committed trained network, on a 64^3 pool + spheres world
that was not in its training set.

Checks: the solve reaches the requested relative residual and the pressure
matches the oracle's FP64 projection (relative L2 <= 1e-9 at rtol 1e-12); to
1e-8 the network needs at most 40 iterations without falling back, under a
quarter of Jacobi-PCG's, while the same loop with the network switched off
stalls; a network that makes no progress at all falls back to MG-PCG, which
still converges.
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
    """The committed network (mac_b200/weights/unet_pool64.npz, trained by
    mac_b200.train_preconditioner on 2000 random masks at 64^3, none of them
    the test world)."""
    import os

    from mac_b200.unet import UNet
    path = os.path.join(os.path.dirname(__file__), "..", "mac_b200", "weights", "unet_pool64.npz")
    net = UNet(0)
    net.load(path)
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


def test_network_cuts_iterations(world, trained):
    """What the trained network gains over the same flexible CG without it
    (network output zero: its Jacobi step alone) and over Jacobi-PCG."""
    from mac_b200.gpu import Context
    from mac_b200.unet import UNet

    def run(net, omega, solver="learned"):
        with Context(world.params, max_bricks=2048, max_particles=1024, solver=solver, rtol=1e-8,
                     max_iters=2000) as ctx:
            ctx.set_preconditioner(net)
            ctx.set_learned_smoothing(omega)
            ctx.upload(world)
            ctx.project(0)
            return ctx.stats()

    st_l = run(trained, 0.8)
    with UNet(0) as zero:
        zero.set_params(np.zeros(zero.nparams, np.float32), 1.0)
        st_0 = run(zero, 0.8)
    st_j = run(None, 0.8, "cg64")
    print("to 1e-8: learned", st_l["iterations"], "network off", st_0["iterations"],
          "(fall-back", st_0["fallbacks"], ") Jacobi-PCG", st_j["iterations"])
    assert st_l["fallbacks"] == 0 and st_l["learned_iterations"] == st_l["iterations"]
    assert st_l["iterations"] <= 40
    assert st_l["iterations"] < 0.25 * st_j["iterations"]
    assert st_0["fallbacks"] >= 1  # without the network the same loop stalls


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

"""Slab decomposition for a sharded step (host side, mac_b200/shard.py): the
plan partitions the bricks and particles, and the ghost exchange and particle
migration give every rank what the owners hold, with two gloo ranks on CPU.
"""
import os
import random
import sys

import numpy as np
import pytest

ROOT = os.path.join(os.path.dirname(__file__), "..")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c1_ref_s30.npz")


def _world():
    from mac_b200.state import State
    return State.load_npz(GOLDEN)


@pytest.mark.parametrize("nranks", [2, 3])
def test_plan_partitions_bricks_and_particles(nranks):
    from mac_b200.shard import SlabPlan
    s = _world()
    plan = SlabPlan.balanced(s, nranks)
    assert plan.nranks == nranks and np.all(plan.z_hi > plan.z_lo)
    assert np.all(plan.z_lo[1:] == plan.z_hi[:-1])
    owned_total, parts = 0, []
    keyset = {tuple(k) for k in s.keys.tolist()}
    for r in range(nranks):
        loc = plan.local(s, r)
        kz = loc.state.keys[:, 2]
        owned_total += int(loc.owned.sum())
        assert np.all((kz[loc.owned] >= plan.z_lo[r]) | (r == 0))
        assert np.all((kz[loc.owned] < plan.z_hi[r]) | (r == nranks - 1))
        ghosts = loc.state.keys[~loc.owned]
        # every brick one layer outside the slab is a ghost, and nothing else is
        want = {k for k in keyset if k[2] in (plan.z_lo[r] - 1, plan.z_hi[r])}
        assert {tuple(k) for k in ghosts.tolist()} == want
        parts.append(loc.state.pos)
        assert np.all(plan.particle_owner(s, loc.state.pos) == r)
    assert owned_total == s.nbricks
    allpos = np.concatenate(parts)
    assert len(allpos) == s.nparticles
    # fluid cells are balanced to within the fluid of one brick layer
    from mac_b200.state import FLUID_TYPES
    isfl = np.isin(s.type, FLUID_TYPES) & (s.exists != 0)
    per_layer = np.bincount(s.keys[:, 2] - s.keys[:, 2].min(), weights=isfl.sum(axis=1))
    fluid = []
    for r in range(nranks):
        loc = plan.local(s, r)
        f = np.isin(loc.state.type, FLUID_TYPES) & (loc.state.exists != 0)
        fluid.append(int(f[loc.owned].sum()))
    assert sum(fluid) == int(isfl.sum())
    assert max(fluid) - min(fluid) <= per_layer.max(), (fluid, per_layer.max())


def _mark(key, rank):
    # a value per cell that says which brick and which owner wrote it
    return key[:, 2:3] * 1e4 + key[:, 1:2] * 1e2 + key[:, 0:1] + np.arange(512)[None, :] * 1e-4 + (rank + 1) * 1e6


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    from mac_b200.shard import SlabPlan, exchange_ghosts, migrate_particles
    from mac_b200.state import BRICK, State
    s = State.load_npz(GOLDEN)
    plan = SlabPlan.balanced(s, world)
    loc = plan.local(s, rank)
    st = loc.state
    st.f64["u0x"][loc.owned] = _mark(st.keys[loc.owned], rank)
    st.layer[loc.owned] = 10 + rank
    n = exchange_ghosts(loc, plan)
    ghost_ok = True
    g = ~loc.owned
    owner = plan.owner(st.keys[g, 2])
    for i, o in zip(np.flatnonzero(g), owner):
        ghost_ok &= bool(np.array_equal(st.f64["u0x"][i], _mark(st.keys[i:i + 1], int(o))[0]))
        ghost_ok &= bool(np.all(st.layer[i] == 10 + int(o)))
    # every particle moves 0.6 brick up (those of the top rank stay in its
    # open-ended slab), then migrates to its new owner
    dz = 0.6 * BRICK * s.params.h[2]
    st.pos = st.pos + np.array([0.0, 0.0, dz])
    recv = migrate_particles(loc, plan)
    mine_ok = bool(np.all(plan.particle_owner(st, st.pos) == rank))
    q.put((rank, n, int(g.sum()), ghost_ok, recv, mine_ok, st.pos.copy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ghost_exchange_and_migration_gloo(world):
    """Two ranks, and three (the middle rank exchanges with both sides)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    s = _world()
    from mac_b200.state import BRICK
    for rank, n, nghost, ghost_ok, recv, mine_ok, _ in res:
        assert n == nghost and nghost > 0, (rank, n, nghost)
        assert ghost_ok, rank
        assert mine_ok, rank
    assert sum(r[4] for r in res) > 0  # particles crossed a slab boundary
    got = np.concatenate([r[6] for r in res])
    want = s.pos + np.array([0.0, 0.0, 0.6 * BRICK * s.params.h[2]])
    key = lambda a: a[np.lexsort(a.T[::-1])]
    assert len(got) == len(want)
    assert np.array_equal(key(got), key(want))

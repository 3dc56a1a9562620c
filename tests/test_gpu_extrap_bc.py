"""Algorithm_Extrapolate_Boundary_Condition (3D form) on the device
(mac_extrapolate_boundary_condition) against the oracle's restatement in the
same fixed order (command extrapbc: boundary cells by colour x, y, z mod 5),
every speed face of every existing cell bit for bit, NaN where NaN. The
oracle's restatement is itself pinned to the reference's own 3D form on
single-chunk worlds and to the 565 known answers of its 2D test
(tests/test_extrapolate_bc.py).
"""
import numpy as np
import pytest

from compare import compare_topology

pytestmark = pytest.mark.gpu


def _exact_speeds(a, b):
    a, b = a.sorted(), b.sorted()
    assert np.array_equal(a.keys, b.keys)
    ex = a.exists.astype(bool)
    for f in ("u0x", "u0y", "u0z"):
        x, y = a.f64[f][ex], b.f64[f][ex]
        same = (x == y) | (np.isnan(x) & np.isnan(y))
        assert same.all(), (f, int((~same).sum()), int(same.size))


def _device(state):
    from mac_b200.gpu import Context
    with Context(state.params, max_bricks=state.nbricks + 64, max_particles=max(state.nparticles, 1) + 1024) as ctx:
        ctx.upload(state)
        ctx.extrapolate_boundary_condition(0)
        return ctx.download()


def _worlds():
    from test_extrapolate_bc import _chunk_world, _jet_like_world
    yield "chunk", _chunk_world(7, 0.1)
    for seed in range(3):
        yield f"blobs{seed}", _jet_like_world(seed)


@pytest.mark.parametrize("index", range(4))
def test_device_matches_oracle_on_blob_worlds(run_oracle, index):
    name, s = list(_worlds())[index]
    want, _ = run_oracle("extrapbc", s)
    got = _device(s)
    compare_topology(got, want)
    _exact_speeds(got, want)


@pytest.mark.parametrize("name", ["c1_ref_s30", "c1_ref_s60", "d_ref_s20"])
def test_device_matches_oracle_on_jet_states(golden, run_oracle, name):
    s = golden(name)
    want, _ = run_oracle("extrapbc", s)
    got = _device(s)
    compare_topology(got, want)
    _exact_speeds(got, want)
    # the stage changed the speed field
    assert not np.array_equal(np.nan_to_num(got.sorted().f64["u0z"]), np.nan_to_num(s.sorted().f64["u0z"]))

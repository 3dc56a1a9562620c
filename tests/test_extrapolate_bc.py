"""Algorithm_Extrapolate_Boundary_Condition's 2D form
(src/Algorithm_Extrapolate_Boundary_Condition.h:254-452) restated in
oracle/extrapolate_bc.py, checked against every known answer of the
reference's own test (test/test_Extrapolate_Boundary.h: 7 tests, 18 runs of
the algorithm, 565 asserts), extracted into tests/golden/extrap_bc_2d.json by
tests/golden/make_extrap_bc_golden.py. Values within the test's own 1e-10,
NaN where it asserts NaN.

The reference visits cells in its hash map's order; the known answers do not
depend on it: they hold for the key-sorted order, the reverse order and
random orders alike.
"""
import json
import math
import os
import random

import pytest

from conftest import GOLDEN

EPS = 1e-10


def _fixture():
    with open(os.path.join(GOLDEN, "extrap_bc_2d.json")) as f:
        return json.load(f)


def _failures(test, order_fn=None):
    import extrapolate_bc as eb
    bad = []
    for op, got in eb.replay(test, order_fn):
        if op["op"] == "expect":
            ok = not math.isnan(got) and abs(got - op["value"]) <= EPS
        else:
            ok = math.isnan(got) == op["isnan"]
        if not ok:
            bad.append((op, got))
    return bad


def test_fixture_holds_every_assert():
    fx = _fixture()
    assert len(fx["tests"]) == 7 and fx["runs"] == 18 and fx["asserts"] == 565


@pytest.mark.parametrize("name", ["test_one_particle", "test_two_particle_plane", "test_3_particle_corner",
                                  "test_square", "test_3_align", "test_3_align_1", "test_4_align_2"])
def test_known_answers_2d(name):
    test = next(t for t in _fixture()["tests"] if t["name"] == name)
    assert _failures(test) == []


def test_known_answers_do_not_depend_on_the_visiting_order():
    for test in _fixture()["tests"]:
        assert _failures(test, lambda w: sorted(w.cells, reverse=True)) == []
        for seed in range(5):
            rng = random.Random(seed)
            assert _failures(test, lambda w: rng.sample(sorted(w.cells), len(w.cells))) == []


# ---- the 3D form (src/Algorithm_Extrapolate_Boundary_Condition.h:454-975)
def _chunk_world(seed, const_frac):
    """One 8^3 chunk, every cell existing: random fluid cells in [2, 5]^3 (so
    every read of a boundary cell's case stays inside the chunk), air
    elsewhere, random face speeds, a fraction of random const faces."""
    import numpy as np
    from mac_b200.state import AIR, FLUID, Params, from_cells
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij"), -1).reshape(-1, 3)
    inner = np.all((g >= 2) & (g <= 5), axis=1)
    fluid = inner & (rng.random(len(g)) < 0.6)
    typ = np.where(fluid, FLUID, AIR).astype(np.uint8)
    flags = np.where(rng.random(len(g)) < const_frac, rng.integers(1, 8, len(g)), 0).astype(np.uint8)
    return from_cells(Params(h=(0.1, 0.1, 0.1)), g, typ, flags, rng.uniform(-1, 1, (len(g), 3)))


def _same_faces(a, b):
    import numpy as np
    a, b = a.sorted(), b.sorted()
    assert np.array_equal(a.keys, b.keys)
    ex = a.exists.astype(bool)
    for f in ("u0x", "u0y", "u0z"):
        x, y = a.f64[f][ex], b.f64[f][ex]
        same = (x == y) | (np.isnan(x) & np.isnan(y))
        assert same.all(), (f, int((~same).sum()))


def test_3d_form_matches_the_reference_in_one_chunk(oracle_lib, tmp_path):
    """The reference's own 3D form (oracle/_ref/mac_ref, command extrapbc, its
    3x3 corner systems solved by the same dense elimination) against the
    restatement visiting the cells in the same order (key order = offset order
    within the one chunk): every face bit for bit, NaN where NaN, on worlds
    with and without const faces."""
    from mac_b200.state import State
    if not oracle_lib.have_ref():
        pytest.skip("oracle/_ref/mac_ref is not built (needs the reference sources)")
    for seed in range(24):
        s = _chunk_world(seed, 0.1 if seed % 2 else 0.0)
        src = str(tmp_path / "in.state")
        s.write(src)
        oracle_lib.run_ref("extrapbc", src, str(tmp_path / "ref.state"))
        oracle_lib.run_oracle("extrapbckey", src, str(tmp_path / "ora.state"))
        _same_faces(State.read(str(tmp_path / "ref.state")), State.read(str(tmp_path / "ora.state")))


def _jet_like_world(seed):
    """A 24^3 box over several chunks: a pool and random blobs of fluid with
    two air layers around them, random face speeds: boundary cells close
    enough to interact."""
    import numpy as np
    from mac_b200.state import AIR, FLUID, Params, from_cells
    rng = np.random.default_rng(seed)
    n = 24
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    inner = np.all((g >= 2) & (g < n - 2), axis=1)
    fluid = inner & ((g[:, 2] < 8) | (rng.random(len(g)) < 0.35))
    typ = np.where(fluid, FLUID, AIR).astype(np.uint8)
    return from_cells(Params(h=(0.1, 0.1, 0.1)), g, typ, np.zeros(len(g), np.uint8),
                      rng.uniform(-1, 1, (len(g), 3)))


def test_3d_cells_of_one_colour_commute(oracle_lib, tmp_path):
    """The fixed order the device uses visits cells by colour (x, y, z mod 5),
    the cells of one colour in parallel. Every read and write of one boundary
    cell's case lies within distance 2, so cells of one colour never touch the
    same face: visiting each colour's cells in the opposite key order gives
    the same faces bit for bit."""
    from mac_b200.state import State
    for seed in range(4):
        src = str(tmp_path / "in.state")
        _jet_like_world(seed).write(src)
        oracle_lib.run_oracle("extrapbc", src, str(tmp_path / "a.state"))
        oracle_lib.run_oracle("extrapbcrev", src, str(tmp_path / "b.state"))
        _same_faces(State.read(str(tmp_path / "a.state")), State.read(str(tmp_path / "b.state")))

"""Known-answer cases of the reference's own tests, rebuilt on small 3D worlds
and checked on the oracle (and, where the reference runner was built here, on
the reference itself):

* particle -> key: test/TestAlgorithm_Layer_Initial_With_Particle.h:106-123
* air layers around one fluid cell: test/TestAlgorithms_Update_CellType_Layer.h:103-149
* upwind convection -1.0 / 0.11 / -1.25: test/old/TestPolicy_Upwind_1_Order.h:99-104,214-215
* staggered interpolation 1, 1.5, 1.4: test/old/TestPolicy_Speed_Interpolation_Linear.h:100-120
* divergence and gradient of simple fields: test/old/TestPolicy_Divergence.h,
  test/old/TestPolicy_Gradiant.h (values -1, -10, 1)
* RK4 particle moves 0.1 / 0.01: test/old/TestAlgorithms_Move_Particles.h:159-567
* the projection of a five-cell plus, 1.25 / 0.2499999999999998890 / 0.75:
  test/old/TestAlgorithms_Solve_Pressure.h:449-470 (2D cases embedded in one
  layer of cells between Neumann faces)
* the material predicates and setters: test/TestData_CellType_Fluid_Air_Solid_Inflow*.h,
  test/Test_Data_CellType_Domain_Fluid.h
* in-chunk neighbour offsets: test/Test_Offset.h
"""
import numpy as np
import pytest

from mac_b200.state import FLUID, Params, from_cells

EPS = 1e-12


def _block(x0, x1, y0, y1, z0, z1):
    z, y, x = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=-1)


def _field_world(h=1.0, ux=None):
    """Fluid cells x in [-2,3], y,z in [-1,1]; u_x set per x column."""
    keys = _block(-2, 3, -1, 1, -1, 1)
    u = np.zeros((len(keys), 3))
    for x, v in (ux or {}).items():
        u[keys[:, 0] == x, 0] = v
    pr = Params(h=(h, h, h), gravity=0.0)
    return from_cells(pr, keys, np.full(len(keys), FLUID, np.uint8), np.zeros(len(keys), np.uint8), u)


def _write(s, tmp_path, name="k.state"):
    p = str(tmp_path / name)
    s.write(p)
    return p


def test_particle_to_key(run_oracle):
    pr = Params(h=(1.0, 1.0, 1.0), layer_max=4)
    s = from_cells(pr, np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros((0, 3)),
                   pos=np.array([[2.2, 4.3, 5.4]]))
    got, _ = run_oracle("topology", s)
    keys = got.cell_keys()
    hit = (keys[..., 0] == 2) & (keys[..., 1] == 4) & (keys[..., 2] == 5)
    assert got.exists[hit].item() == 1
    assert got.layer[hit].item() == 0
    assert got.type[hit].item() == FLUID


def _layer_of(s, k):
    keys = s.cell_keys()
    hit = (keys[..., 0] == k[0]) & (keys[..., 1] == k[1]) & (keys[..., 2] == k[2])
    if not hit.any() or not s.exists[hit].item():
        return None
    return s.layer[hit].item()


def test_layers_around_one_fluid_cell(run_oracle):
    pr = Params(h=(1.0, 1.0, 1.0), layer_max=1)
    s = from_cells(pr, np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros((0, 3)), pos=np.array([[0.0, 0, 0]]))
    got, _ = run_oracle("topology", s)
    assert _layer_of(got, (0, 0, 0)) == 0
    for k in [(1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        assert _layer_of(got, k) == 1, k
    # the reference's 2D expectations (slice z = 0) of the LayerMax+1 ring
    for k in [(2, 0, 0), (1, 1, 0), (1, -1, 0), (0, 2, 0), (-1, 1, 0)]:
        assert _layer_of(got, k) == 2, k
    # ring = +e_i faces of the layer-1 cells only
    assert _layer_of(got, (-2, 0, 0)) is None
    assert _layer_of(got, (-1, -1, 0)) is None


def test_upwind_known_answers(oracle_lib, tmp_path):
    s = _field_world(ux={0: 0.0, 1: 1.0})
    p = _write(s, tmp_path)
    assert abs(oracle_lib.probe(p, "convection", key=(1, 0, 0), i=0) - (-1.0)) < EPS
    s = _field_world(ux={0: -0.1, 1: 1.0})
    p = _write(s, tmp_path, "k2.state")
    assert abs(oracle_lib.probe(p, "convection", key=(0, 0, 0), i=0) - 0.11) < EPS


@pytest.mark.parametrize("sym", [0, 1])
def test_interpolation_known_answers(oracle_lib, tmp_path, sym):
    p = _write(_field_world(ux={0: 1.0, 1: 1.0}), tmp_path)
    assert abs(oracle_lib.probe(p, "speed", pos=(0.0, 0, 0), sym=sym)[0] - 1.0) < EPS
    assert abs(oracle_lib.probe(p, "speed", pos=(0.1, 0, 0), sym=sym)[0] - 1.0) < EPS
    p = _write(_field_world(ux={0: 2.0, 1: 1.0}), tmp_path, "k2.state")
    assert abs(oracle_lib.probe(p, "speed", pos=(0.0, 0, 0), sym=sym)[0] - 1.5) < EPS
    assert abs(oracle_lib.probe(p, "speed", pos=(0.1, 0, 0), sym=sym)[0] - 1.4) < EPS


def test_divergence_and_gradient(oracle_lib, tmp_path):
    p = _write(_field_world(h=1.0, ux={0: 1.0}), tmp_path)
    assert abs(oracle_lib.probe(p, "divergence", key=(0, 0, 0)) - (-1.0)) < EPS
    p = _write(_field_world(h=0.1, ux={0: 1.0}), tmp_path, "k2.state")
    assert abs(oracle_lib.probe(p, "divergence", key=(0, 0, 0)) - (-10.0)) < 1e-9
    s = _field_world()
    keys = s.cell_keys()
    s.f64["p"][(keys[..., 0] == 0) & s.exists.astype(bool)] = 1.0
    p = _write(s, tmp_path, "k3.state")
    assert abs(oracle_lib.probe(p, "gradient", key=(0, 0, 0), i=0) - 1.0) < EPS
    assert abs(oracle_lib.probe(p, "gradient", key=(0, 0, 0), i=1)) < EPS


def test_brick_layout_and_floor_division():
    """Chunk key = floor(key / 8), slot x + 8y + 64z (src/ChunkHashTable.tpp:180-196,
    src/Offset.h:14-24)."""
    pr = Params()
    keys = np.array([[-1, 0, 0], [-8, 0, 0], [-9, 0, 0], [7, 7, 7], [8, 0, 0]])
    s = from_cells(pr, keys, np.zeros(5), np.zeros(5), np.zeros((5, 3)))
    bk = {tuple(k) for k in s.keys.tolist()}
    assert bk == {(-1, 0, 0), (-2, 0, 0), (0, 0, 0), (1, 0, 0)}
    ck = s.cell_keys()[s.exists.astype(bool)]
    assert sorted(map(tuple, ck.tolist())) == sorted(map(tuple, keys.tolist()))


def _cells(entries, params):
    """entries: {(x, y, z): (type, flags, (ux, uy, uz))}."""
    keys = np.array(list(entries.keys()), dtype=np.int64)
    vals = list(entries.values())
    return from_cells(params, keys, np.array([v[0] for v in vals], np.uint8), np.array([v[1] for v in vals], np.uint8),
                      np.array([v[2] for v in vals], np.float64))


def _at(s, k, field):
    keys = s.cell_keys()
    hit = (keys[..., 0] == k[0]) & (keys[..., 1] == k[1]) & (keys[..., 2] == k[2]) & s.exists.astype(bool)
    return s.f64[field][hit].item()


def test_upwind_known_answer_diagonal(oracle_lib, tmp_path):
    """test/old/TestPolicy_Upwind_1_Order.h:106-215 (2D): speeds zero on a 3x3
    block except (1, 1) = (1, 1); the convection of both components there is
    -1.25 (x: U = 1, backward difference 1; y: U at the bound = 1/4, backward
    difference 1). Here a 3x3x3 block of fluid cells, the middle layer as the
    2D case; the z term vanishes (U_z = 0)."""
    cells = {(x, y, z): (FLUID, 0, (0.0, 0.0, 0.0)) for x in range(3) for y in range(3) for z in (-1, 0, 1)}
    cells[(1, 1, 0)] = (FLUID, 0, (1.0, 1.0, 0.0))
    p = _write(_cells(cells, Params(h=(1.0, 1.0, 1.0), gravity=0.0)), tmp_path)
    assert abs(oracle_lib.probe(p, "convection", key=(1, 1, 0), i=0) - (-1.25)) < EPS
    assert abs(oracle_lib.probe(p, "convection", key=(1, 1, 0), i=1) - (-1.25)) < EPS


@pytest.mark.parametrize("stage", ["movelin", "move"])
@pytest.mark.parametrize("h,dt,want", [(1.0, 0.1, 0.1), (0.1, 0.01, 0.01)])
def test_particle_move_known_answers(run_oracle, stage, h, dt, want):
    """test/old/TestAlgorithms_Move_Particles.h:49-567: a uniform unit speed,
    a particle at the origin moved by RK4 over dt: 0.1 at h = 1, dt = 0.1 and
    0.01 at h = 0.1, dt = 0.01, in every component (the reference's linear
    interpolation; the symmetric one gives the same on a uniform field)."""
    cells = {(x, y, z): (FLUID, 0, (1.0, 1.0, 1.0))
             for x in range(-2, 3) for y in range(-2, 3) for z in range(-2, 3)}
    pr = Params(h=(h, h, h), gravity=0.0, dt=dt)
    s = _cells(cells, pr)
    s.pos = np.zeros((1, 3))
    got, st = run_oracle(stage, s)
    assert np.allclose(got.pos[0], [want, want, want], rtol=0, atol=1e-10), got.pos[0]
    assert st["invalid_reads"] == 0


def test_projection_known_answers(run_oracle):
    """test/old/TestAlgorithms_Solve_Pressure.h:202-470 (2D): a plus of five
    fluid cells, (0, 0) at speed (2, 2) and its four neighbours at (1, 1), air
    (p = 0) around. After the projection (0, 0) has (1.25, 1.25), (1, 0) has
    (1.25, 0.25), (0, 1) has (0.25, 1.25) and (-1, 0), (0, -1) have (0.75,
    0.75). Here the plus lies in the layer z = 0 between solid layers whose
    faces towards it are const (Neumann), so the z terms drop out of the
    operator and the 3D projection is the 2D one."""
    plus = {(0, 0): (2.0, 2.0), (1, 0): (1.0, 1.0), (-1, 0): (1.0, 1.0), (0, 1): (1.0, 1.0), (0, -1): (1.0, 1.0)}
    cells = {}
    for x in range(-2, 3):
        for y in range(-2, 3):
            u = plus.get((x, y))
            cells[(x, y, 0)] = (FLUID if u else 0, 4, (u[0], u[1], 0.0) if u else (0.0, 0.0, 0.0))
            cells[(x, y, -1)] = (2, 0, (0.0, 0.0, 0.0))  # solid below
            cells[(x, y, 1)] = (2, 4, (0.0, 0.0, 0.0))   # solid above, its -z face const
    got, st = run_oracle("project", _cells(cells, Params(h=(1.0, 1.0, 1.0), gravity=0.0)))
    want = {(0, 0): (1.25, 1.25), (1, 0): (1.25, 0.24999999999999988898), (0, 1): (0.24999999999999988898, 1.25),
            (-1, 0): (0.75, 0.75), (0, -1): (0.75, 0.75)}
    for (x, y), (wx, wy) in want.items():
        assert abs(_at(got, (x, y, 0), "u0x") - wx) < 1e-10, (x, y)
        assert abs(_at(got, (x, y, 0), "u0y") - wy) < 1e-10, (x, y)
        assert _at(got, (x, y, 0), "u0z") == 0.0
    assert abs(_at(got, (0, 0, 0), "p") - 1.0) < 1e-10
    assert st["relres"] <= 1e-14


# material: (GetIsFluid, GetIsAir) from test/TestData_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.h:29-58
# (the 0_Pres material of that variant is not on this path)
MATERIAL_TABLE = {"Air": (False, True), "Fluid": (True, False), "Solid": (False, True),
                  "Inflow": (True, False), "Interior": (True, False)}


def test_material_rules_match_the_reference_tables(oracle_lib):
    from mac_b200.state import AIR, INFLOW, INTERIOR, SOLID
    code = {"Air": AIR, "Fluid": FLUID, "Solid": SOLID, "Inflow": INFLOW, "Interior": INTERIOR}
    # MaterialToInt: Fluid 1, Air 0 (test/TestData_CellType_Fluid_Air_Solid_Inflow.h:19-20)
    assert code["Fluid"] == 1 and code["Air"] == 0
    for name, (fluid, air) in MATERIAL_TABLE.items():
        m = oracle_lib.material(code[name])
        assert m["is_fluid"] == fluid and m["is_air"] == air, name
        # the solve's domain is the fluid cells (test/Test_Data_CellType_Domain_Fluid.h:22-23)
        assert m["in_domain"] == fluid, name
    # SetFluid puts an air cell in the domain, SetAir takes it out
    # (test/Test_Data_CellType_Domain_Fluid.h:29-32)
    assert oracle_lib.material(oracle_lib.material(AIR)["after_set_fluid"])["in_domain"]
    assert not oracle_lib.material(oracle_lib.material(FLUID)["after_set_air"])["in_domain"]
    # the setters are sticky: SetAir changes only fluid and interior cells, SetFluid
    # only air and interior cells (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior.tpp:178-193)
    for name in MATERIAL_TABLE:
        m = oracle_lib.material(code[name])
        assert m["after_set_air"] == (AIR if name in ("Fluid", "Interior") else code[name]), name
        assert m["after_set_fluid"] == (FLUID if name in ("Air", "Interior") else code[name]), name


def test_brick_neighbour_offsets_match_the_offset_tests():
    """test/Test_Offset.h:30-43 (N = 4, 3D): from offset 0 the +x, +y, +z
    neighbours stay in the chunk at offsets 1, N, N^2 and the -x, -y, -z ones
    leave it, wrapping to N-1, N(N-1), N^2(N-1). The device's 8^3 bricks follow
    the same rule with N = 8: 1, 8, 64 inside, 7, 56, 448 in the neighbour brick."""
    pr = Params()
    cases = {(1, 0, 0): ((0, 0, 0), 1), (0, 1, 0): ((0, 0, 0), 8), (0, 0, 1): ((0, 0, 0), 64),
             (-1, 0, 0): ((-1, 0, 0), 7), (0, -1, 0): ((0, -1, 0), 56), (0, 0, -1): ((0, 0, -1), 448)}
    keys = np.array([[0, 0, 0]] + [list(k) for k in cases], dtype=np.int64)
    s = from_cells(pr, keys, np.zeros(len(keys)), np.zeros(len(keys)), np.zeros((len(keys), 3)))
    where = {}
    for b, bk in enumerate(s.keys.tolist()):
        for off in np.flatnonzero(s.exists[b]):
            x, y, z = off % 8, (off // 8) % 8, off // 64
            where[(bk[0] * 8 + x, bk[1] * 8 + y, bk[2] * 8 + z)] = (tuple(bk), int(off))
    assert where[(0, 0, 0)] == ((0, 0, 0), 0)
    for k, want in cases.items():
        assert where[k] == want, k

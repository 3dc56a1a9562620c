"""Headless VTK-XML output: the pressure, speed and particle datasets of the
reference's output policies written from a reference-produced state (the
32x32x64 jet after 30 steps) and read back: geometry rules, connectivity,
values bit for bit, and the .pvd collection."""
import numpy as np

from mac_b200 import vtk
from mac_b200.state import FLUID, INFLOW


def test_pressure_dataset(golden, tmp_path):
    s = golden("c1_ref_t30")
    f = vtk.write_pressure(s, str(tmp_path / "p30.vtu"))
    d = vtk.read_vtu(f)
    h = np.asarray(s.params.h)
    ex = s.exists.astype(bool)
    keys = s.cell_keys()[ex]
    # points: every existing cell's corner plus the +e_i corners of missing neighbours
    kset = {tuple(k) for k in keys}
    extra = set()
    for k in keys:
        for a in range(3):
            k2 = list(k)
            k2[a] += 1
            if tuple(k2) not in kset:
                extra.add(tuple(k2))
    assert d["points"].shape[0] == len(kset | extra)
    np.testing.assert_array_equal(d["types"], vtk.VTK_VOXEL)
    p = d["points"]
    c = d["cells"]
    for j, step in enumerate(vtk._VOXEL):
        d_ = p[c[:, j]] - p[c[:, 0]]
        np.testing.assert_allclose(d_, np.broadcast_to(step * h, d_.shape), atol=1e-12)
    # every voxel sits on an existing cell and carries its pressure and material
    anchor = np.rint(p[c[:, 0]] / h + 0.5).astype(np.int64)
    bi = {tuple(k): i for i, k in enumerate(keys)}
    idx = np.array([bi[tuple(k)] for k in anchor])
    np.testing.assert_array_equal(d["cell_data"]["Pressure"], s.f64["p"][ex][idx])
    typ = s.type[ex][idx]
    np.testing.assert_array_equal(d["cell_data"]["Fluid"], ((typ == FLUID) | (typ == INFLOW)).astype(np.int32))
    assert d["cell_data"]["Fluid"].sum() == s.fluid_cells()  # every fluid cell has all corners


def test_speed_and_particle_datasets(golden, tmp_path):
    s = golden("c1_ref_t30")
    files = vtk.write_speed(s, str(tmp_path / "speed"), 30)
    assert [f.split("/")[-1] for f in files] == ["speed_1_30.vtu", "speed_2_30.vtu", "speed_3_30.vtu"]
    h = np.asarray(s.params.h)
    m = s.exists.astype(bool) & (s.layer >= 0)
    for i, f in enumerate(files):
        d = vtk.read_vtu(f)
        name = ("speedx", "speedy", "speedz")[i]
        k = np.rint(d["points"] / h + 0.5 * (np.arange(3) == i)).astype(np.int64)
        assert d["points"].shape[0] == int(m.sum())
        lut = {tuple(kk): v for kk, v in zip(s.cell_keys()[m], s.f64["u0" + "xyz"[i]][m])}
        np.testing.assert_array_equal(d["point_data"][name], np.array([lut[tuple(kk)] for kk in k]))
    f = vtk.write_particles(s, str(tmp_path / "part"), 30)
    d = vtk.read_vtu(f)
    np.testing.assert_array_equal(d["points"], s.pos)
    assert d["cells"].shape == (s.nparticles, 1)


def test_pvd_collection(tmp_path):
    entries = [(0.0, 0, "a0.vtu"), (0.0125, 1, "a1.vtu")]
    f = vtk.write_pvd(str(tmp_path / "anim.pvd"), entries)
    assert vtk.read_pvd(f) == entries

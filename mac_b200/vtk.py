"""Headless VTK-XML output (and input) of a world, without the VTK library.

The reference writes its state with VTK's XML writers (`src/Policy_Output_*.h`);
this module writes the same datasets as `.vtu` files directly (appended-free
"binary" data arrays: base64 of a UInt64 byte count followed by the raw
little-endian values, readable by ParaView and VTK) and reads them back:

* pressure (`src/Policy_Output_Grid_Pressure.h:74-222`): points at the cell
  corners (key - 1/2) h of every existing cell, plus the +e_i corners of cells
  whose +e_i neighbour does not exist; one voxel per existing cell whose eight
  corners are all points; cell data `Pressure` (Float64), `Fluid` and `Solid`
  (Int32);
* speed component i (`src/Policy_Output_Grid_Speed.h:38-178`): points at the
  face centres of cells with a non-empty layer (coordinate i shifted by -1/2);
  a voxel per such cell whose +x, +y, +z neighbour chain (7 cells) all have a
  non-empty layer; point data `speedx` / `speedy` / `speedz`; files
  `<pref>_<i>_<step>.vtu`;
* particles (`src/Policy_Output_Particle.h:36-73`): one vertex per particle;
* the collection (`src/Policy_Output_Animation.h:30-50`): a `.pvd` listing each
  file with its time.

The reference numbers points in its hash tables' iteration order; these files
number them in ascending key order (z, y, x), so the datasets are equal as sets
of points, cells and values.
"""
import base64
import os
import re
import xml.etree.ElementTree as ET

import numpy as np

from .state import FLUID, INFLOW, SOLID, State

VTK_VERTEX, VTK_VOXEL = 1, 11
_VTK_TYPES = {np.dtype(np.float64): "Float64", np.dtype(np.float32): "Float32", np.dtype(np.int32): "Int32",
              np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}
_NP_TYPES = {v: k for k, v in _VTK_TYPES.items()}


def _enc(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


def _dec(text: str, dtype) -> np.ndarray:
    raw = base64.b64decode("".join(text.split()))
    n = int(np.frombuffer(raw[:8], dtype="<u8")[0])
    return np.frombuffer(raw[8:8 + n], dtype=np.dtype(dtype).newbyteorder("<")).copy()


def _array(name, a, ncomp=1):
    a = np.asarray(a)
    return (f'<DataArray type="{_VTK_TYPES[a.dtype]}" Name="{name}" NumberOfComponents="{ncomp}" '
            f'format="binary">{_enc(a)}</DataArray>')


def write_vtu(path, points, cells, cell_type, point_data=None, cell_data=None):
    """Writes an UnstructuredGrid: points (n, 3) float64, cells (m, k) int64
    connectivity of one VTK cell type, and name -> array dicts."""
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    m, k = (cells.shape[0], cells.shape[1]) if cells.size else (0, 1)
    parts = ['<?xml version="1.0"?>',
             '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
             '<UnstructuredGrid>', f'<Piece NumberOfPoints="{points.shape[0]}" NumberOfCells="{m}">',
             '<Points>', _array("Points", points.ravel(), 3), '</Points>', '<Cells>',
             _array("connectivity", cells.ravel()),
             _array("offsets", (np.arange(1, m + 1, dtype=np.int64) * k)),
             _array("types", np.full(m, cell_type, np.uint8)), '</Cells>']
    for tag, data in (("PointData", point_data), ("CellData", cell_data)):
        if data:
            parts.append(f"<{tag}>")
            parts += [_array(n, v) for n, v in data.items()]
            parts.append(f"</{tag}>")
    parts += ['</Piece>', '</UnstructuredGrid>', '</VTKFile>']
    with open(path, "w") as f:
        f.write("\n".join(parts))
    return path


def read_vtu(path):
    """Reads a file written by write_vtu: dict with points, cells, types,
    point_data and cell_data."""
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {"point_data": {}, "cell_data": {}}

    def arr(el):
        return _dec(el.text or "", _NP_TYPES[el.get("type")])
    out["points"] = arr(piece.find("Points/DataArray")).reshape(-1, 3)
    cells = {el.get("Name"): arr(el) for el in piece.findall("Cells/DataArray")}
    m = int(piece.get("NumberOfCells"))
    out["types"] = cells["types"]
    out["cells"] = cells["connectivity"].reshape(m, -1) if m else np.zeros((0, 1), np.int64)
    for tag, key in (("PointData", "point_data"), ("CellData", "cell_data")):
        for el in piece.findall(f"{tag}/DataArray"):
            out[key][el.get("Name")] = arr(el)
    return out


# ------------------------------------------------------------------ worlds
def _cells(s: State, mask=None):
    """Keys (n, 3) and flat (brick, slot) indices of the existing cells (optionally masked)."""
    ex = s.exists.astype(bool) if mask is None else mask
    b, o = np.nonzero(ex)
    return s.cell_keys()[b, o].astype(np.int64), b, o


def _pack(k):
    k = np.asarray(k, dtype=np.int64) + (1 << 20)
    return k[..., 0] | (k[..., 1] << 21) | (k[..., 2] << 42)


def _lookup(sorted_codes, codes):
    """Position of each code in sorted_codes, -1 when absent."""
    i = np.searchsorted(sorted_codes, codes)
    i = np.clip(i, 0, max(len(sorted_codes) - 1, 0))
    ok = (len(sorted_codes) > 0) & (sorted_codes[i] == codes) if len(sorted_codes) else np.zeros(codes.shape, bool)
    return np.where(ok, i, -1)


_VOXEL = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]])


def write_pressure(s: State, path: str) -> str:
    """The pressure dataset of Policy_Output_Grid_Pressure::OutputGridPressure."""
    h = np.asarray(s.params.h, dtype=np.float64)
    keys, b, o = _cells(s)
    codes = _pack(keys)
    order = np.argsort(codes)
    keys, b, o, codes = keys[order], b[order], o[order], codes[order]
    # corner points: every existing cell, plus +e_i corners where that cell is missing
    extra = []
    for a in range(3):
        k2 = keys.copy()
        k2[:, a] += 1
        missing = _lookup(codes, _pack(k2)) < 0
        extra.append(k2[missing])
    pkeys = np.unique(np.concatenate([keys] + extra), axis=0)
    pkeys = pkeys[np.argsort(_pack(pkeys))]
    pcodes = _pack(pkeys)
    corner = np.stack([_lookup(pcodes, _pack(keys + d)) for d in _VOXEL], axis=1)
    full = np.all(corner >= 0, axis=1)
    bb, oo = b[full], o[full]
    typ = s.type[bb, oo]
    cell_data = {"Pressure": s.f64["p"][bb, oo].astype(np.float64),
                 "Fluid": ((typ == FLUID) | (typ == INFLOW)).astype(np.int32),
                 "Solid": (typ == SOLID).astype(np.int32)}
    return write_vtu(path, (pkeys - 0.5) * h, corner[full], VTK_VOXEL, cell_data=cell_data)


def write_speed(s: State, pref: str, step: int, buffer: int = 0) -> list:
    """The three speed datasets of Policy_Output_Grid_Speed::OutputGridSpeed
    (speed buffer 0 by default); returns the file names."""
    h = np.asarray(s.params.h, dtype=np.float64)
    mask = s.exists.astype(bool) & (s.layer >= 0)
    keys, b, o = _cells(s, mask)
    codes = _pack(keys)
    order = np.argsort(codes)
    keys, b, o, codes = keys[order], b[order], o[order], codes[order]
    corner = np.stack([_lookup(codes, _pack(keys + d)) for d in _VOXEL], axis=1)
    full = np.all(corner >= 0, axis=1)
    files = []
    for i, name in enumerate(("speedx", "speedy", "speedz")):
        pts = keys.astype(np.float64)
        pts[:, i] -= 0.5
        val = s.f64[f"u{buffer}{'xyz'[i]}"][b, o]
        path = f"{pref}_{i + 1}_{step}.vtu"
        files.append(write_vtu(path, pts * h, corner[full], VTK_VOXEL, point_data={name: val}))
    return files


def write_particles(s: State, pref: str, step: int) -> str:
    """Policy_Output_Particle::OutputParticle: one vertex per particle."""
    n = s.nparticles
    return write_vtu(f"{pref}{step}.vtu", s.pos, np.arange(n, dtype=np.int64).reshape(-1, 1), VTK_VERTEX)


def write_pvd(path: str, entries) -> str:
    """Collection file: entries are (time, part, file name) in output order."""
    lines = ['<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">', "<Collection>"]
    for t, part, f in entries:
        lines.append(f' <DataSet timestep="{float(t)!r}" group="" part="{int(part)}" file="{os.path.basename(f)}" />')
    lines += ["</Collection>", "</VTKFile>"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def read_pvd(path: str):
    text = open(path).read()
    return [(float(t), int(p), f) for t, p, f in
            re.findall(r'timestep="([^"]+)" group="" part="([^"]+)" file="([^"]+)"', text)]

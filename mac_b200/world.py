"""World set-up on the host: the one-time passes that precede the first step.

``setup_passes`` restates Algorithms_Solid_To_Const (src/Algorithms_Solid_To_Const.h:24-63)
and Algorithms_Speed_Constant_Mirror (src/Algorithms_Speed_Constant_Mirror.h:22-70)
vectorised over the cell set; ``first_init`` then runs the device passes of the
reference's first init (test/TestJetDEau_Basic.cpp:329-330, 433): Initialize_MacCell,
Create_Fluid_Particle, Layer_Initial_With_Particle, Update_CellType_Layer,
Delete_MacCell and Algorithms_Extrapolate.
"""
from __future__ import annotations

import numpy as np

from .state import BRICK, BRICK_CELLS, FLAG_NODELETE, SOLID, State, empty_state

_OFF = 1 << 20


def _code(k):
    k = np.asarray(k, dtype=np.int64)
    return ((k[..., 0] + _OFF) | ((k[..., 1] + _OFF) << 21) | ((k[..., 2] + _OFF) << 42))


class _Grid:
    """Cell addressing over a State with brick creation (grid[key] semantics,
    src/ChunkHashTable.tpp:62-87)."""

    def __init__(self, s: State):
        self.s = s
        self._index()

    def _index(self):
        codes = _code(self.s.keys)
        self.order = np.argsort(codes)
        self.sorted_codes = codes[self.order]

    def locate(self, keys, create: bool):
        keys = np.asarray(keys, dtype=np.int64).reshape(-1, 3)
        bk = np.floor_divide(keys, BRICK)
        codes = _code(bk)
        pos = np.searchsorted(self.sorted_codes, codes)
        pos_c = np.minimum(pos, len(self.sorted_codes) - 1) if len(self.sorted_codes) else pos
        found = (len(self.sorted_codes) > 0) & (self.sorted_codes[pos_c] == codes) if len(self.sorted_codes) else \
            np.zeros(len(codes), bool)
        if create and not found.all():
            missing = np.unique(bk[~found], axis=0)
            self._append(missing)
            return self.locate(keys, create)
        bi = np.where(found, self.order[pos_c] if len(self.sorted_codes) else 0, -1)
        loc = keys - bk * BRICK
        off = loc[:, 0] + 8 * loc[:, 1] + 64 * loc[:, 2]
        if create:
            self.s.exists[bi, off] = 1
        return bi, off

    def _append(self, bkeys):
        s = self.s
        add = empty_state(s.params, bkeys.astype(np.int32))
        s.keys = np.concatenate([s.keys, add.keys])
        s.exists = np.concatenate([s.exists, add.exists])
        for n in s.f64:
            s.f64[n] = np.concatenate([s.f64[n], add.f64[n]])
        s.flags = np.concatenate([s.flags, add.flags])
        s.type = np.concatenate([s.type, add.type])
        s.layer = np.concatenate([s.layer, add.layer])
        s.id = np.concatenate([s.id, add.id])
        s.depth = np.concatenate([s.depth, add.depth])
        self._index()


def _cells_where(s: State, mask) -> np.ndarray:
    b, o = np.nonzero(mask)
    ck = s.cell_keys()
    return ck[b, o]


def solid_to_const(s: State) -> State:
    """Algorithms_Solid_To_Const: every solid cell and each +e_i neighbour become
    no-delete with pressure 0, speed 0 through the non-forced Set and const face
    i set. Every face it makes const is zeroed just before, so the result does
    not depend on the order the reference's stack visits the solids in."""
    g = _Grid(s)
    solid = _cells_where(s, s.exists.astype(bool) & (s.type == SOLID))
    if len(solid) == 0:
        return s
    touched = [solid] + [solid + np.eye(3, dtype=np.int64)[i] for i in range(3)]
    const_of = [None, 1, 2, 4]
    # const bits before the pass decide which values survive the zeroing
    allk = np.concatenate(touched)
    bi, off = g.locate(allk, create=True)
    before = s.flags[bi, off].copy()
    for j, name in enumerate(("u0x", "u0y", "u0z")):
        keep = (before >> j) & 1
        s.f64[name][bi, off] = np.where(keep == 1, s.f64[name][bi, off], 0.0)
    s.f64["p"][bi, off] = 0.0
    s.flags[bi, off] |= FLAG_NODELETE
    n = len(solid)
    sb, so = bi[:n], off[:n]
    s.flags[sb, so] |= 7
    for i in range(3):
        nb, no = bi[(i + 1) * n:(i + 2) * n], off[(i + 1) * n:(i + 2) * n]
        s.flags[nb, no] |= const_of[i + 1]
    return s


def constant_mirror(s: State) -> State:
    """Algorithms_Speed_Constant_Mirror: for every cell with a const face, the
    three +e_i neighbours get speed 0 (non-forced), then each const face value
    is copied onto the opposite face of the cell (non-forced)."""
    g = _Grid(s)
    m = s.exists.astype(bool) & ((s.flags & 7) != 0)
    ks = _cells_where(s, m)
    if len(ks) == 0:
        return s
    names = ("u0x", "u0y", "u0z")
    for i in range(3):
        nb, no = g.locate(ks + np.eye(3, dtype=np.int64)[i], create=True)
        for j in range(3):
            free = ((s.flags[nb, no] >> j) & 1) == 0
            s.f64[names[j]][nb[free], no[free]] = 0.0
    b0, o0 = g.locate(ks, create=False)
    for i in range(3):
        nb, no = g.locate(ks + np.eye(3, dtype=np.int64)[i], create=True)
        src_const = ((s.flags[b0, o0] >> i) & 1) == 1
        dst_free = ((s.flags[nb, no] >> i) & 1) == 0
        w = src_const & dst_free
        s.f64[names[i]][nb[w], no[w]] = s.f64[names[i]][b0[w], o0[w]]
    return s


def setup_passes(s: State) -> State:
    s = solid_to_const(s)
    s = constant_mirror(s)
    return s.sorted()


def first_init(ctx, s: State) -> State:
    """The reference's first init on the device (after the host set-up passes)."""
    s = setup_passes(s)
    ctx.upload(s)
    ctx.first_init_topology()
    ctx.extrapolate()
    return s

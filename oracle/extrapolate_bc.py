"""Oracle (test infrastructure only): a restatement of the reference's
boundary extrapolation, Algorithm_Extrapolate_Boundary_Condition
(src/Algorithm_Extrapolate_Boundary_Condition.h:52-986), in pure Python on a
sparse dict grid, for the small worlds of the reference's own test
(test/test_Extrapolate_Boundary.h). Nothing in the product imports it.

A world is {key tuple: Cell}; Cell.u[i] is the speed on the face between the
cell and its -e_i neighbour (staggered-left, src/Data_Staggered_Left.h:93-126),
Cell.fluid the fluid/air predicate of the cell type (GetIsFluid; every other
material counts as air, src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:25-44).
A neighbour outside the world is "not valid" (Offset_Base_Neighbour::GetNeighbour,
src/Offset_Base_Neighbour.h:14-33).

Reference details kept on purpose:
* GetNeighbour(i, 0) is the -e_i neighbour (the neighbour tables index
  (sign + 1) >> 1, src/Offset_GetNeighbour.h:52-57,
  src/Neighbour_List_Empty.tpp:18-24), so apply_nan_extrap's average over
  s = -1, 0, 1 counts the -e_i neighbour twice
  (src/Algorithm_Extrapolate_Boundary_Condition.h:221-235);
* Apply_Div_3d keeps only the last tangential term of its loop
  (src/Algorithm_Extrapolate_Boundary_Condition.h:918-931);
* in the 3D n == 1 case the "b" flag is never cleared
  (src/Algorithm_Extrapolate_Boundary_Condition.h:789-826).

The cells are visited in the order given (the reference visits its hash
map's order); `order` defaults to the key-sorted order. A neighbour the
reference would read through a null chunk reads as NaN here.
"""
from __future__ import annotations

import math

NAN = float("nan")


class Cell:
    __slots__ = ("fluid", "u")

    def __init__(self, fluid: bool, u):
        self.fluid = fluid
        self.u = list(u)


class World:
    def __init__(self, dim: int, h):
        self.dim = dim
        self.h = list(h)
        self.ih = [1.0 / x for x in h]
        self.cells: dict = {}

    # ---- grid access
    def nb(self, key, i, s):
        """Neighbour key along axis i (1-based); s = 0 means -1 (see above)."""
        k = list(key)
        k[i - 1] += -1 if s <= 0 else 1
        return tuple(k)

    def valid(self, key):
        return key in self.cells

    def u(self, key, i):
        c = self.cells.get(key)
        return NAN if c is None else c.u[i - 1]

    def set_u(self, key, i, v):
        c = self.cells.get(key)
        if c is not None:
            c.u[i - 1] = v

    def fluid(self, key):
        return self.cells[key].fluid

    def air(self, key):
        return not self.cells[key].fluid

    # ---- Algorithm_Extrapolate_Boundary_Condition_Common
    def is_boundary(self, key):
        """IsBoundary(neigh, dir, sign, n) (:89-119): (boundary?, dirs, signs, n)."""
        if self.air(key):
            return False, [], [], None
        dirs, signs = [], []
        for i in range(1, self.dim + 1):
            for s in (-1, 1):
                k2 = self.nb(key, i, s)
                if self.valid(k2) and self.air(k2):
                    dirs.append(i)
                    signs.append(s)
        return len(dirs) > 0, dirs, signs, len(dirs)

    def apply_set_nan(self, key):
        """apply_set_nan (:149-177)."""
        if not self.air(key):
            return
        for i in range(1, self.dim + 1):
            for s in (-1, 1):
                k2 = self.nb(key, i, s)
                if self.valid(k2):
                    if self.air(k2):
                        self.set_u(key if s == -1 else k2, i, NAN)
                elif s == -1:
                    self.set_u(key, i, NAN)

    def apply_nan_extrap(self, key):
        """apply_nan_extrap (:183-251)."""
        tab = []
        for i in range(1, self.dim + 1):
            v1 = self.u(key, i)
            v2 = self.u(self.nb(key, i, 1), i)
            if math.isnan(v1):
                tab.append((i, 0))
            if math.isnan(v2):
                tab.append((i, 1))
        if not tab:
            return
        for d, sg in tab:
            k2 = key if sg == 0 else self.nb(key, d, 1)
            vtemp = 0.0
            nb = 0
            for d2 in range(1, self.dim + 1):
                for s in (-1, 0, 1):
                    add = self.u(self.nb(k2, d2, s), d)
                    if not math.isnan(add):
                        vtemp += add
                        nb += 1
            if nb != 0:
                vtemp /= nb
            self.set_u(k2, d, vtemp)
        div = 0.0
        for i in range(1, self.dim + 1):
            v1 = self.u(key, i)
            v2 = self.u(self.nb(key, i, 1), i)
            div += self.ih[i - 1] * (v2 - v1)
        cor = div / len(tab)
        for d, sg in tab:
            k2 = key if sg == 0 else self.nb(key, d, 1)
            self.set_u(k2, d, self.u(k2, d) - (2 * sg - 1) * self.h[d - 1] * cor)

    def speed_in_domain(self, key, d):
        """Policy_Is_In_Domain_Speed::Get_Is_Speed_In_Domain (src/Policy_Is_In_Domain_Speed.h:15-48)."""
        k2 = self.nb(key, d, -1)
        if not self.valid(k2):
            return self.fluid(key)
        f1, f2 = self.fluid(key), self.fluid(k2)
        if f1 and f2:
            return True
        if not f1 and not f2:
            return False
        k3 = self.nb(key, d, 1) if f1 else self.nb(k2, d, -1)
        if not self.valid(k3):
            return True
        return not self.fluid(k3)

    def nan_if_not_in_domain(self, key, d, s):
        k3 = key if s == -1 else self.nb(key, d, 1)
        if not self.speed_in_domain(key, d):
            self.set_u(k3, d, NAN)

    # ---- the 2D form (:254-452)
    def do_2d(self, order=None):
        order = sorted(self.cells) if order is None else order
        for k in order:
            self.apply_set_nan(k)
        for k in order:
            b, dirs, signs, n = self.is_boundary(k)
            if b:
                self.choose_2d(k, dirs, signs, n)
        for k in order:
            if self.is_boundary(k)[0]:
                self.apply_nan_extrap(k)

    def _ntemp(self, key):
        """IsBoundary's count for a neighbour; 0 for an air or missing one (the
        reference leaves its counter unset there)."""
        if not self.valid(key) or self.air(key):
            return 0, []
        _, dirs, _, n = self.is_boundary(key)
        return n, dirs

    def choose_2d(self, key, dirs, signs, n):
        """Choose_Boundary_Case_2d (:298-363)."""
        if n == 1:
            dir2 = 2 if dirs[0] == 1 else 1
            b = True
            for i in (-1, 1):
                k2 = self.nb(key, dir2, i)
                nt, dt = self._ntemp(k2)
                if nt == 1 and dt[0] == dirs[0]:
                    b = False
                    if i < 0:
                        self.plane_2d(k2, key, dirs[0], signs[0])
                    else:
                        self.plane_2d(key, k2, dirs[0], signs[0])
            if b:
                k3 = key if signs[0] != 1 else self.nb(key, dirs[0], 1)
                if not self.speed_in_domain(key, dirs[0]):
                    self.set_u(k3, dirs[0], NAN)
        elif n == 2:
            if dirs[0] != dirs[1]:
                sa, sb = signs[0], signs[1]
                if dirs[0] > dirs[1]:
                    sa, sb = signs[1], signs[0]
                self.plane_45_2d(key, sa, sb)
        else:
            for i in range(n):
                k2 = key if signs[i] != 1 else self.nb(key, dirs[i], 1)
                if not self.speed_in_domain(k2, dirs[i]):
                    self.set_u(k2, dirs[i], NAN)

    def div_2d(self, key, d, sign):
        """Apply_Div_2d (:370-386)."""
        n = self.nb(key, d, 1)
        v = self.u(key, d)
        if sign == -1:
            v = self.u(n, d)
            n = key
        d2 = 2 if d == 1 else 1
        v2 = self.u(key, d2)
        v3 = self.u(self.nb(key, d2, 1), d2)
        self.set_u(n, d, v - sign * self.ih[d2 - 1] * self.h[d - 1] * (v3 - v2))

    def plane_2d(self, k1, k2, d, sign):
        """Apply_2d_Plane (:394-415)."""
        self.div_2d(k1, d, sign)
        self.div_2d(k2, d, sign)
        d2 = 2 if d == 1 else 1
        n, n2 = k1, k2
        if sign == 1:
            n, n2 = self.nb(k1, d, 1), self.nb(k2, d, 1)
        v1 = self.u(n, d)
        v2 = self.u(n2, d)
        v3 = self.u(k2, d2)
        v = -sign * self.ih[d2 - 1] * self.h[d - 1] * (v2 - v1) + v3
        self.set_u(self.nb(k2, d, sign), d2, v)

    def plane_45_2d(self, key, sa, sb):
        """Apply_2d_Plane_45 (:422-440)."""
        v1, v2 = self.u(key, 1), self.u(key, 2)
        n1, n2 = self.nb(key, 1, 1), self.nb(key, 2, 1)
        if sa == -1:
            v1 = self.u(self.nb(key, 1, 1), 1)
            n1 = key
        if sb == -1:
            v2 = self.u(self.nb(key, 2, 1), 2)
            n2 = key
        self.set_u(n1, 1, v1)
        self.set_u(n2, 2, v2)


def replay(test: dict, order_fn=None):
    """Runs one test of the fixture (make_extrap_bc_golden.py) and returns the
    list of (op, got) for its asserts. A cell first touched by an assert is
    created as air with zero speed, as grid[v] creates it."""
    w = World(2, test["h"])
    out = []
    for op in test["ops"]:
        k = tuple(op["key"]) if "key" in op else None
        if k is not None and k not in w.cells:
            w.cells[k] = Cell(False, [0.0, 0.0])
        if op["op"] == "speed":
            w.cells[k].u = list(op["u"])
        elif op["op"] == "type":
            # SetFluid / SetAir between air and fluid (sticky rules are moot for them)
            w.cells[k].fluid = op["fluid"]
        elif op["op"] == "do":
            w.do_2d(order_fn(w) if order_fn else None)
        else:
            out.append((op, w.u(k, op["dim"])))
    return out

"""State comparison used by the parity tests."""
from __future__ import annotations

import numpy as np

from mac_b200.state import CELL_F64, FLUID_TYPES, State

SPEEDS = ("u0x", "u0y", "u0z")


def _align(a: State, b: State):
    a, b = a.sorted(), b.sorted()
    if a.keys.shape != b.keys.shape or not np.array_equal(a.keys, b.keys):
        sa = {tuple(k) for k in a.keys.tolist()}
        sb = {tuple(k) for k in b.keys.tolist()}
        raise AssertionError(f"brick sets differ: only-a {sorted(sa - sb)[:8]} only-b {sorted(sb - sa)[:8]}")
    return a, b


def compare_topology(a: State, b: State, check_stale=True) -> None:
    """Bit-exact: live bricks, existence, material, layer, depth, const/no-delete bits."""
    a, b = _align(a, b)
    ex = a.exists.astype(bool)
    if not np.array_equal(a.exists, b.exists):
        idx = np.argwhere(a.exists != b.exists)[:5]
        raise AssertionError(f"existence differs at {idx.tolist()} keys {a.cell_keys()[tuple(idx.T)].tolist()}")
    mask = np.ones_like(ex) if check_stale else ex
    for name in ("type", "layer", "depth", "flags"):
        x, y = getattr(a, name), getattr(b, name)
        # the layer and depth of an erased cell are never read before they are
        # rewritten; only existing cells' layers and depths are compared
        bad = (x != y) & (ex if name in ("layer", "depth") else mask)
        if bad.any():
            idx = np.argwhere(bad)[:5]
            raise AssertionError(f"{name} differs ({int(bad.sum())} cells) e.g. at keys "
                                 f"{a.cell_keys()[tuple(idx.T)].tolist()}: {x[tuple(idx.T)]} vs {y[tuple(idx.T)]}")


def rel_err(x, y, mask=None):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if mask is not None:
        x, y = x[mask], y[mask]
    d = np.linalg.norm((x - y).ravel())
    n = np.linalg.norm(y.ravel())
    return d / n if n > 0 else d


def field_errors(a: State, b: State, fields=CELL_F64, existing_only=True) -> dict:
    a, b = _align(a, b)
    m = a.exists.astype(bool) if existing_only else None
    out = {}
    for f in fields:
        x, y = a.f64[f], b.f64[f]
        both_nan = np.isnan(x) & np.isnan(y)
        xx = np.where(both_nan, 0.0, x)
        yy = np.where(both_nan, 0.0, y)
        out[f] = rel_err(xx, yy, m)
    return out


def max_abs_diff(a: State, b: State, fields=CELL_F64, existing_only=True) -> dict:
    a, b = _align(a, b)
    m = a.exists.astype(bool) if existing_only else np.ones_like(a.exists, dtype=bool)
    out = {}
    for f in fields:
        x, y = a.f64[f][m], b.f64[f][m]
        same = (x == y) | (np.isnan(x) & np.isnan(y))
        out[f] = 0.0 if same.all() else float(np.nanmax(np.abs(x - y)))
    return out


def sorted_particles(s: State) -> np.ndarray:
    p = s.pos
    order = np.lexsort((p[:, 2], p[:, 1], p[:, 0]))
    return p[order]


def compare_particles(a: State, b: State, rtol=0.0, atol=0.0) -> float:
    if a.nparticles != b.nparticles:
        raise AssertionError(f"particle counts differ: {a.nparticles} vs {b.nparticles}")
    pa, pb = sorted_particles(a), sorted_particles(b)
    d = float(np.max(np.abs(pa - pb))) if len(pa) else 0.0
    if not np.allclose(pa, pb, rtol=rtol, atol=atol):
        raise AssertionError(f"particles differ, max abs {d}")
    return d


def fluid_mask(s: State):
    return s.exists.astype(bool) & np.isin(s.type, FLUID_TYPES)

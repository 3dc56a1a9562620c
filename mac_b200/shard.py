"""Slab decomposition of a brick world across ranks (host side).

The plan for a sharded step gives each rank a contiguous range of brick
z-keys, balanced by fluid cells, plus one layer of ghost bricks on each side
in z: every read a step makes from an owned cell (7-point stencils, the
convection's edge cells, the extrapolation's reach of two cells, the particle
move's 2x2x2 stencils of a particle that moves less than a cell) stays within
one brick of it. This module holds that decomposition and its two exchanges
over ``torch.distributed`` (gloo on the CPU, NCCL between GPUs):

* ``SlabPlan.balanced`` splits the z-keys; ``SlabPlan.local`` cuts a rank's
  owned and ghost bricks (and its particles) out of a world;
* ``exchange_ghosts`` refreshes the ghost bricks' fields from their owners;
* ``migrate_particles`` hands particles that left a rank's slab to the rank
  that owns them now.

The device step itself is not sharded: each rank would run the brick kernels
on its slab and call these exchanges at the step's phase boundaries (the
per-phase plan is in the design notes). The exchanges use point-to-point
messages with the neighbour ranks only, every rank taking the same steps in
the same order.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .state import BRICK, BRICK_CELLS, CELL_F64, FLUID_TYPES, State

# per-cell fields carried by the ghost exchange
GHOST_FIELDS = CELL_F64 + ("exists", "flags", "type", "layer", "depth")


@dataclasses.dataclass
class LocalSlab:
    """One rank's part of a world: its owned bricks, the ghost bricks around
    them (both in ``state``, owned first) and the particles in its slab."""
    rank: int
    state: State
    owned: np.ndarray  # (nb,) bool: brick owned (else ghost)


def _subset(state: State, sel: np.ndarray, pos: np.ndarray) -> State:
    return State(params=state.params, keys=state.keys[sel].copy(), exists=state.exists[sel].copy(),
                 f64={k: v[sel].copy() for k, v in state.f64.items()}, flags=state.flags[sel].copy(),
                 type=state.type[sel].copy(), layer=state.layer[sel].copy(), id=state.id[sel].copy(),
                 pos=pos.copy(), depth=state.depth[sel].copy())


@dataclasses.dataclass
class SlabPlan:
    z_lo: np.ndarray  # (nranks,) first owned brick z-key
    z_hi: np.ndarray  # (nranks,) one past the last owned brick z-key

    @property
    def nranks(self) -> int:
        return len(self.z_lo)

    @classmethod
    def balanced(cls, state: State, nranks: int) -> "SlabPlan":
        """Contiguous z ranges with about the same number of fluid cells each
        (every rank at least one z-layer of bricks)."""
        kz = state.keys[:, 2]
        z0, z1 = int(kz.min()), int(kz.max()) + 1
        if z1 - z0 < nranks:
            raise ValueError(f"{z1 - z0} brick layers cannot be split over {nranks} ranks")
        fluid = (np.isin(state.type, FLUID_TYPES) & (state.exists != 0)).sum(axis=1)
        per_layer = np.bincount(kz - z0, weights=fluid, minlength=z1 - z0).astype(np.float64)
        # cells of empty layers still count a little, so every layer has a weight
        per_layer += 1e-3 * BRICK_CELLS
        cum = np.concatenate([[0.0], np.cumsum(per_layer)])
        cuts = [z0]
        for r in range(1, nranks):
            target = cum[-1] * r / nranks
            c = z0 + int(np.searchsorted(cum, target))
            c = max(c, cuts[-1] + 1)                 # at least one layer for rank r - 1
            c = min(c, z1 - (nranks - r))            # leave one layer for each later rank
            cuts.append(c)
        cuts.append(z1)
        return cls(z_lo=np.array(cuts[:-1]), z_hi=np.array(cuts[1:]))

    def owner(self, kz: np.ndarray) -> np.ndarray:
        """Rank owning brick z-key kz (the end ranks also own everything
        beyond the planned range on their side)."""
        r = np.searchsorted(self.z_hi, kz, side="right")
        return np.clip(r, 0, self.nranks - 1)

    def particle_owner(self, state: State, pos: np.ndarray) -> np.ndarray:
        """Owning rank of each particle: by the brick of the cell holding it
        (cell key = round(pos / h), as the reference's Particle_To_Key)."""
        kz_cell = np.rint(pos[:, 2] / state.params.h[2]).astype(np.int64)
        return self.owner(np.floor_divide(kz_cell, BRICK))

    def local(self, state: State, rank: int) -> LocalSlab:
        kz = state.keys[:, 2]
        lo, hi = int(self.z_lo[rank]), int(self.z_hi[rank])
        own = self.owner(kz) == rank
        ghost = ~own & ((kz == lo - 1) | (kz == hi))
        order = np.concatenate([np.flatnonzero(own), np.flatnonzero(ghost)])
        pos = state.pos[self.particle_owner(state, state.pos) == rank] if len(state.pos) else state.pos
        sub = _subset(state, order, pos)
        return LocalSlab(rank=rank, state=sub, owned=np.arange(len(order)) < int(own.sum()))


def _field(state: State, name: str) -> np.ndarray:
    return state.f64[name] if name in state.f64 else getattr(state, name)


def _pack(state: State, sel: np.ndarray):
    keys = state.keys[sel].astype(np.int64)
    parts = [np.ascontiguousarray(_field(state, f)[sel]).view(np.uint8).reshape(len(keys), -1) for f in GHOST_FIELDS]
    return keys, np.concatenate(parts, axis=1) if len(keys) else np.zeros((0, 0), np.uint8)


def _unpack(state: State, rows: np.ndarray, blob: np.ndarray) -> None:
    col = 0
    for f in GHOST_FIELDS:
        a = _field(state, f)
        width = BRICK_CELLS * a.dtype.itemsize
        a[rows] = blob[:, col:col + width].copy().view(a.dtype).reshape(len(rows), BRICK_CELLS)
        col += width


def _exchange(arrays_to, group):
    """Send arrays_to[peer] (an int64 or uint8 numpy array) to each neighbour
    peer and receive theirs; sizes travel first. Non-blocking both ways so
    that neither side waits on the other's receive."""
    import torch
    import torch.distributed as dist
    peers = sorted(arrays_to)
    shapes = {}
    reqs = []
    for p in peers:
        a = arrays_to[p]
        hdr = torch.tensor([a.shape[0], a.shape[1] if a.ndim > 1 else 0, 1 if a.dtype == np.uint8 else 0],
                           dtype=torch.int64)
        reqs.append(dist.isend(hdr, p, group=group))
        shapes[p] = torch.zeros(3, dtype=torch.int64)
        reqs.append(dist.irecv(shapes[p], p, group=group))
    for r in reqs:
        r.wait()
    reqs, got = [], {}
    for p in peers:
        a = np.ascontiguousarray(arrays_to[p])
        if a.size:
            reqs.append(dist.isend(torch.from_numpy(a.copy()), p, group=group))
        n, m, is_u8 = (int(v) for v in shapes[p])
        shape = (n, m) if m else (n,)
        buf = torch.zeros(shape, dtype=torch.uint8 if is_u8 else torch.int64)
        if buf.numel():
            reqs.append(dist.irecv(buf, p, group=group))
        got[p] = buf
    for r in reqs:
        r.wait()
    return {p: got[p].numpy() for p in peers}


def _neighbours(plan: SlabPlan, rank: int):
    return [p for p in (rank - 1, rank + 1) if 0 <= p < plan.nranks]


def exchange_ghosts(local: LocalSlab, plan: SlabPlan, group=None) -> int:
    """Refresh every ghost brick of ``local`` with its owner's fields (all
    cell fields of ``GHOST_FIELDS``); returns the ghost bricks written."""
    st, rank = local.state, local.rank
    kz = st.keys[:, 2]
    lo, hi = int(plan.z_lo[rank]), int(plan.z_hi[rank])
    keys_to, blob_to = {}, {}
    for p in _neighbours(plan, rank):
        edge = lo if p < rank else hi - 1
        sel = np.flatnonzero(local.owned & (kz == edge))
        keys_to[p], blob_to[p] = _pack(st, sel)
    keys_in = _exchange({p: k.reshape(-1, 3) if k.size else np.zeros((0, 3), np.int64) for p, k in keys_to.items()},
                        group)
    blobs_in = _exchange(blob_to, group)
    index = {tuple(k): i for i, k in enumerate(st.keys.tolist())}
    written = 0
    for p in keys_in:
        k = keys_in[p].reshape(-1, 3)
        rows = np.array([index.get(tuple(int(v) for v in kk), -1) for kk in k], dtype=np.int64)
        ok = rows >= 0
        if ok.any():
            _unpack(st, rows[ok], blobs_in[p][ok])
            written += int(ok.sum())
    return written


def migrate_particles(local: LocalSlab, plan: SlabPlan, group=None) -> int:
    """Send the particles that left this rank's slab to the neighbour rank
    owning them (a particle moves less than a brick per step) and append the
    ones received; returns the number received."""
    st, rank = local.state, local.rank
    pos = st.pos
    own = plan.particle_owner(st, pos) if len(pos) else np.zeros(0, np.int64)
    send = {}
    for p in _neighbours(plan, rank):
        send[p] = np.ascontiguousarray(pos[own == p]).view(np.int64).reshape(-1, 3)
    stray = (own != rank) & ~np.isin(own, _neighbours(plan, rank))
    if stray.any():
        raise ValueError(f"rank {rank}: {int(stray.sum())} particles moved past a neighbour slab")
    got = _exchange(send, group)
    keep = pos[own == rank]
    recv = [got[p].reshape(-1, 3).view(np.float64) for p in sorted(got)]
    st.pos = np.concatenate([keep] + recv, axis=0) if recv else keep
    return int(sum(len(r) for r in recv))

"""Host-side state container for the sparse brick grid.

A state mirrors one Mac world: the chunk grid of ``src/ChunkHashTable.h:22-160``
with 8^3 chunks (called bricks here), every cell's two staggered speed buffers and
acceleration (``src/Data_Chunk_Speed.h:13-15``), pressure, material
(``src/Data_CellType_Fluid_Air_Solid_Inflow.h:24``), no-delete mark, const-face
bits (``src/Data_Grid_Speed.h:54-59``), layer and solver id, plus the particle
list (``src/TableContainerList.h:24-25``) and the timing data
(``src/Data_Timing_Time.h:7-9``).

All 512 cells of a live brick are kept, existing or not: the reference keeps the
data of erased cells of a live chunk and reuses it when ``operator[]`` re-creates
the cell (``src/ChunkHashTable.tpp:62-87``).

The binary file layout is the one documented in ``oracle/state_format.h`` (the
tests exchange states with the checkers through it).
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

BRICK = 8
BRICK_CELLS = 512
AIR, FLUID, SOLID, INFLOW = 0, 1, 2, 3
# The Interior material of Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres
# (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:3-22): a fluid cell
# deep enough below the surface to carry no particles (depth composition only).
INTERIOR = 4
FLUID_TYPES = (FLUID, INFLOW, INTERIOR)
FLAG_CONST = (1, 2, 4)
FLAG_NODELETE = 8

_HDR = struct.Struct("<8sqq3d6dii Q ii d 6i 104x")
assert _HDR.size == 256

CELL_F64 = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")


@dataclasses.dataclass
class Params:
    """World parameters (spacing, CFL factor, dt clamp, gravity, layer depth)."""
    h: tuple = (0.05, 0.05, 0.05)
    t: float = 0.0
    dt: float = 0.0
    cfl_factor: float = 0.5
    dt_min: float = 0.0
    dt_max: float = 0.1
    gravity: float = -9.81
    gravity_axis: int = 3
    layer_max: int = 4
    step: int = 0
    interp_symmetric: int = 1
    viscosity: float = 0.0
    # depth composition of the topology (test/Jet3.cpp:519-549): Policy_Depth(max,
    # interior, remove); 0 = the pipeline-A topology without depth
    depth_mode: int = 0
    depth_max: int = 0
    depth_interior: int = 0
    depth_remove: int = 0
    # inflow refill: 0 = 8 jittered particles, n >= 1 = Policy_Add_Particle_Cube(n)
    refill_cube: int = 0
    # 0: pipeline A step (RK2-TVD); 1: pipeline B step (Algorithms_RungeKutta_all),
    # a run-time choice, not stored in state files
    pipeline: int = 0


@dataclasses.dataclass
class State:
    params: Params
    keys: np.ndarray          # (nb, 3) int32 brick keys
    exists: np.ndarray        # (nb, 512) uint8
    f64: dict                 # name -> (nb, 512) float64, names in CELL_F64
    flags: np.ndarray         # (nb, 512) uint8
    type: np.ndarray          # (nb, 512) uint8
    layer: np.ndarray         # (nb, 512) int32
    id: np.ndarray            # (nb, 512) int32
    pos: np.ndarray           # (np, 3) float64
    depth: np.ndarray = None  # (nb, 512) int32, -1 = empty (src/Data_Grid_Depth_Empty.h:6-14)

    def __post_init__(self):
        if self.depth is None:
            self.depth = np.full(self.layer.shape, -1, dtype=np.int32)

    @property
    def nbricks(self) -> int:
        return int(self.keys.shape[0])

    @property
    def nparticles(self) -> int:
        return int(self.pos.shape[0])

    # ------------------------------------------------------------------ io
    def write(self, path: str) -> None:
        pr = self.params
        hdr = _HDR.pack(b"MACST002", self.nbricks, self.nparticles, *pr.h, pr.t, pr.dt,
                        pr.cfl_factor, pr.dt_min, pr.dt_max, pr.gravity, pr.gravity_axis,
                        pr.layer_max, pr.step, pr.interp_symmetric, 0, pr.viscosity, pr.depth_mode,
                        pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube, 0)
        with open(path, "wb") as f:
            f.write(hdr)
            f.write(np.ascontiguousarray(self.keys, dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(self.exists, dtype="u1").tobytes())
            for n in CELL_F64:
                f.write(np.ascontiguousarray(self.f64[n], dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(self.flags, dtype="u1").tobytes())
            f.write(np.ascontiguousarray(self.type, dtype="u1").tobytes())
            f.write(np.ascontiguousarray(self.layer, dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(self.id, dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(self.depth, dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(self.pos, dtype="<f8").tobytes())

    @staticmethod
    def read(path: str) -> "State":
        with open(path, "rb") as f:
            buf = f.read()
        (magic, nb, npart, h0, h1, h2, t, dt, cfl, dtmin, dtmax, g, gax, lmax, step, isym,
         _r, visc, dmode, dmax, dint, drem, cube, _r2) = _HDR.unpack_from(buf, 0)
        if magic != b"MACST002":
            raise ValueError(f"{path}: not a state file")
        off = _HDR.size
        nc = nb * BRICK_CELLS

        def take(dtype, count, shape):
            nonlocal off
            a = np.frombuffer(buf, dtype=dtype, count=count, offset=off).reshape(shape).copy()
            off += a.nbytes
            return a

        keys = take("<i4", nb * 3, (nb, 3))
        exists = take("u1", nc, (nb, BRICK_CELLS))
        f64 = {n: take("<f8", nc, (nb, BRICK_CELLS)) for n in CELL_F64}
        flags = take("u1", nc, (nb, BRICK_CELLS))
        typ = take("u1", nc, (nb, BRICK_CELLS))
        layer = take("<i4", nc, (nb, BRICK_CELLS))
        ids = take("<i4", nc, (nb, BRICK_CELLS))
        depth = take("<i4", nc, (nb, BRICK_CELLS))
        pos = take("<f8", npart * 3, (npart, 3))
        params = Params(h=(h0, h1, h2), t=t, dt=dt, cfl_factor=cfl, dt_min=dtmin, dt_max=dtmax,
                        gravity=g, gravity_axis=gax, layer_max=lmax, step=step,
                        interp_symmetric=isym, viscosity=visc, depth_mode=dmode, depth_max=dmax,
                        depth_interior=dint, depth_remove=drem, refill_cube=cube)
        return State(params, keys, exists, f64, flags, typ, layer, ids, pos, depth)

    def save_npz(self, path: str) -> None:
        """Compressed copy (used for the committed fixtures)."""
        pr = self.params
        hdr = np.array([*pr.h, pr.t, pr.dt, pr.cfl_factor, pr.dt_min, pr.dt_max, pr.gravity, pr.gravity_axis,
                        pr.layer_max, pr.step, pr.interp_symmetric, pr.viscosity, pr.depth_mode, pr.depth_max,
                        pr.depth_interior, pr.depth_remove, pr.refill_cube], dtype=np.float64)
        np.savez_compressed(path, hdr=hdr, keys=self.keys, exists=self.exists, flags=self.flags, type=self.type,
                            layer=self.layer, id=self.id, pos=self.pos, depth=self.depth, **self.f64)

    @staticmethod
    def load_npz(path: str) -> "State":
        z = np.load(path)
        h = z["hdr"]
        pr = Params(h=(h[0], h[1], h[2]), t=h[3], dt=h[4], cfl_factor=h[5], dt_min=h[6], dt_max=h[7],
                    gravity=h[8], gravity_axis=int(h[9]), layer_max=int(h[10]), step=int(h[11]),
                    interp_symmetric=int(h[12]), viscosity=float(h[13]) if h.size > 13 else 0.0)
        if h.size > 18:
            pr.depth_mode, pr.depth_max, pr.depth_interior, pr.depth_remove, pr.refill_cube = (int(v) for v in h[14:19])
        return State(pr, z["keys"], z["exists"], {n: z[n] for n in CELL_F64}, z["flags"], z["type"], z["layer"],
                     z["id"], z["pos"], z["depth"] if "depth" in z.files else None)

    @staticmethod
    def load(path: str) -> "State":
        return State.load_npz(path) if path.endswith(".npz") else State.read(path)

    # ------------------------------------------------------------- queries
    def cell_keys(self) -> np.ndarray:
        """(nb, 512, 3) integer cell keys of every slot."""
        o = np.arange(BRICK_CELLS)
        local = np.stack([o % 8, (o // 8) % 8, o // 64], axis=-1)
        return self.keys[:, None, :].astype(np.int64) * BRICK + local[None, :, :]

    def fluid_cells(self) -> int:
        ex = self.exists.astype(bool)
        return int(np.count_nonzero(ex & np.isin(self.type, FLUID_TYPES)))

    def sorted(self) -> "State":
        """Bricks in (z, y, x) key order (the canonical order of state files)."""
        order = np.lexsort((self.keys[:, 0], self.keys[:, 1], self.keys[:, 2]))
        return State(self.params, self.keys[order], self.exists[order],
                     {n: v[order] for n, v in self.f64.items()}, self.flags[order],
                     self.type[order], self.layer[order], self.id[order], self.pos, self.depth[order])


def from_cells(params: Params, keys, typ, flags, u, pos=None) -> State:
    """Builds a state from a list of existing cells (an experiment's ``main()``
    creates them one by one with ``grid[v]``: ``test/TestJetDEau_Basic.cpp:273-284``).
    ``keys`` (n,3) int, ``typ``/``flags`` (n,) uint8, ``u`` (n,3) float64 speed 0;
    later duplicates of a key override earlier ones."""
    keys = np.asarray(keys, dtype=np.int64).reshape(-1, 3)
    n = keys.shape[0]
    bk = np.floor_divide(keys, BRICK)
    ub, inv = np.unique(bk, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    order = np.lexsort((ub[:, 0], ub[:, 1], ub[:, 2]))
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    ub = ub[order]
    bidx = rank[inv]
    loc = keys - bk * BRICK
    off = loc[:, 0] + 8 * loc[:, 1] + 64 * loc[:, 2]
    st = empty_state(params, ub.astype(np.int32))
    st.exists[bidx, off] = 1
    st.type[bidx, off] = np.asarray(typ, dtype=np.uint8).reshape(n)
    st.flags[bidx, off] = np.asarray(flags, dtype=np.uint8).reshape(n)
    u = np.asarray(u, dtype=np.float64).reshape(n, 3)
    st.f64["u0x"][bidx, off] = u[:, 0]
    st.f64["u0y"][bidx, off] = u[:, 1]
    st.f64["u0z"][bidx, off] = u[:, 2]
    if pos is not None:
        st.pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    return st


def _box(x0, x1, y0, y1, z0, z1):
    z, y, x = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1),
                          indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=-1)


def empty_state(params: Params, keys: np.ndarray) -> State:
    nb = keys.shape[0]
    z = lambda dt: np.zeros((nb, BRICK_CELLS), dtype=dt)
    return State(params, keys.astype(np.int32), z(np.uint8), {n: z(np.float64) for n in CELL_F64},
                 z(np.uint8), z(np.uint8), np.full((nb, BRICK_CELLS), -1, np.int32),
                 np.full((nb, BRICK_CELLS), -1, np.int32), np.zeros((0, 3), np.float64))


def jet_world(nx=32, ny=32, nz=64, h=0.05, r_inflow=4.0, w_inflow=1.0, pool_depth=0,
              layer_max=4, cfl=0.5, dt_max=0.1, particles_per_cell=8, seed=1) -> State:
    """Vertical water jet in a walled box (the jet experiments' setup, with solid
    side walls and floor): cells 0..nx-1 x 0..ny-1 x 0..nz-1 are open, the walls
    at x,y = -1 / n and the floor at z = -1 are Solid, a disc of radius
    ``r_inflow`` cells centred on the floor is Inflow with a const face speed
    ``w_inflow`` (``test/Jet3.cpp:448-470`` builds its inflow the same way).
    ``pool_depth`` > 0 fills z < pool_depth with fluid particles at
    ``particles_per_cell`` jittered particles per cell (seeded)."""
    pr = Params(h=(h, h, h), cfl_factor=cfl, dt_max=dt_max, layer_max=layer_max)
    walls = [
        _box(-1, -1, -1, ny, -1, nz - 1), _box(nx, nx, -1, ny, -1, nz - 1),
        _box(0, nx - 1, -1, -1, -1, nz - 1), _box(0, nx - 1, ny, ny, -1, nz - 1),
        _box(0, nx - 1, 0, ny - 1, -1, -1),
    ]
    wk = np.concatenate(walls, axis=0)
    fl = _box(0, nx - 1, 0, ny - 1, 0, 0)
    cx, cy = (nx - 1) / 2.0, (ny - 1) / 2.0
    disc = fl[(fl[:, 0] - cx) ** 2 + (fl[:, 1] - cy) ** 2 <= r_inflow ** 2]
    keys = np.concatenate([wk, disc], axis=0)
    typ = np.concatenate([np.full(len(wk), SOLID, np.uint8), np.full(len(disc), INFLOW, np.uint8)])
    flags = np.concatenate([np.zeros(len(wk), np.uint8), np.full(len(disc), FLAG_CONST[2], np.uint8)])
    u = np.zeros((len(keys), 3))
    u[len(wk):, 2] = w_inflow
    pos = None
    if pool_depth > 0:
        pos = pool_particles(nx, ny, pool_depth, h, particles_per_cell, seed)
    return from_cells(pr, keys, typ, flags, u, pos)


def lateral_jet_world(nx=384, ny=192, nz=192, h=0.01, r_inflow=16.0, speed=3.0, angle_deg=15.0, z_centre=None,
                      layer_max=4, cfl=0.5, dt_max=0.01) -> State:
    """Lateral jet: cells 0..nx-1 x 0..ny-1 x 0..nz-1 open, solid walls at
    x = -1 / nx, y = -1 / ny and the floor z = -1. A disc of radius
    ``r_inflow`` cells on the x = 0 plane (centred at y = (ny-1)/2, z =
    ``z_centre``, default nz/4) is Inflow with face speed ``speed`` aimed
    ``angle_deg`` above horizontal and all three faces const, as the reference's
    lateral jet sets its inflow cells (``test/Lateral_jet_3.cpp:416-440``)."""
    pr = Params(h=(h, h, h), cfl_factor=cfl, dt_max=dt_max, layer_max=layer_max)
    walls = [
        _box(-1, -1, -1, ny, -1, nz - 1), _box(nx, nx, -1, ny, -1, nz - 1),
        _box(0, nx - 1, -1, -1, -1, nz - 1), _box(0, nx - 1, ny, ny, -1, nz - 1),
        _box(0, nx - 1, 0, ny - 1, -1, -1),
    ]
    wk = np.concatenate(walls, axis=0)
    plane = _box(0, 0, 0, ny - 1, 0, nz - 1)
    cy = (ny - 1) / 2.0
    cz = nz / 4.0 if z_centre is None else float(z_centre)
    disc = plane[(plane[:, 1] - cy) ** 2 + (plane[:, 2] - cz) ** 2 <= r_inflow ** 2]
    keys = np.concatenate([wk, disc], axis=0)
    typ = np.concatenate([np.full(len(wk), SOLID, np.uint8), np.full(len(disc), INFLOW, np.uint8)])
    flags = np.concatenate([np.zeros(len(wk), np.uint8), np.full(len(disc), 7, np.uint8)])
    u = np.zeros((len(keys), 3))
    a = np.deg2rad(angle_deg)
    u[len(wk):, 0] = speed * np.cos(a)
    u[len(wk):, 2] = speed * np.sin(a)
    return from_cells(pr, keys, typ, flags, u)


def pool_spheres_world(n=128, nspheres=12, r_range=(6.0, 20.0), pool_frac=0.4, seed=2, vel_seed=3) -> State:
    """Standalone pressure-solve world: cells 0..n-1 on each axis with h = 1/n,
    fluid where z < pool_frac*n or inside one of ``nspheres`` balls (radius
    uniform in ``r_range`` cells, centre uniform in [r, n-r]^3, seeded), air
    elsewhere, and a solid shell on all six box faces. Every face speed of the
    open cells is uniform in [-1, 1] (seeded). Run ``world.setup_passes`` on it
    before use (const faces of the shell, as Algorithms_Solid_To_Const)."""
    h = 1.0 / n
    pr = Params(h=(h, h, h), cfl_factor=0.5, dt_max=0.01, layer_max=4)
    rng = np.random.default_rng(seed)
    cells = _box(0, n - 1, 0, n - 1, 0, n - 1)
    fluid = cells[:, 2] < pool_frac * n
    for _ in range(nspheres):
        r = rng.uniform(r_range[0], r_range[1])
        c = rng.uniform(r, n - r, size=3)
        fluid |= ((cells - c) ** 2).sum(axis=1) <= r * r
    shell = _box(-1, n, -1, n, -1, n)
    shell = shell[(shell.min(axis=1) < 0) | (shell.max(axis=1) >= n)]
    keys = np.concatenate([shell, cells], axis=0)
    typ = np.concatenate([np.full(len(shell), SOLID, np.uint8), np.where(fluid, FLUID, AIR).astype(np.uint8)])
    u = np.zeros((len(keys), 3))
    u[len(shell):] = np.random.default_rng(vel_seed).uniform(-1.0, 1.0, size=(len(cells), 3))
    s = from_cells(pr, keys, typ, np.zeros(len(keys), np.uint8), u)
    # fluid cells are layer 0 and the air cells layer 1, as after a topology pass
    s.layer[:] = np.where(s.exists.astype(bool), np.where(s.type == FLUID, 0, 1), -1)
    return s


def pool_particles(nx, ny, depth, h, ppc=8, seed=1):
    """Jittered 2x2x2 lattice (offsets +-h/4 plus uniform jitter in (-h/4, h/4))
    in every cell of the slab 0..nx-1 x 0..ny-1 x 0..depth-1."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(depth), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=-1).astype(np.float64)
    out = []
    for s in range(ppc):
        o = np.array([0.25 if (s >> i) & 1 else -0.25 for i in range(3)])
        j = (rng.random(base.shape) - 0.5) * 0.499
        out.append((base + o + j) * h)
    # cell-major: the particles of one cell are consecutive, cells in (z, y, x) order
    return np.stack(out, axis=1).reshape(-1, 3)

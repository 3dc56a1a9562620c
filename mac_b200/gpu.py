"""Python host binding of the C-ABI in include/mac_gpu.h (libmac_gpu.so).

The device library is the product; this module only moves numpy states across
the boundary and names the reference algorithms each call stands in for. It
fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .state import BRICK_CELLS, CELL_F64, Params, State

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmac_gpu.so")

MAC_OK = 0
ERRORS = {-1: "invalid", -2: "cuda", -3: "capacity", -4: "not converged", -5: "no device",
          -6: "out of memory", -7: "timeout", -8: "matrix form"}
SOLVERS = {"mgpcg64": 0, "mixed": 1, "cg64": 2, "learned": 3, "learned_mixed": 4}


class MacError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")
        self.code = code


class mac_params(ctypes.Structure):
    _fields_ = [("h", ctypes.c_double * 3), ("cfl_factor", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("dt_max", ctypes.c_double), ("gravity", ctypes.c_double), ("gravity_axis", ctypes.c_int32),
                ("layer_max", ctypes.c_int32), ("interp_symmetric", ctypes.c_int32), ("solver", ctypes.c_int32),
                ("rtol", ctypes.c_double), ("max_iters", ctypes.c_int32), ("warm_start", ctypes.c_int32),
                ("max_bricks", ctypes.c_int64), ("max_particles", ctypes.c_int64), ("device", ctypes.c_int32),
                ("div_check", ctypes.c_int32), ("viscosity", ctypes.c_double), ("depth_mode", ctypes.c_int32),
                ("depth_max", ctypes.c_int32), ("depth_interior", ctypes.c_int32), ("depth_remove", ctypes.c_int32),
                ("refill_cube", ctypes.c_int32), ("pipeline", ctypes.c_int32)]


_P = ctypes.POINTER


class mac_host_state(ctypes.Structure):
    _fields_ = [("nbricks", ctypes.c_int64), ("nparticles", ctypes.c_int64), ("keys", _P(ctypes.c_int32)),
                ("exists", _P(ctypes.c_uint8)), ("u", (_P(ctypes.c_double) * 3) * 2), ("acc", _P(ctypes.c_double) * 3),
                ("p", _P(ctypes.c_double)), ("flags", _P(ctypes.c_uint8)), ("type", _P(ctypes.c_uint8)),
                ("layer", _P(ctypes.c_int32)), ("pos", _P(ctypes.c_double)), ("t", ctypes.c_double),
                ("dt", ctypes.c_double), ("step", ctypes.c_uint64), ("depth", _P(ctypes.c_int32))]


class mac_stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("solves", ctypes.c_int32), ("relres", ctypes.c_double),
                ("max_div", ctypes.c_double), ("fluid_cells", ctypes.c_int64), ("unknowns", ctypes.c_int64),
                ("live_bricks", ctypes.c_int64), ("particles", ctypes.c_int64),
                ("total_iterations", ctypes.c_int64), ("learned_iterations", ctypes.c_int32),
                ("fallbacks", ctypes.c_int32)]


EXPORTS = ["mac_default_params", "mac_ctx_create", "mac_ctx_destroy", "mac_get_stats", "mac_error_string",
           "mac_upload_state", "mac_query_sizes", "mac_download_state", "mac_upload_field", "mac_download_field",
           "mac_pressure_init", "mac_pressure_divergence_projection", "mac_pressure_end", "mac_initialize_maccell",
           "mac_layer_initial_with_particle", "mac_create_fluid_particle", "mac_update_celltype_layer",
           "mac_delete_maccell", "mac_calculate_time_step", "mac_topology_rebuild", "mac_forces",
           "mac_pressure_project", "mac_extrapolate_boundary_condition", "mac_rk2tvd", "mac_rungekutta_all", "mac_extrapolate", "mac_move_particles", "mac_step", "mac_sync",
           "mac_stream", "mac_launch_count", "mac_set_profiling", "mac_get_profile",
           "mac_csc_factorize", "mac_csc_solve", "mac_csc_clean", "mac_csc_solve_noalloc",
           "mac_unet_create", "mac_unet_destroy", "mac_unet_nparams", "mac_unet_init", "mac_unet_get_params",
           "mac_unet_set_params", "mac_unet_forward", "mac_unet_loss_grad", "mac_unet_adam_step",
           "mac_unet_make_dataset", "mac_unet_make_dataset_ext", "mac_unet_get_sample", "mac_unet_train", "mac_unet_launch_count",
           "mac_set_preconditioner_net", "mac_set_learned_smoothing", "mac_set_multigrid", "mac_set_dependent_launch", "mac_set_concurrent_binning", "mac_set_coarse_block", "mac_set_smoother", "mac_unet_set_loss", "mac_unet_time_forward",
           "mac_unet_set_conv"]
PHASES = ["topology", "forces", "setup", "divergence", "spmv", "cg_vector", "vcycle", "gradient", "extrapolate",
          "move"]

_lib = None


def load(path: str = LIB_PATH):
    """Loads libmac_gpu.so; raises if it is absent (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m mac_b200.build`")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.mac_default_params.argtypes = [_P(mac_params)]
    lib.mac_default_params.restype = None
    lib.mac_ctx_create.argtypes = [_P(mac_params), _P(vp)]
    lib.mac_ctx_destroy.argtypes = [vp]
    lib.mac_get_stats.argtypes = [vp, _P(mac_stats)]
    lib.mac_error_string.argtypes = [ctypes.c_int]
    lib.mac_error_string.restype = ctypes.c_char_p
    lib.mac_upload_state.argtypes = [vp, _P(mac_host_state)]
    lib.mac_query_sizes.argtypes = [vp, _P(ctypes.c_int64), _P(ctypes.c_int64)]
    lib.mac_download_state.argtypes = [vp, _P(mac_host_state)]
    for n in ["mac_initialize_maccell", "mac_layer_initial_with_particle", "mac_create_fluid_particle",
              "mac_update_celltype_layer", "mac_delete_maccell", "mac_topology_rebuild", "mac_rk2tvd",
              "mac_rungekutta_all",
              "mac_extrapolate", "mac_move_particles", "mac_step", "mac_sync", "mac_csc_clean",
              "mac_pressure_init", "mac_pressure_end"]:
        getattr(lib, n).argtypes = [vp]
    lib.mac_calculate_time_step.argtypes = [vp, _P(ctypes.c_double)]
    lib.mac_forces.argtypes = [vp, ctypes.c_int]
    lib.mac_extrapolate_boundary_condition.argtypes = [vp, ctypes.c_int]
    lib.mac_pressure_project.argtypes = [vp, ctypes.c_int]
    lib.mac_pressure_divergence_projection.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.mac_upload_field.argtypes = [vp, ctypes.c_int, _P(ctypes.c_double)]
    lib.mac_download_field.argtypes = [vp, ctypes.c_int, _P(ctypes.c_double)]
    lib.mac_csc_factorize.argtypes = [vp, ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_double)]
    lib.mac_csc_solve.argtypes = [vp, ctypes.c_int, _P(ctypes.c_double), _P(ctypes.c_double)]
    lib.mac_stream.argtypes = [vp, _P(vp)]
    lib.mac_launch_count.argtypes = [vp, _P(ctypes.c_int64)]
    lib.mac_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.mac_get_profile.argtypes = [vp, _P(ctypes.c_double), _P(ctypes.c_int64), ctypes.c_int]
    # Device pointers are passed as integers (c_void_p).
    lib.mac_csc_solve_noalloc.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int,
                                          _P(ctypes.c_int), _P(ctypes.c_double)]
    i32, i64, f32, f64 = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double
    lib.mac_unet_create.argtypes = [i32, _P(vp)]
    lib.mac_unet_destroy.argtypes = [vp]
    lib.mac_unet_nparams.argtypes = [vp, _P(i64)]
    lib.mac_unet_init.argtypes = [vp, ctypes.c_uint64]
    lib.mac_unet_get_params.argtypes = [vp, _P(f32), _P(f32)]
    lib.mac_unet_set_params.argtypes = [vp, _P(f32), f32]
    lib.mac_unet_forward.argtypes = [vp, i32, i32, i32, i32, _P(f32), _P(ctypes.c_int8), _P(f32)]
    lib.mac_unet_loss_grad.argtypes = [vp, i32, i32, i32, i32, _P(f32), _P(ctypes.c_int8), _P(f32), _P(f64),
                                       _P(f32)]
    lib.mac_unet_adam_step.argtypes = [vp, _P(f32), f32]
    lib.mac_unet_make_dataset.argtypes = [vp, i32, i32, i32, i32, ctypes.c_uint64, _P(f64)]
    lib.mac_unet_make_dataset_ext.argtypes = [vp, i32, i32, i32, i32, ctypes.c_uint64, _P(ctypes.c_int8), i32,
                                              _P(f64)]
    lib.mac_unet_get_sample.argtypes = [vp, i32, _P(f32), _P(f32), _P(ctypes.c_int8)]
    lib.mac_unet_train.argtypes = [vp, i32, i32, f32, ctypes.c_uint64, _P(f32)]
    lib.mac_unet_launch_count.argtypes = [vp, _P(i64)]
    lib.mac_set_preconditioner_net.argtypes = [vp, vp]
    lib.mac_set_learned_smoothing.argtypes = [vp, f64]
    lib.mac_set_multigrid.argtypes = [vp, i32, i32]
    lib.mac_set_dependent_launch.argtypes = [vp, i32]
    lib.mac_set_concurrent_binning.argtypes = [vp, i32]
    lib.mac_set_coarse_block.argtypes = [vp, i32]
    lib.mac_set_smoother.argtypes = [vp, f64, f64, f64, f64]
    lib.mac_unet_set_loss.argtypes = [vp, i32]
    lib.mac_unet_time_forward.argtypes = [vp, i32, i32, i32, i32, i32, _P(f64), _P(f64)]
    lib.mac_unet_set_conv.argtypes = [vp, i32]
    _lib = lib
    return lib


def _ptr(a, ct):
    return a.ctypes.data_as(_P(ct))


def make_params(pr: Params, max_bricks: int, max_particles: int, solver="mgpcg64", rtol=1e-8, max_iters=500,
                warm_start=False, device=0, div_check=True) -> mac_params:
    p = mac_params()
    load().mac_default_params(ctypes.byref(p))
    for i in range(3):
        p.h[i] = pr.h[i]
    p.cfl_factor = pr.cfl_factor
    p.dt_min = pr.dt_min
    p.dt_max = pr.dt_max
    p.gravity = pr.gravity
    p.gravity_axis = pr.gravity_axis
    p.layer_max = pr.layer_max
    p.interp_symmetric = pr.interp_symmetric
    p.solver = SOLVERS[solver]
    p.rtol = rtol
    p.max_iters = max_iters
    p.warm_start = int(warm_start)
    p.max_bricks = int(max_bricks)
    p.max_particles = int(max_particles)
    p.device = device
    p.div_check = int(div_check)
    p.viscosity = float(getattr(pr, "viscosity", 0.0))
    for k in ("depth_mode", "depth_max", "depth_interior", "depth_remove", "refill_cube", "pipeline"):
        setattr(p, k, int(getattr(pr, k, 0)))
    return p


class HostState:
    """Host arrays laid out as mac_host_state expects (optionally in pinned
    memory); ``depth`` carries the per-cell depth of the depth composition."""

    # speed buffer 1 and the acceleration: RK2-TVD's stage buffers
    STAGE = ("u1x", "u1y", "u1z", "ax", "ay", "az")

    def __init__(self, nbricks: int, nparticles: int, pinned: bool = False, depth: bool = False,
                 stage_buffers: bool = True):
        """stage_buffers=False leaves speed buffer 1 and the acceleration out
        (NULL in mac_host_state: not transferred either way)."""
        nc = nbricks * BRICK_CELLS
        if pinned:
            import torch
            alloc = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
            f64 = lambda n: alloc(n, torch.float64)
            u8 = lambda n: alloc(n, torch.uint8)
            i32 = lambda n: alloc(n, torch.int32)
        else:
            f64 = lambda n: np.empty(n, np.float64)
            u8 = lambda n: np.empty(n, np.uint8)
            i32 = lambda n: np.empty(n, np.int32)
        self.nbricks, self.nparticles = nbricks, nparticles
        self.cap_bricks, self.cap_particles = nbricks, nparticles
        self.keys = i32(3 * max(nbricks, 1))
        self.exists = u8(max(nc, 1))
        self.fields = [n for n in CELL_F64 if stage_buffers or n not in self.STAGE]
        self.f64 = {n: f64(max(nc, 1)) for n in self.fields}
        self.flags = u8(max(nc, 1))
        self.type = u8(max(nc, 1))
        self.layer = i32(max(nc, 1))
        self.depth = i32(max(nc, 1)) if depth else None
        self.pos = f64(3 * max(nparticles, 1))
        self.t = self.dt = 0.0
        self.step = 0

    def fill(self, s: State) -> "HostState":
        nb, nc = s.nbricks, s.nbricks * BRICK_CELLS
        self.keys[:3 * nb] = s.keys.reshape(-1)
        self.exists[:nc] = s.exists.reshape(-1)
        for n in self.fields:
            self.f64[n][:nc] = s.f64[n].reshape(-1)
        self.flags[:nc] = s.flags.reshape(-1)
        self.type[:nc] = s.type.reshape(-1)
        self.layer[:nc] = s.layer.reshape(-1)
        if self.depth is not None:
            self.depth[:nc] = s.depth.reshape(-1)
        self.pos[:3 * s.nparticles] = s.pos.reshape(-1)
        self.nbricks, self.nparticles = nb, s.nparticles
        self.t, self.dt, self.step = s.params.t, s.params.dt, s.params.step
        return self

    def nbytes(self) -> int:
        """Bytes of the current state content (what one transfer moves)."""
        nc = self.nbricks * BRICK_CELLS
        per_cell = 1 + 8 * len(self.fields) + 1 + 1 + 4 + (4 if self.depth is not None else 0)
        return 12 * self.nbricks + nc * per_cell + 24 * self.nparticles

    def c_struct(self) -> mac_host_state:
        h = mac_host_state()
        h.nbricks, h.nparticles = self.nbricks, self.nparticles
        h.keys = _ptr(self.keys, ctypes.c_int32)
        h.exists = _ptr(self.exists, ctypes.c_uint8)
        f = lambda n: _ptr(self.f64[n], ctypes.c_double) if n in self.f64 else None
        for b in range(2):
            for i in range(3):
                h.u[b][i] = f(CELL_F64[3 * b + i])
        for i in range(3):
            h.acc[i] = f(CELL_F64[6 + i])
        h.p = _ptr(self.f64["p"], ctypes.c_double)
        h.flags = _ptr(self.flags, ctypes.c_uint8)
        h.type = _ptr(self.type, ctypes.c_uint8)
        h.layer = _ptr(self.layer, ctypes.c_int32)
        h.depth = _ptr(self.depth, ctypes.c_int32) if self.depth is not None else None
        h.pos = _ptr(self.pos, ctypes.c_double)
        h.t, h.dt, h.step = self.t, self.dt, self.step
        return h

    def to_state(self, params: Params) -> State:
        nb, nc, npart = self.nbricks, self.nbricks * BRICK_CELLS, self.nparticles
        shp = (nb, BRICK_CELLS)
        pr = Params(**{**params.__dict__})
        pr.t, pr.dt, pr.step = self.t, self.dt, self.step
        return State(pr, self.keys[:3 * nb].reshape(nb, 3).copy(), self.exists[:nc].reshape(shp).copy(),
                     {n: (self.f64[n][:nc].reshape(shp).copy() if n in self.f64 else np.zeros(shp))
                      for n in CELL_F64},
                     self.flags[:nc].reshape(shp).copy(), self.type[:nc].reshape(shp).copy(),
                     self.layer[:nc].reshape(shp).copy(), np.full(shp, -1, np.int32),
                     self.pos[:3 * npart].reshape(npart, 3).copy(),
                     self.depth[:nc].reshape(shp).copy() if self.depth is not None else None).sorted()


class Context:
    """One device context (one CUDA stream, its own device memory)."""

    def __init__(self, params: Params, max_bricks=4096, max_particles=1 << 20, **kw):
        self.lib = load()
        self.params = params
        self.cp = make_params(params, max_bricks, max_particles, **kw)
        h = ctypes.c_void_p()
        self._check(self.lib.mac_ctx_create(ctypes.byref(self.cp), ctypes.byref(h)), "mac_ctx_create")
        self.h = h

    def _check(self, rc, what, allow=()):
        if rc != MAC_OK and rc not in allow:
            raise MacError(rc, what)
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.mac_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- transfer
    def upload(self, s: State | None, host: HostState | None = None):
        """Uploads a State, or the content already held in ``host``."""
        host = host or HostState(s.nbricks, s.nparticles, depth=bool(s.params.depth_mode)).fill(s)
        self._host_in = host
        st = host.c_struct()
        self._check(self.lib.mac_upload_state(self.h, ctypes.byref(st)), "mac_upload_state")

    def sizes(self):
        nb, npart = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.mac_query_sizes(self.h, ctypes.byref(nb), ctypes.byref(npart)), "mac_query_sizes")
        return nb.value, npart.value

    def download(self, host: HostState | None = None, to_state: bool = True):
        """Reads the device state through mac_download_state into ``host`` (a
        new HostState if it is missing or too small). Returns it as a State
        (key-sorted copies of the arrays), or, with ``to_state=False``, the
        HostState itself with the arrays as the C-ABI wrote them."""
        nb, npart = self.sizes()
        if host is None or host.cap_bricks < nb or host.cap_particles < npart:
            host = HostState(nb, npart, depth=bool(self.params.depth_mode))
        host.nbricks, host.nparticles = nb, npart
        st = host.c_struct()
        self._check(self.lib.mac_download_state(self.h, ctypes.byref(st)), "mac_download_state")
        host.nbricks, host.nparticles = st.nbricks, st.nparticles
        host.t, host.dt, host.step = st.t, st.dt, st.step
        return host.to_state(self.params) if to_state else host

    def stats(self) -> dict:
        s = mac_stats()
        self._check(self.lib.mac_get_stats(self.h, ctypes.byref(s)), "mac_get_stats")
        return {k: getattr(s, k) for k, _ in mac_stats._fields_}

    # ---- the reference algorithms
    def topology(self):
        return self._check(self.lib.mac_topology_rebuild(self.h), "mac_topology_rebuild")

    def first_init_topology(self):
        """Initialize_MacCell, Create_Fluid_Particle, Layer_Initial_With_Particle,
        Update_CellType_Layer, Delete_MacCell in the first-init order
        (test/TestJetDEau_Basic.cpp:329-330)."""
        for n in ["mac_initialize_maccell", "mac_create_fluid_particle", "mac_layer_initial_with_particle",
                  "mac_update_celltype_layer", "mac_delete_maccell"]:
            self._check(getattr(self.lib, n)(self.h), n)

    def dt(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.mac_calculate_time_step(self.h, ctypes.byref(v)), "mac_calculate_time_step")
        return v.value

    def extrapolate_boundary_condition(self, ispeed=0):
        """Algorithm_Extrapolate_Boundary_Condition (3D form) in the device's fixed colour order."""
        return self._check(self.lib.mac_extrapolate_boundary_condition(self.h, ispeed),
                           "mac_extrapolate_boundary_condition")

    def forces(self, ispeed=0):
        return self._check(self.lib.mac_forces(self.h, ispeed), "mac_forces")

    def project(self, ispeed=0, allow_not_converged=False):
        return self._check(self.lib.mac_pressure_project(self.h, ispeed), "mac_pressure_project",
                           allow=(-4,) if allow_not_converged else ())

    # ---- the projection at Algorithms_Solve_Pressure's composable interface
    def pressure_init(self):
        """Init_Iteration (src/Algorithms_Solve_Pressure.h:44): the system of the current cells."""
        self._check(self.lib.mac_pressure_init(self.h), "mac_pressure_init")

    def divergence_projection(self, ispeed=0, accel=False, allow_not_converged=False):
        """Divergence_Projection (src/Algorithms_Solve_Pressure.h:168) on the last init's system."""
        return self._check(self.lib.mac_pressure_divergence_projection(self.h, ispeed, 1 if accel else 0),
                           "mac_pressure_divergence_projection", allow=(-4,) if allow_not_converged else ())

    def pressure_end(self):
        """End_Iteration (src/Algorithms_Solve_Pressure.h:158)."""
        self._check(self.lib.mac_pressure_end(self.h), "mac_pressure_end")

    FIELDS = ("u0x", "u0y", "u0z", "u1x", "u1y", "u1z", "ax", "ay", "az", "p")

    def upload_field(self, name, values):
        """One FP64 cell field, [nbricks * 512] in the device's brick order (that of download())."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self.lib.mac_upload_field(self.h, self.FIELDS.index(name), _ptr(v, ctypes.c_double)),
                    "mac_upload_field")

    def download_field(self, name):
        nb, _ = self.sizes()
        out = np.empty(nb * BRICK_CELLS, np.float64)
        self._check(self.lib.mac_download_field(self.h, self.FIELDS.index(name), _ptr(out, ctypes.c_double)),
                    "mac_download_field")
        return out

    def rk2tvd(self, allow_not_converged=False):
        return self._check(self.lib.mac_rk2tvd(self.h), "mac_rk2tvd", allow=(-4,) if allow_not_converged else ())

    def rungekutta_all(self, allow_not_converged=False):
        """Algorithms_RungeKutta_all of pipeline B (contexts created with pipeline=1)."""
        return self._check(self.lib.mac_rungekutta_all(self.h), "mac_rungekutta_all",
                           allow=(-4,) if allow_not_converged else ())

    def extrapolate(self):
        return self._check(self.lib.mac_extrapolate(self.h), "mac_extrapolate")

    def move(self):
        return self._check(self.lib.mac_move_particles(self.h), "mac_move_particles")

    def step(self, allow_not_converged=False):
        return self._check(self.lib.mac_step(self.h), "mac_step", allow=(-4,) if allow_not_converged else ())

    def sync(self):
        return self._check(self.lib.mac_sync(self.h), "mac_sync")

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.mac_stream(self.h, ctypes.byref(s)), "mac_stream")
        return s.value or 0

    def launches(self) -> int:
        n = ctypes.c_int64()
        self._check(self.lib.mac_launch_count(self.h, ctypes.byref(n)), "mac_launch_count")
        return n.value

    def set_profiling(self, on: bool):
        self._check(self.lib.mac_set_profiling(self.h, int(on)), "mac_set_profiling")

    def profile(self) -> dict:
        """Per-phase device milliseconds and region counts since the last call."""
        n = len(PHASES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        self._check(self.lib.mac_get_profile(self.h, ms, cnt, n), "mac_get_profile")
        return {PHASES[i]: (ms[i], cnt[i]) for i in range(n)}

    def set_preconditioner(self, net):
        """Attaches a mac_b200.unet.UNet (or None) for the "learned" solvers."""
        self._check(self.lib.mac_set_preconditioner_net(self.h, net.h if net is not None else None),
                    "mac_set_preconditioner_net")
        self._net = net

    def set_learned_smoothing(self, omega):
        self._check(self.lib.mac_set_learned_smoothing(self.h, float(omega)), "mac_set_learned_smoothing")

    def set_smoother(self, w1=0.5711, w2=1.8216, w_single=0.9, coarse_scale=0.6):
        """Multigrid smoother weights and coarse-operator scale (mac_set_smoother)."""
        self._check(self.lib.mac_set_smoother(self.h, float(w1), float(w2), float(w_single), float(coarse_scale)),
                    "mac_set_smoother")

    def set_multigrid(self, sweeps0=2, prefetch=False):
        """Jacobi sweeps before and after the coarse correction on the finest
        level (1 or 2); prefetch: the V-cycle's first kernel prefetches bricks
        with asynchronous bulk copies."""
        self._check(self.lib.mac_set_multigrid(self.h, int(sweeps0), 1 if prefetch else 0), "mac_set_multigrid")

    def set_dependent_launch(self, on=True):
        """CG-loop kernels launched with programmatic stream serialisation
        (default on) or in plain stream order; bit-identical results."""
        self._check(self.lib.mac_set_dependent_launch(self.h, 1 if on else 0), "mac_set_dependent_launch")

    def set_coarse_block(self, max_cells=1024):
        """Dense multigrid levels above max_cells cells as device-wide sweeps,
        the rest in the one-block coarse solve."""
        self._check(self.lib.mac_set_coarse_block(self.h, int(max_cells)), "mac_set_coarse_block")

    def set_concurrent_binning(self, on=True):
        """Particle binning on a second stream during RK2-TVD or inside the
        move (the default); bit-identical results."""
        self._check(self.lib.mac_set_concurrent_binning(self.h, 1 if on else 0), "mac_set_concurrent_binning")

    # ---- drop-in CSC solver
    def csc_solve(self, offset, indice, value, b):
        off = np.ascontiguousarray(offset, dtype=np.int32)
        ind = np.ascontiguousarray(indice, dtype=np.int32)
        val = np.ascontiguousarray(value, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        n = len(off) - 1
        x = np.zeros(n, np.float64)
        self._check(self.lib.mac_csc_factorize(self.h, n, _ptr(off, ctypes.c_int), _ptr(ind, ctypes.c_int),
                                               _ptr(val, ctypes.c_double)), "mac_csc_factorize")
        self._check(self.lib.mac_csc_solve(self.h, n, _ptr(bb, ctypes.c_double), _ptr(x, ctypes.c_double)),
                    "mac_csc_solve")
        self._check(self.lib.mac_csc_clean(self.h), "mac_csc_clean")
        return x

"""Benchmark: fluid cell-steps/s of the full Mac step at Poisson relative residual 1e-8.

Workload (default): the 256x256x512 vertical jet (h = 0.01 m, inflow radius 24
cells at w = 2.0 m/s, gravity -9.81 z, solid side walls and floor, LayerMax 4,
CFL 0.5) in a synthetic spun-up state: a pool of depth 122 cells (~8.0M fluid
cells) with 8 jittered particles per fluid cell (~64M particles). Each step is
the reference's whole step (test/TestJetDEau_Basic.cpp:434-441): topology
rebuild, CFL time step, RK2-TVD with gravity + upwind convection and two
pressure projections (FP64 CG with the FP32 multigrid preconditioner, to an
FP64 relative residual of 1e-8; --solver mgpcg64 for the all-FP64 form), air-layer
extrapolation, RK4 particle move.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The timed steps run without per-phase events; the phase times and rooflines
in the line come from a few further, profiled steps of the same run.

--impl reference times the reference's own code (compiled from its headers into
oracle/_ref/mac_ref; its solver stand-in is FP64 Jacobi-CG at 1e-8) on the
host cores, one single-threaded process per core, each on a bounded sub-box of
the same jet.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fluid cell-steps/s at Poisson rel-resid 1e-8 (full advect+project step)"
UNIT = "cell-steps/s"

WORKLOADS = {
    # name: (nx, ny, nz, h, r_inflow, w_inflow, pool_depth, dt_max, max_bricks, max_particles)
    "jet256": (256, 256, 512, 0.01, 24.0, 2.0, 122, 0.01, 40000, 80_000_000),
    "jet128": (128, 128, 256, 0.01, 24.0, 2.0, 61, 0.01, 8000, 12_000_000),
    "jet32": (32, 32, 64, 0.05, 4.0, 1.0, 0, 0.1, 1024, 1 << 20),
}
# Bounded sample of the jet for the CPU arms: a sub-box with the same spacing,
# inflow and pool fraction.
CPU_SAMPLE = (48, 48, 96, 0.01, 12.0, 2.0, 23, 0.01)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ world
def make_world(name):
    from mac_b200.state import jet_world
    nx, ny, nz, h, r, w, depth, dt_max = WORKLOADS[name][:8]
    return jet_world(nx, ny, nz, h=h, r_inflow=r, w_inflow=w, pool_depth=depth, dt_max=dt_max, seed=1)


def sample_world():
    from mac_b200.state import jet_world
    nx, ny, nz, h, r, w, depth, dt_max = CPU_SAMPLE
    return jet_world(nx, ny, nz, h=h, r_inflow=r, w_inflow=w, pool_depth=depth, dt_max=dt_max, seed=1)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- CPU arms
def _ref_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "mac_ref")
    return p if os.path.exists(p) else None


def cpu_reference_run(steps, procs, tmpdir):
    """Runs the reference's own code (or, when it was not built, the oracle port)
    on `procs` independent replicas of the bounded sample, `steps` steps each,
    concurrently; returns (fluid cell-steps/s, kind, seconds, fluid_cell_steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    s = sample_world()
    setup = os.path.join(tmpdir, "sample_setup.state")
    s.write(setup)
    init = os.path.join(tmpdir, "sample_s0.state")
    ref = _ref_binary()
    kind = "reference" if ref else "port"
    env = dict(os.environ, MAC_REF_RTOL="1e-8")
    if ref:
        subprocess.run([ref, "firstinit", setup, init], check=True, capture_output=True, env=env)
        cmds = [[ref, "bench", init, os.path.join(tmpdir, f"out{i}.state"), str(steps)] for i in range(procs)]
        t0 = time.perf_counter()
        ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env) for c in cmds]
        outs = [p.communicate() for p in ps]
        wall = time.perf_counter() - t0
        fcs = 0
        secs = 0.0
        for o, _e in outs:
            d = json.loads(o.strip().splitlines()[-1])
            fcs += d["fluid_cell_steps"]
            secs = max(secs, d["seconds"])
        return fcs / secs, kind, secs, fcs, wall
    oracle.run_oracle("firstinit", setup, init)
    t0 = time.perf_counter()
    st = oracle.run_oracle("bench", init, "", steps, 1e-8)
    secs = time.perf_counter() - t0
    return st["fluid_cell_steps"] / secs, kind, secs, st["fluid_cell_steps"], secs


def sample_desc(steps, procs):
    nx, ny, nz, h, r, w, depth, _ = CPU_SAMPLE
    return (f"{procs} concurrent single-thread replica(s) of a {nx}x{ny}x{nz} sub-box of the same jet "
            f"(h={h}, inflow r={r:g} at w={w}, pool depth {depth}), {steps} steps each after the first init, "
            f"solver stand-in FP64 Jacobi-CG at rel-resid 1e-8")


# ------------------------------------------------------------- ranks
def reduce_over_ranks(seconds: float, count: float, device) -> tuple:
    """Replicas only: every rank runs its own world; the job's time is the
    slowest rank's, its work the sum over ranks. Returns (max seconds, summed
    count); a no-op without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return seconds, count
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


# ------------------------------------------------------------- our arm
def roofline_models(ctx_stats, prof, np_count, n_exist, mg_bytes=8, cg_iterations=0, sweeps0=2):
    """Achieved GB/s per phase from algorithmic bytes (every array element a
    kernel must touch, read or written once) over the measured event times.
    A "launch" is one timed region of the phase (one particle move, one SpMV),
    except for the V-cycle phase: its regions hold one V-cycle per CG
    iteration, whose first kernel also applies the iteration's update
    x += alpha p, r -= alpha q, and one region per solve with the last update
    alone, so its launch is one CG iteration (a V-cycle and an update)."""
    unk = ctx_stats["unknowns"]
    # V-cycle: per cell of a level, 2 pre + 2 post sweeps of 17 B, residual 25 B,
    # restriction 8 B and prolongation 16 B at FP64 (117 B), the levels adding
    # up to 8/7 of the finest; FP32 storage halves it. The update: x, p, r, q
    # read, x, r written, 48 B at FP64.
    # With one sweep on the finest level its pre- and post-sweep count once each:
    # (2 x 17 + 49) B there, the coarser levels (1/7 of 117 B) unchanged.
    vc = ((4.0 * 17.0 + 49.0) * 8.0 / 7.0 if sweeps0 == 2 else 2.0 * 17.0 + 49.0 + 117.0 / 7.0) * (mg_bytes / 8.0)
    models = {
        # phase: (bytes per launch, description, launches or None for the region count)
        "move": (48.0 * np_count, "48 B per particle (read + write 3 FP64 positions)", None),
        "vcycle": ((vc + 48.0) * unk, f"{vc + 48.0:.1f} B per unknown per CG iteration: a V-cycle ({vc:.1f} B, "
                   f"levels 0.. at {mg_bytes} B per value) and the update it applies (48 B)", cg_iterations),
        "spmv": (34.0 * unk, "34 B per unknown (read z, p_old 16, face mask 2, write p, q 16)", None),
        "forces": (75.0 * n_exist, "75 B per existing cell (mean of stage 1: 51, stage 2: 99)", None),
        "gradient": (67.0 * n_exist, "67 B per existing cell (x 8, flags 3, p 8, u read+write 48)", None),
        "divergence": (42.0 * unk, "42 B per unknown (u 24, mask 2, rhs 8, x 8)", None),
    }
    out = {}
    for ph, (nbytes, desc, count) in models.items():
        ms, n = prof.get(ph, (0.0, 0))
        n = count if count else n
        if n:
            out[ph] = {"ms_total": ms, "launches": n, "avg_ms": ms / n,
                       "gbs": nbytes / (ms / n * 1e-3) / 1e9, "bytes_per_launch": nbytes, "model": desc}
    return out


POISSON_N = 128
POISSON_RTOL = 1e-10
WEIGHTS = os.path.join(ROOT, "mac_b200", "weights", "unet_pool64.npz")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def poisson_solves(dev, mg_sweeps=2, prefetch=False, reps=3):
    """Standalone pressure solve of the 128^3 pool + 12 spheres world (solid box,
    face speeds uniform in [-1, 1]) to a relative residual of 1e-10: device time
    of one projection and of its solve (system set-up + CG iterations), per
    solver form, with the pressure error against an FP64 MG-PCG solve to 1e-13.
    The learned forms use the weights trained by mac_b200.train_preconditioner
    (skipped when the weights file is absent); the network's forward pass on the
    solve's dense grid is timed alone for its tensor-pipe roofline."""
    import torch
    from mac_b200.gpu import Context
    from mac_b200.state import FLUID, pool_spheres_world
    from mac_b200.world import setup_passes
    net = None
    if os.path.exists(WEIGHTS):
        from mac_b200.unet import UNet
        net = UNet(dev)
        net.load(WEIGHTS)

    s = setup_passes(pool_spheres_world(POISSON_N))
    dom = s.exists.astype(bool) & (s.type == FLUID)
    res = {"workload": f"pool z<0.4n + 12 spheres r~U[6,20], {POISSON_N}^3, solid box, u~U[-1,1] (seeds 2, 3)",
           "rtol": POISSON_RTOL}
    p_ref = None
    forms = [("reference", "mgpcg64", 1e-13), ("plain", "mgpcg64", POISSON_RTOL), ("mixed", "mixed", POISSON_RTOL)]
    if net is not None:
        forms += [("learned", "learned", POISSON_RTOL), ("learned_mixed", "learned_mixed", POISSON_RTOL)]
    for name, solver, rtol in forms:
        with Context(s.params, max_bricks=8192, max_particles=1024, solver=solver, rtol=rtol, max_iters=1000,
                     device=dev) as ctx:
            ctx.set_multigrid(mg_sweeps, prefetch)
            if net is not None:
                ctx.set_preconditioner(net)
            stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
            times, solve = [], []
            for r in range(reps + 1):
                ctx.upload(s)
                ctx.sync()
                ctx.set_profiling(True)
                ctx.profile()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.project(0)
                e1.record(stream)
                e1.synchronize()
                prof = ctx.profile()
                if r:
                    times.append(e0.elapsed_time(e1))
                    solve.append(sum(prof[k][0] for k in ("setup", "spmv", "cg_vector", "vcycle")))
            st = ctx.stats()
            p = ctx.download().sorted().f64["p"]
        p = p[dom] if p.shape == dom.shape else None
        if name == "reference":
            p_ref = p
            res["unknowns"] = int(st["unknowns"])
            continue
        err = None
        if p is not None and p_ref is not None:
            err = float(np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref))
        res[name] = {"project_ms": round(float(np.median(times)), 3), "solve_ms": round(float(np.median(solve)), 3),
                     "iterations": int(st["iterations"]), "relres": st["relres"], "p_rel_err_vs_fp64": err}
        if solver.startswith("learned"):
            res[name].update({"learned_iterations": int(st["learned_iterations"]),
                              "fallback_to_mgpcg": bool(st["fallbacks"])})
    if net is not None:
        ms, flops = net.time_forward(1, POISSON_N, POISSON_N, POISSON_N, reps=5)
        pk = _peaks()
        peak = pk.get("bf16_tflops", 1590.0)
        tf = flops / (ms * 1e-3) / 1e12
        res["network_roofline"] = {"bound": "tensor", "grid": f"{POISSON_N}^3", "ms_per_forward": round(ms, 3),
                                   "flops_per_forward": flops, "achieved": round(tf, 1), "peak": peak,
                                   "unit": "TFLOP/s", "frac": round(tf / peak, 4),
                                   "peak_source": "measured" if "bf16_tflops" in pk else "fallback"}
        net.close()
    return res


def learned_evaluation(dev, mg_sweeps=2, prefetch=False, sizes=(128, 256), rtol=1e-8):
    """The learned preconditioner's evaluation: the pool + 12 spheres world at
    128^3 and 256^3 (radii scaled with the box) solved to a relative residual
    of 1e-8 with plain FP64 MG-PCG, the mixed form and the learned + mixed
    form: device ms of the projection (median of 2 after one warm-up), CG
    iterations, network iterations and whether MG-PCG took over."""
    import torch
    from mac_b200.gpu import Context
    from mac_b200.state import pool_spheres_world
    from mac_b200.unet import UNet
    from mac_b200.world import setup_passes
    if not os.path.exists(WEIGHTS):
        return None
    net = UNet(dev)
    net.load(WEIGHTS)
    out = {"rtol": rtol}
    for n in sizes:
        s = setup_passes(pool_spheres_world(n, r_range=(6.0 * n / 128, 20.0 * n / 128)))
        row = {}
        for solver in ("mgpcg64", "mixed", "learned_mixed"):
            with Context(s.params, max_bricks=int(s.nbricks * 1.2) + 64, max_particles=1024, solver=solver,
                         rtol=rtol, max_iters=1000, device=dev) as ctx:
                ctx.set_multigrid(mg_sweeps, prefetch)
                ctx.set_preconditioner(net)
                stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
                times = []
                for r in range(3):
                    ctx.upload(s)
                    ctx.sync()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ctx.project(0)
                    e1.record(stream)
                    e1.synchronize()
                    if r:
                        times.append(e0.elapsed_time(e1))
                st = ctx.stats()
            row[solver] = {"project_ms": round(float(np.median(times)), 3), "iterations": int(st["iterations"]),
                           "relres": st["relres"]}
            if solver.startswith("learned"):
                row[solver].update({"learned_iterations": int(st["learned_iterations"]),
                                    "fallback_to_mgpcg": bool(st["fallbacks"])})
        row["unknowns"] = int(st["unknowns"])
        row["speedup_vs_mgpcg64"] = {f: round(row["mgpcg64"]["project_ms"] / row[f]["project_ms"], 3)
                                     for f in ("mixed", "learned_mixed")}
        out[f"pool{n}"] = row
        log(f"[learned eval] {n}^3: {row}")
    net.close()
    return out


SOLVER_NAMES = {"mgpcg64": "plain FP64 MG-PCG", "mixed": "FP32 MG in FP64 PCG", "cg64": "FP64 Jacobi-PCG",
                "learned": "learned preconditioner in FP64 flexible CG (FP64 MG-PCG fall-back)",
                "learned_mixed": "learned preconditioner in FP64 flexible CG (FP32 MG fall-back)"}


def solver_forms(args, dev, params, host, wl, steps=5, warmup=2):
    """The same spun-up jet state (host, pinned) stepped with each solver form
    in turn: device ms per step (CUDA events on the library's stream), fluid
    cell-steps/s, CG iterations per solve, and the step-time ratios against
    the plain FP64 MG-PCG form (the denominator of the learned + mixed
    target)."""
    import torch
    from mac_b200.gpu import Context
    forms = ["mgpcg64", "mixed"]
    net = None
    if os.path.exists(WEIGHTS):
        from mac_b200.unet import UNet
        net = UNet(dev)
        net.load(WEIGHTS)
        forms.append("learned_mixed")
    out = {"steps": steps, "warmup": warmup, "rtol": 1e-8, "mg_sweeps0": args.mg_sweeps}
    for form in forms:
        with Context(params, max_bricks=wl[8], max_particles=wl[9], solver=form, rtol=1e-8, max_iters=1000,
                     device=dev, div_check=True) as ctx:
            ctx.set_multigrid(args.mg_sweeps, args.prefetch)
            if form.startswith("learned"):
                ctx.set_preconditioner(net)
            ctx.upload(None, host)
            stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
            for _ in range(warmup):
                ctx.step()
            ctx.sync()
            it0 = ctx.stats()["total_iterations"]
            fb0 = ctx.stats()["fallbacks"]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            fluid = 0
            learned_its = []
            e0.record(stream)
            for _ in range(steps):
                ctx.step()
                st = ctx.stats()
                fluid += st["fluid_cells"]
                learned_its.append(st["learned_iterations"])
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            st = ctx.stats()
            r = {"solver": SOLVER_NAMES[form], "ms_per_step": round(ms / steps, 3),
                 "value": fluid / (ms * 1e-3), "cg_iters_per_solve": (st["total_iterations"] - it0) / (2 * steps),
                 "relres_last": st["relres"], "max_div_last": st["max_div"]}
            if form.startswith("learned"):
                r["fallback_solves"] = st["fallbacks"] - fb0
                r["learned_iters_last"] = learned_its[-1] if learned_its else 0
            out[form] = r
        log(f"[forms] {form}: {out[form]}")
    if net is not None:
        net.close()
    base = out["mgpcg64"]["ms_per_step"]
    out["speedup_vs_mgpcg64"] = {f: round(base / out[f]["ms_per_step"], 3) for f in forms}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from mac_b200.gpu import Context, HostState
    from mac_b200.world import first_init

    dev = local_rank
    torch.cuda.set_device(dev)
    wl = WORKLOADS[args.workload]
    t0 = time.perf_counter()
    s = make_world(args.workload)
    log(f"[rank {rank}] world built in {time.perf_counter() - t0:.1f}s: {s.nbricks} bricks, {s.nparticles} particles")
    ctx = Context(s.params, max_bricks=wl[8], max_particles=wl[9], solver=args.solver, rtol=1e-8, max_iters=1000,
                  device=dev, div_check=True, warm_start=args.warm_start)
    ctx.set_multigrid(args.mg_sweeps, args.prefetch)
    ctx.set_dependent_launch(not args.no_dependent_launch)
    ctx.set_concurrent_binning(args.concurrent_binning)
    if args.solver.startswith("learned"):
        from mac_b200.unet import UNet
        net_main = UNet(dev)
        net_main.load(WEIGHTS)
        ctx.set_preconditioner(net_main)
    t0 = time.perf_counter()
    first_init(ctx, s)
    ctx.sync()
    log(f"[rank {rank}] first init {time.perf_counter() - t0:.1f}s")
    params = s.params
    del s
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)

    for _ in range(args.warmup):
        ctx.step()
    ctx.sync()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = ctx.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    fluid_steps = 0
    iters = []
    it0 = ctx.stats()["total_iterations"]
    e0.record(stream)
    for _ in range(args.steps):
        ctx.step()
        st = ctx.stats()
        fluid_steps += st["fluid_cells"]
        iters.append(st["iterations"])
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches() - l0
    sec, total_fluid_steps = reduce_over_ranks(ms / 1e3, fluid_steps, f"cuda:{dev}")
    value = total_fluid_steps / sec

    # Per-phase times for the rooflines, from further steps of the same run
    # with an event pair around each phase. The events sit between kernels the
    # CG loop otherwise chains with programmatic dependent launches, so these
    # steps run slightly slower than the timed ones: the phase figures are
    # conservative.
    prof_steps = max(1, min(args.steps, 5))
    ctx.set_profiling(True)
    ctx.profile()  # reset
    it0 = ctx.stats()["total_iterations"]
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(prof_steps):
        ctx.step()
    p1.record(stream)
    p1.synchronize()
    prof_ms_per_step = p0.elapsed_time(p1) / prof_steps
    prof = ctx.profile()
    ctx.set_profiling(False)
    st = ctx.stats()
    cg_iterations = st["total_iterations"] - it0

    # e2e through the C-ABI with pinned host buffers: upload, step, download per step
    nb, npart = ctx.sizes()
    # RK2-TVD's stage buffers (speed 1, acceleration) are written before they
    # are read in every step: left out of both transfers
    host = HostState(int(nb * 1.1) + 64, int(npart * 1.02) + 4096, pinned=True, stage_buffers=False)
    ctx.download(host, to_state=False)
    e2e_steps = max(1, min(args.steps, 3))
    bi = bo = 0
    f2 = 0
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(e2e_steps):
        bi += host.nbytes()
        ctx.upload(None, host)
        ctx.step()
        f2 += ctx.stats()["fluid_cells"]
        # the C-ABI read into the pinned buffers, as a C or C++ caller makes
        # it (no conversion into a key-sorted Python State)
        ctx.download(host, to_state=False)
        bo += host.nbytes()
    a1.record(stream)
    a1.synchronize()
    e2e_sec, f2 = reduce_over_ranks(a0.elapsed_time(a1) / 1e3, f2, f"cuda:{dev}")
    e2e = {"value": f2 / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": bi // e2e_steps,
           "d2h_bytes_per_step": bo // e2e_steps, "steps": e2e_steps,
           "fields": "keys, existence, speed 0, pressure, flags, material, layer, particles each way (speed "
                     "buffer 1 and the acceleration, RK2-TVD's stage buffers, left out)"}

    n_exist = int(st["live_bricks"] * 512)  # upper bound of existing cells (slots of live bricks)
    rl = roofline_models(st, prof, st["particles"], n_exist, 4 if args.solver == "mixed" else 8, cg_iterations,
                         args.mg_sweeps)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max(rl, key=lambda k: rl[k]["ms_total"]) if rl else None
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get(dom)
    except (OSError, ValueError):
        pass
    roofline = None
    if dom:
        r = rl[dom]
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(r["gbs"], 1), "peak": peak, "unit": "GB/s",
                    "frac": round(r["gbs"] / peak, 4), "peak_source": peak_src,
                    "traffic": traffic, "bytes_per_launch": r["bytes_per_launch"], "model": r["model"]}
    phases = {k: {"ms": round(v[0], 3), "n": v[1]} for k, v in prof.items() if v[1]}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded spun-up jet state)",
        "config": {"workload": f"jet {wl[0]}x{wl[1]}x{wl[2]} h={wl[3]} inflow r={wl[4]:g} w={wl[5]}, pool depth "
                               f"{wl[6]}, 8 particles/fluid cell, LayerMax 4, CFL 0.5",
                   "solver": SOLVER_NAMES[args.solver], "mg_sweeps0": args.mg_sweeps,
                   "mg_prefetch": args.prefetch,
                   "dependent_launch": not args.no_dependent_launch,
                   "concurrent_binning": args.concurrent_binning,
                   "rtol": 1e-8, "initial_guess": "last pressure" if args.warm_start else "zero",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (state > 3 GB)",
                   "fluid_cells_last": st["fluid_cells"], "particles": st["particles"],
                   "live_bricks": st["live_bricks"], "cg_iters_per_solve_last": st["iterations"],
                   "cg_iters_mean": float(np.mean(iters)) if iters else None},
        "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "roofline": roofline,
        "phases_ms": phases, "phase_steps": prof_steps, "phase_ms_per_step": round(prof_ms_per_step, 3),
        "phase_rooflines": {k: {"gbs": round(v["gbs"], 1), "avg_ms": round(v["avg_ms"], 4)}
                                                 for k, v in rl.items()},
    }
    ctx.close()
    if rank == 0 and not args.no_forms:
        out["solver_forms"] = solver_forms(args, dev, params, host, wl)
    del host
    if rank == 0 and not args.no_poisson:
        out["poisson"] = poisson_solves(dev, args.mg_sweeps, args.prefetch)
        out["learned_evaluation"] = learned_evaluation(dev, args.mg_sweeps, args.prefetch)
    return out


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="jet256")
    ap.add_argument("--solver", choices=sorted(SOLVER_NAMES), default="mixed",
                    help="projection solver: mixed = FP64 CG with the FP32 multigrid (default), "
                         "mgpcg64 = plain FP64 MG-PCG, cg64 = FP64 Jacobi-PCG, learned[_mixed] = the network "
                         "in flexible CG")
    ap.add_argument("--mg-sweeps", type=int, choices=[1, 2], default=2,
                    help="Jacobi sweeps before and after the coarse correction on the finest multigrid level")
    ap.add_argument("--no-forms", action="store_true", help="skip stepping the jet with every solver form")
    ap.add_argument("--prefetch", action="store_true",
                    help="run the V-cycle's first kernel as resident blocks prefetching bricks with bulk copies")
    ap.add_argument("--no-dependent-launch", action="store_true",
                    help="launch the CG loop's kernels in plain stream order")
    ap.add_argument("--concurrent-binning", action="store_true",
                    help="bin the particles on a second stream during RK2-TVD instead of inside the move")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-poisson", action="store_true", help="skip the standalone 128^3 pressure-solve timing")
    ap.add_argument("--warm-start", action="store_true",
                    help="start each pressure solve from the previous pressure (the reference starts from zero)")
    ap.add_argument("--cpu-steps", type=int, default=2)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        procs = max(1, min(os.cpu_count() or 1, 8))
        with tempfile.TemporaryDirectory() as td:
            # warm-up steps are run too (each replica runs warmup + steps), the
            # timed value covers all of them
            v, kind, secs, fcs, wall = cpu_reference_run(args.steps + args.warmup, procs, td)
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": secs * 1e3 / (args.steps + args.warmup),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded jet sub-box)", "impl": "reference",
                "config": {"workload": "jet sub-box, see cpu_baseline.sample", "rtol": 1e-8},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": kind,
                                 "sample": sample_desc(args.steps + args.warmup, procs)},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            v, kind, secs, fcs, wall = cpu_reference_run(args.cpu_steps, 1, td)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": kind,
                               "sample": sample_desc(args.cpu_steps, 1), "seconds": round(secs, 2)}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())

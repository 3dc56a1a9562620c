"""Standalone pressure solves on the pool + 12 spheres world.

    python -m mac_b200.solve_pool [--n 128] [--solver mixed] [--rtol 1e-10] [--solves 3]

Builds the n^3 world (solid box, fluid below 0.4 n plus 12 spheres of radius
3n/64..10n/64 cells, face speeds uniform in [-1, 1], seeds 2 and 3), uploads
it and runs the projection `--solves` times from the same state, printing the
device time (CUDA events on the library's stream), CG iterations and final
relative residual of each solve as one JSON line. `--weights` attaches a
network for the learned solvers.
"""
import argparse
import json

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--solver", default="mixed", choices=["mgpcg64", "mixed", "cg64", "learned", "learned_mixed"])
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()

    import torch

    from .gpu import Context
    from .state import pool_spheres_world
    from .world import setup_passes

    n = a.n
    s = setup_passes(pool_spheres_world(n, r_range=(6.0 * n / 128, 20.0 * n / 128)))
    net = None
    if a.weights:
        from .unet import UNet
        net = UNet(a.device)
        net.load(a.weights)
    out = {"n": n, "solver": a.solver, "rtol": a.rtol, "solves": []}
    with Context(s.params, max_bricks=int(s.nbricks * 1.2) + 64, max_particles=1024, solver=a.solver, rtol=a.rtol,
                 max_iters=2000, device=a.device) as ctx:
        if net is not None:
            ctx.set_preconditioner(net)
        stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=a.device)
        for _ in range(a.solves):
            ctx.upload(s)
            ctx.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.project(0)
            e1.record(stream)
            e1.synchronize()
            st = ctx.stats()
            out["unknowns"] = int(st["unknowns"])
            out["solves"].append({"ms": round(e0.elapsed_time(e1), 3), "iterations": int(st["iterations"]),
                                  "relres": st["relres"]})
    if net is not None:
        net.close()
    out["median_ms"] = float(np.median([x["ms"] for x in out["solves"]]))
    print(json.dumps(out))


if __name__ == "__main__":
    main()

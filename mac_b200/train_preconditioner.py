"""Trains the learned preconditioner on the device and saves its weights.

    python -m mac_b200.train_preconditioner [--masks 2000] [--size 64] [--steps 20000]
        [--batch 16] [--lr 1e-3] [--loss energy] [--out mac_b200/weights/unet_pool64.npz]

Training pairs (residual, exact error) come from plain FP64 CG iterates on
random fluid masks (a pool z < 0.4 size plus 12 spheres of radius 3..10 cells
at size 64, solid box), generated on the device by mac_unet_make_dataset; the
network is trained with Adam by the device's own forward and backward kernels
(mac_unet_train). The saved file holds the FP32 parameters, the output scale
and the loss curve; mac_b200.unet.UNet.load reads it back.
"""
import argparse
import json
import os
import time

import numpy as np

from .unet import UNet

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "weights", "unet_pool64.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--masks", type=int, default=2000)
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--snapshots", type=int, default=8)
    ap.add_argument("--cg-iters", type=int, default=1200)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--loss", choices=["mse", "energy"], default="energy")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    with UNet(a.device, seed=a.seed) as net:
        net.set_loss(a.loss)
        t0 = time.perf_counter()
        info = net.make_dataset(a.masks, a.size, a.snapshots, a.cg_iters, seed=1000 + a.seed)
        t_data = time.perf_counter() - t0
        print(f"training set: {info['samples']} pairs in {t_data:.1f}s, worst CG relres {info['worst_relres']:.1e}, "
              f"output scale {info['tscale']:.4g}", flush=True)
        losses = []
        t0 = time.perf_counter()
        chunk = 1000
        for k in range(0, a.steps, chunk):
            n = min(chunk, a.steps - k)
            losses.append(net.train(n, a.batch, a.lr, seed=a.seed * 1000003 + k))
            print(f"step {k + n}: loss {losses[-1][-100:].mean():.5f} ({time.perf_counter() - t0:.0f}s)", flush=True)
        t_train = time.perf_counter() - t0
        losses = np.concatenate(losses)
        p, tscale = net.params()
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        meta = {"masks": a.masks, "size": a.size, "snapshots": a.snapshots, "cg_iters": a.cg_iters, "steps": a.steps,
                "batch": a.batch, "lr": a.lr, "loss": a.loss, "seed": a.seed, "train_seconds": t_train,
                "ms_per_step": 1e3 * t_train / a.steps, "dataset_seconds": t_data}
        np.savez_compressed(a.out, params=p, tscale=np.float32(tscale),
                            loss_every_100=losses.reshape(-1, 100).mean(axis=1) if a.steps % 100 == 0 else losses,
                            meta=json.dumps(meta))
        print(json.dumps(meta))


if __name__ == "__main__":
    main()

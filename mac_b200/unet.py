"""Host side of the learned preconditioner: a thin ctypes wrapper over the
mac_unet_* entry points of libmac_gpu.so (include/mac_gpu.h)."""
import ctypes

import numpy as np

from .gpu import MacError, load

_P = ctypes.POINTER


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class UNet:
    """The 3-level U-Net (16/32/64 channels) on one device."""

    def __init__(self, device: int = 0, seed: int | None = None):
        self.lib = load()
        h = ctypes.c_void_p()
        self._check(self.lib.mac_unet_create(device, ctypes.byref(h)), "mac_unet_create")
        self.h = h
        n = ctypes.c_int64()
        self._check(self.lib.mac_unet_nparams(self.h, ctypes.byref(n)), "mac_unet_nparams")
        self.nparams = int(n.value)
        if seed is not None:
            self._check(self.lib.mac_unet_init(self.h, seed), "mac_unet_init")

    def _check(self, rc, what):
        if rc != 0:
            raise MacError(rc, what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mac_unet_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def params(self):
        p = np.zeros(self.nparams, np.float32)
        t = ctypes.c_float()
        self._check(self.lib.mac_unet_get_params(self.h, p.ctypes.data_as(_P(ctypes.c_float)), ctypes.byref(t)),
                    "mac_unet_get_params")
        return p, float(t.value)

    def set_params(self, p, tscale):
        p = _f32(p)
        assert p.size == self.nparams
        self._check(self.lib.mac_unet_set_params(self.h, p.ctypes.data_as(_P(ctypes.c_float)), float(tscale)),
                    "mac_unet_set_params")

    def set_conv(self, staged=True):
        """Forward 3x3x3 convolutions through the staged-tile kernel (True) or the per-tap gather."""
        self._check(self.lib.mac_unet_set_conv(self.h, 1 if staged else 0), "mac_unet_set_conv")

    def forward(self, r, mask):
        r = _f32(r)
        m = np.ascontiguousarray(mask, dtype=np.int8)
        n, d, h, w = r.shape
        out = np.zeros_like(r)
        self._check(self.lib.mac_unet_forward(self.h, n, d, h, w, r.ctypes.data_as(_P(ctypes.c_float)),
                                              m.ctypes.data_as(_P(ctypes.c_int8)),
                                              out.ctypes.data_as(_P(ctypes.c_float))), "mac_unet_forward")
        return out

    def loss_grad(self, r, mask, e):
        r, e = _f32(r), _f32(e)
        m = np.ascontiguousarray(mask, dtype=np.int8)
        n, d, h, w = r.shape
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_double()
        self._check(self.lib.mac_unet_loss_grad(self.h, n, d, h, w, r.ctypes.data_as(_P(ctypes.c_float)),
                                                m.ctypes.data_as(_P(ctypes.c_int8)),
                                                e.ctypes.data_as(_P(ctypes.c_float)), ctypes.byref(loss),
                                                g.ctypes.data_as(_P(ctypes.c_float))), "mac_unet_loss_grad")
        return float(loss.value), g

    def adam_step(self, grad, lr):
        g = _f32(grad)
        self._check(self.lib.mac_unet_adam_step(self.h, g.ctypes.data_as(_P(ctypes.c_float)), float(lr)),
                    "mac_unet_adam_step")

    def make_dataset(self, nmasks, size=64, nsnap=8, niter=1000, seed=1000, masks=None):
        """nmasks masks of size^3: the given ones first (int8 [k][size][size][size]:
        1 fluid, 0 air, -1 solid), random pools with spheres for the rest."""
        st = (ctypes.c_double * 2)()
        if masks is None:
            self._check(self.lib.mac_unet_make_dataset(self.h, nmasks, size, nsnap, niter, seed, st),
                        "mac_unet_make_dataset")
        else:
            m = np.ascontiguousarray(masks, dtype=np.int8).reshape(-1, size, size, size)
            self._check(self.lib.mac_unet_make_dataset_ext(self.h, nmasks, size, nsnap, niter, seed,
                                                           m.ctypes.data_as(_P(ctypes.c_int8)), len(m), st),
                        "mac_unet_make_dataset_ext")
        self.size = size
        return {"worst_relres": st[0], "tscale": st[1], "samples": nmasks * nsnap}

    def sample(self, index):
        s = self.size
        r = np.zeros((s, s, s), np.float32)
        e = np.zeros((s, s, s), np.float32)
        m = np.zeros((s, s, s), np.int8)
        self._check(self.lib.mac_unet_get_sample(self.h, index, r.ctypes.data_as(_P(ctypes.c_float)),
                                                 e.ctypes.data_as(_P(ctypes.c_float)),
                                                 m.ctypes.data_as(_P(ctypes.c_int8))), "mac_unet_get_sample")
        return r, e, m

    def train(self, steps, batch=16, lr=1e-3, seed=7):
        losses = np.zeros(steps, np.float32)
        self._check(self.lib.mac_unet_train(self.h, steps, batch, float(lr), seed,
                                            losses.ctypes.data_as(_P(ctypes.c_float))), "mac_unet_train")
        return losses

    def set_loss(self, kind):
        """Training loss: "mse" (mean squared error) or "energy" (energy norm of the error)."""
        self._check(self.lib.mac_unet_set_loss(self.h, {"mse": 0, "energy": 1}[kind]), "mac_unet_set_loss")

    def save(self, path):
        p, t = self.params()
        np.savez_compressed(path, params=p, tscale=np.float32(t))

    def load(self, path):
        """Weights saved by save() or by mac_b200.train_preconditioner."""
        d = np.load(path)
        self.set_params(d["params"], float(d["tscale"]))

    def time_forward(self, n, d, h, w, reps=5):
        """(ms per forward pass, algorithmic FLOPs per pass) on an n x d x h x w grid."""
        ms, fl = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mac_unet_time_forward(self.h, n, d, h, w, reps, ctypes.byref(ms), ctypes.byref(fl)),
                    "mac_unet_time_forward")
        return ms.value, fl.value

    def launches(self):
        n = ctypes.c_int64()
        self._check(self.lib.mac_unet_launch_count(self.h, ctypes.byref(n)), "mac_unet_launch_count")
        return int(n.value)

"""CPU oracle of the learned preconditioner's network (test infrastructure only:
imported by tests/ and by nothing in the product).

The same 3-level U-Net as mac_b200/csrc/mac_unet.cu, written with numpy:
forward, loss and a hand-derived backward. With ``bf16=True`` it rounds to
BF16 at the points where the device stores BF16 (network input, every
activation, every activation gradient, the pooled and unpooled tensors), with
FP64 accumulation in between, so the device's results (FP32 accumulation) are
expected within a few BF16 ulps; with ``bf16=False`` it is plain FP64, which
the tests pin against finite differences.

The network has no counterpart in the reference; its definition is this
project's (layer table below, identical to the device's kLayers).
"""
import numpy as np

# cin, cout, taps, relu, real_cin, real_cout
LAYERS = [
    (16, 16, 27, 1, 2, 16), (16, 16, 27, 1, 16, 16), (16, 32, 27, 1, 16, 32), (32, 32, 27, 1, 32, 32),
    (32, 64, 27, 1, 32, 64), (64, 64, 27, 1, 64, 64), (64, 32, 1, 0, 64, 32), (64, 32, 27, 1, 64, 32),
    (32, 32, 27, 1, 32, 32), (32, 16, 1, 0, 32, 16), (32, 16, 27, 1, 32, 16), (16, 16, 27, 1, 16, 16),
    (16, 16, 1, 0, 16, 1),
]


def offsets():
    """(weight offset, bias offset) per layer and the total, as the device lays them out."""
    o, out = 0, []
    for cin, cout, taps, *_ in LAYERS:
        w = o
        o += taps * cout * cin
        b = o
        o += cout
        o = (o + 7) // 8 * 8
        out.append((w, b))
    return out, o


def unpack(params):
    offs, _ = offsets()
    ws, bs = [], []
    for (wo, bo), (cin, cout, taps, *_r) in zip(offs, LAYERS):
        ws.append(np.asarray(params[wo:wo + taps * cout * cin], np.float64).reshape(taps, cout, cin))
        bs.append(np.asarray(params[bo:bo + cout], np.float64))
    return ws, bs


def pack_grads(dws, dbs):
    offs, n = offsets()
    g = np.zeros(n)
    for (wo, bo), dw, db in zip(offs, dws, dbs):
        g[wo:wo + dw.size] = dw.ravel()
        g[bo:bo + db.size] = db
    return g


def to_bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _taps(taps):
    if taps == 1:
        return [(0, 0, 0)]
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def _shifted(xp, dz, dy, dx, d, h, w):
    return xp[:, 1 + dz:1 + dz + d, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w, :]


def conv(x, W, taps):
    """y[v] = sum_t x[v + off_t] @ W_t^T (zero outside the grid); x [n, d, h, w, cin]."""
    if taps == 1:
        return x @ W[0].T
    n, d, h, w, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    y = 0.0
    for t, (dz, dy, dx) in enumerate(_taps(taps)):
        y = y + _shifted(xp, dz, dy, dx, d, h, w) @ W[t].T
    return y


def conv_input_grad(g, W, taps):
    """dx[q] = sum_t g[q - off_t] @ W_t."""
    if taps == 1:
        return g @ W[0]
    n, d, h, w, _ = g.shape
    gp = np.pad(g, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = 0.0
    for t, (dz, dy, dx) in enumerate(_taps(taps)):
        out = out + _shifted(gp, -dz, -dy, -dx, d, h, w) @ W[t]
    return out


def conv_weight_grad(x, g, taps):
    """dW_t[co][ci] = sum_v g[v][co] x[v + off_t][ci]."""
    cout, cin = g.shape[-1], x.shape[-1]
    g2 = g.reshape(-1, cout)
    if taps == 1:
        return (g2.T @ x.reshape(-1, cin))[None]
    n, d, h, w, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    return np.stack([g2.T @ _shifted(xp, dz, dy, dx, d, h, w).reshape(-1, cin) for dz, dy, dx in _taps(taps)])


def pool(x, scale):
    n, d, h, w, c = x.shape
    return x.reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4, 6)) * scale


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


class Net:
    def __init__(self, params, tscale, bf16=True):
        self.W, self.b = unpack(params)
        self.tscale = float(tscale)
        self.q = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
        self.f32 = (lambda a: np.asarray(a, np.float32).astype(np.float64)) if bf16 else self.q
        if bf16:
            self.W = [to_bf16(w) for w in self.W]

    def scale(self, r, m):
        """Per-sample rms of r over fluid cells (1 where it vanishes)."""
        s = []
        for k in range(r.shape[0]):
            f = m[k] == 1
            c = f.sum()
            v = np.sqrt(np.sum(r[k][f].astype(np.float64) ** 2) / c) if c else 0.0
            s.append(v if v > 0 else 1.0)
        return np.array(s)

    def forward(self, r, m):
        """r, m: [n, d, h, w]; returns (output [n, d, h, w], cache)."""
        q, W, b = self.q, self.W, self.b
        s = self.scale(r, m)
        n = r.shape[0]
        x = np.zeros(r.shape + (16,))
        inv = (1.0 / s).astype(np.float32)
        for k in range(n):
            x[k, ..., 0] = np.where(m[k] == 1, r[k].astype(np.float32) * inv[k], 0.0)
        x[..., 1] = m
        x = q(x)

        def layer(i, xin):
            y = conv(xin, W[i], LAYERS[i][2]) + b[i]
            if LAYERS[i][3]:
                y = np.maximum(y, 0.0)
            return y

        c = {"in0": x, "s": s}
        c["a1"] = q(layer(0, x))
        c["s1"] = q(layer(1, c["a1"]))
        c["p1"] = q(pool(c["s1"], 0.125))
        c["a2"] = q(layer(2, c["p1"]))
        c["s2"] = q(layer(3, c["a2"]))
        c["p2"] = q(pool(c["s2"], 0.125))
        c["a3"] = q(layer(4, c["p2"]))
        c["b3"] = q(layer(5, c["a3"]))
        c["u2"] = q(layer(6, c["b3"]))
        c["x7"] = np.concatenate([c["s2"], up(c["u2"])], axis=-1)
        c["c2"] = q(layer(7, c["x7"]))
        c["d2"] = q(layer(8, c["c2"]))
        c["u1"] = q(layer(9, c["d2"]))
        c["x10"] = np.concatenate([c["s1"], up(c["u1"])], axis=-1)
        c["c1"] = q(layer(10, c["x10"]))
        c["d1"] = q(layer(11, c["c1"]))
        out = layer(12, c["d1"])[..., 0]
        return out, c

    def correction(self, r, m):
        out, c = self.forward(r, m)
        return np.where(m == 1, out * (c["s"][:, None, None, None] * self.tscale), 0.0)

    def loss_grad(self, r, m, e, kind="mse"):
        """Loss and the flattened parameter gradient (device layout). kind
        "mse": mean squared error of the output against e / (rms(r) tscale);
        "energy": sum d (M d) / count with d that difference and M the
        unit-spacing operator of the mask."""
        q, W = self.q, self.W
        out, c = self.forward(r, m)
        s = c["s"]
        fluid = m == 1
        count = fluid.sum()
        t = e / (s[:, None, None, None] * self.tscale)
        g = np.zeros(out.shape + (16,))
        if kind == "energy":
            d = np.where(fluid, self.f32(out - t), 0.0)
            Md = np.stack([dense_operator_apply(d[k], m[k]) for k in range(d.shape[0])])
            loss = float(np.sum(d * Md) / count)
            g[..., 0] = q(np.where(fluid, 2.0 * Md / count, 0.0))
        else:
            diff = np.where(fluid, out - t, 0.0)
            loss = float(np.sum(diff ** 2) / count)
            g[..., 0] = q(2.0 * diff / count)
        dW = [None] * 13
        dB = [None] * 13

        def back(i, xin, y, gy):
            """Weight/bias gradients of layer i; returns the (unrounded) input gradient."""
            gg = gy * (y > 0) if LAYERS[i][3] else gy
            dW[i] = conv_weight_grad(xin, gg, LAYERS[i][2])
            dB[i] = gg.reshape(-1, gg.shape[-1]).sum(axis=0)
            return conv_input_grad(gg, W[i], LAYERS[i][2])

        g_d1 = q(back(12, c["d1"], None, g))
        g_c1 = q(back(11, c["c1"], c["d1"], g_d1))
        gx10 = q(back(10, c["x10"], c["c1"], g_c1))
        g_s1, g_up1 = gx10[..., :16], gx10[..., 16:]
        g_u1 = q(pool(g_up1, 1.0))
        g_d2 = q(back(9, c["d2"], None, g_u1))
        g_c2 = q(back(8, c["c2"], c["d2"], g_d2))
        gx7 = q(back(7, c["x7"], c["c2"], g_c2))
        g_s2, g_up2 = gx7[..., :32], gx7[..., 32:]
        g_u2 = q(pool(g_up2, 1.0))
        g_b3 = q(back(6, c["b3"], None, g_u2))
        g_a3 = q(back(5, c["a3"], c["b3"], g_b3))
        g_p2 = q(back(4, c["p2"], c["a3"], g_a3))
        g_s2 = q(g_s2 + 0.125 * up(g_p2))
        g_a2 = q(back(3, c["a2"], c["s2"], g_s2))
        g_p1 = q(back(2, c["p1"], c["a2"], g_a2))
        g_s1 = q(g_s1 + 0.125 * up(g_p1))
        g_a1 = q(back(1, c["a1"], c["s1"], g_s1))
        back(0, c["in0"], c["a1"], g_a1)
        return loss, pack_grads(dW, dB)


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """Reference Adam update (FP32, as the device's k_adam)."""
    p, g, m, v = (np.asarray(a, np.float32) for a in (p, g, m, v))
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    bc1 = np.float32(1 - b1 ** t)
    bc2 = np.float32(1 - b2 ** t)
    p = p - np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return p, m, v


def dense_operator_apply(p, m):
    """(M p)[c] for fluid c: sum over the in-grid, non-solid neighbours n of
    p[c] - [n fluid] p[n] (air: Dirichlet 0; outside the grid or solid: Neumann);
    unit spacing. p, m: [d, h, w]."""
    f = m == 1
    out = np.zeros_like(p, dtype=np.float64)
    pf = np.where(f, p, 0.0)
    for ax in range(3):
        for sgn in (-1, 1):
            nb_p = np.roll(pf, -sgn, axis=ax)
            nb_m = np.roll(m, -sgn, axis=ax)
            valid = np.ones_like(f)
            idx = [slice(None)] * 3
            idx[ax] = -1 if sgn == 1 else 0
            valid[tuple(idx)] = False
            valid &= nb_m != -1
            out += np.where(valid & f, pf - nb_p, 0.0)
    return out

"""The learned preconditioner's network: the numpy oracle pinned by finite
differences (CPU), then the device's forward, loss, gradients, Adam step,
training-pair generator and training against it (GPU, through the C-ABI).

Device tolerances: the device stores activations and activation gradients in
BF16 exactly where the oracle rounds them, but accumulates in FP32 (the oracle
in FP64), so a rounding can land on the other side of a BF16 step: relative L2
error <= 2e-2 for the network output and the loss, <= 5e-2 for each layer's
weight gradient (1e-1 under the energy loss), 1e-5 for the FP32 Adam update.
"""
import numpy as np
import pytest

import unet_oracle as U


def _random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    offs, n = U.offsets()
    p = np.zeros(n)
    for (wo, bo), (cin, cout, taps, relu, rcin, rcout) in zip(offs, U.LAYERS):
        w = np.zeros((taps, cout, cin))
        b = np.sqrt((6.0 if relu else 3.0) / (taps * rcin)) * scale
        w[:, :rcout, :rcin] = rng.uniform(-b, b, size=(taps, rcout, rcin))
        p[wo:wo + w.size] = w.ravel()
        p[bo:bo + rcout] = rng.uniform(-0.05, 0.05, size=rcout)
    return p


def _problem(n, s, seed):
    rng = np.random.default_rng(seed)
    z = np.arange(s)[:, None, None]
    m = np.where(z < s // 2, 1, 0) * np.ones((n, s, s, s), np.int8)
    m[:, :, : s // 4, : s // 4] = -1  # a solid block
    m[:, s // 2:, s // 2:, s // 2:] = 1  # a fluid block above the pool
    r = np.where(m == 1, rng.standard_normal((n, s, s, s)), 0.0).astype(np.float32)
    e = np.where(m == 1, rng.standard_normal((n, s, s, s)), 0.0).astype(np.float32)
    return r, m.astype(np.int8), e


def _layer_slices():
    offs, _ = U.offsets()
    return [(wo, wo + taps * cout * cin) for (wo, _b), (cin, cout, taps, *_r) in zip(offs, U.LAYERS)]


# ----------------------------------------------------------------- CPU: oracle
def test_oracle_gradient_matches_finite_differences():
    p = _random_params(3)
    r, m, e = _problem(1, 8, 4)
    net = U.Net(p, 0.7, bf16=False)
    loss, g = net.loss_grad(r, m, e)
    rng = np.random.default_rng(5)
    offs, _ = U.offsets()
    checked = 0
    for (wo, bo), (cin, cout, taps, relu, rcin, rcout) in zip(offs, U.LAYERS):
        idx = [wo + (int(rng.integers(taps)) * cout + int(rng.integers(rcout))) * cin + int(rng.integers(rcin))
               for _ in range(2)] + [bo + int(rng.integers(rcout))]
        for i in idx:
            h = 1e-6 * max(1.0, abs(p[i]))
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd = (U.Net(pp, 0.7, bf16=False).loss_grad(r, m, e)[0] - U.Net(pm, 0.7, bf16=False).loss_grad(r, m, e)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd), abs(g[i])), (i, fd, g[i])
            checked += 1
    assert checked == 3 * len(U.LAYERS)


def test_oracle_energy_gradient_matches_finite_differences():
    p = _random_params(7)
    r, m, e = _problem(1, 8, 8)
    _, g = U.Net(p, 0.7, bf16=False).loss_grad(r, m, e, kind="energy")
    rng = np.random.default_rng(9)
    offs, _ = U.offsets()
    for (wo, bo), (cin, cout, taps, relu, rcin, rcout) in list(zip(offs, U.LAYERS))[::3]:
        i = wo + (int(rng.integers(taps)) * cout + int(rng.integers(rcout))) * cin + int(rng.integers(rcin))
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = U.Net(pp, 0.7, bf16=False).loss_grad(r, m, e, kind="energy")[0]
        lm = U.Net(pm, 0.7, bf16=False).loss_grad(r, m, e, kind="energy")[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd), abs(g[i])), (i, fd, g[i])


def test_oracle_padding_gradients_vanish():
    p = _random_params(3)
    r, m, e = _problem(1, 8, 4)
    _, g = U.Net(p, 0.7, bf16=False).loss_grad(r, m, e)
    offs, _ = U.offsets()
    (w0, _), (w12, b12) = offs[0], offs[12]
    w = g[w0:w0 + 27 * 16 * 16].reshape(27, 16, 16)
    assert np.all(w[:, :, 2:] == 0)  # padded input channels of the first layer
    assert np.all(g[w12 + 16:w12 + 256] == 0) and np.all(g[b12 + 1:b12 + 16] == 0)  # padded output rows


def test_dense_operator_is_spd():
    rng = np.random.default_rng(1)
    _, m, _ = _problem(1, 8, 2)
    m = m[0]
    x = np.where(m == 1, rng.standard_normal(m.shape), 0.0)
    y = np.where(m == 1, rng.standard_normal(m.shape), 0.0)
    Mx, My = U.dense_operator_apply(x, m), U.dense_operator_apply(y, m)
    assert abs(np.sum(y * Mx) - np.sum(x * My)) <= 1e-10 * np.abs(np.sum(y * Mx))
    assert np.sum(x * Mx) > 0


# ----------------------------------------------------------------- GPU: device
@pytest.fixture(scope="module")
def unet():
    from mac_b200.unet import UNet
    with UNet(0) as net:
        yield net


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.gpu
def test_device_forward_matches_oracle(unet):
    p = _random_params(11).astype(np.float32)
    assert unet.nparams == p.size
    unet.set_params(p, 0.5)
    r, m, _ = _problem(2, 16, 12)
    got = unet.forward(r, m)
    want = U.Net(p, 0.5).correction(r, m)
    assert np.all(got[m != 1] == 0)
    assert _rel(got, want) <= 2e-2, _rel(got, want)


@pytest.mark.gpu
def test_device_gradients_match_oracle(unet):
    p = _random_params(21).astype(np.float32)
    unet.set_params(p, 0.5)
    r, m, e = _problem(2, 16, 22)
    loss, g = unet.loss_grad(r, m, e)
    wl, wg = U.Net(p, 0.5).loss_grad(r, m, e)
    assert abs(loss - wl) <= 2e-2 * wl, (loss, wl)
    errs = [_rel(g[a:b], wg[a:b]) for a, b in _layer_slices()]
    assert max(errs) <= 5e-2, errs
    offs, _ = U.offsets()
    for (wo, bo), (cin, cout, *_r) in zip(offs, U.LAYERS):
        assert _rel(g[bo:bo + cout], wg[bo:bo + cout]) <= 5e-2


@pytest.mark.gpu
def test_device_energy_loss_gradients_match_oracle(unet):
    p = _random_params(25).astype(np.float32)
    unet.set_params(p, 0.5)
    unet.set_loss("energy")
    try:
        r, m, e = _problem(2, 16, 26)
        loss, g = unet.loss_grad(r, m, e)
    finally:
        unet.set_loss("mse")
    wl, wg = U.Net(p, 0.5).loss_grad(r, m, e, kind="energy")
    assert abs(loss - wl) <= 2e-2 * wl, (loss, wl)
    # the energy gradient 2 M d / count differences neighbouring output errors,
    # so the BF16 rounding flips weigh about twice as much as in the MSE case
    errs = [_rel(g[a:b], wg[a:b]) for a, b in _layer_slices()]
    assert max(errs) <= 1e-1, errs


@pytest.mark.gpu
def test_device_adam_step(unet):
    p = _random_params(31).astype(np.float32)
    unet.set_params(p, 0.5)
    g = np.random.default_rng(32).standard_normal(p.size).astype(np.float32)
    unet.adam_step(g, 1e-3)
    got, _ = unet.params()
    want, _, _ = U.adam_step(p, g, np.zeros_like(p), np.zeros_like(p), 1, 1e-3)
    assert np.max(np.abs(got - want)) <= 1e-5 * max(1.0, np.max(np.abs(want)))


@pytest.mark.gpu
def test_training_pairs_are_residual_error_pairs(unet):
    st = unet.make_dataset(nmasks=4, size=32, nsnap=4, niter=600, seed=77)
    assert st["worst_relres"] <= 1e-9, st
    assert st["tscale"] > 0
    for idx in (0, 5, 15):
        r, e, m = unet.sample(idx)
        assert np.all(r[m != 1] == 0) and np.any(m == 1)
        Me = U.dense_operator_apply(e.astype(np.float64), m)
        assert _rel(np.where(m == 1, Me, 0), r) <= 1e-5


@pytest.mark.gpu
def test_training_lowers_the_loss(unet):
    unet.set_params(_random_params(41).astype(np.float32), 1.0)
    unet.make_dataset(nmasks=16, size=32, nsnap=4, niter=600, seed=78)
    losses = unet.train(80, batch=8, lr=1e-3, seed=9)
    assert np.all(np.isfinite(losses))
    assert losses[-10:].mean() < 0.8 * losses[:10].mean(), (losses[:10].mean(), losses[-10:].mean())


def _box_problem(n, d, h, w, seed):
    rng = np.random.default_rng(seed)
    m = np.where(rng.random((n, d, h, w)) < 0.7, 1, 0).astype(np.int8)
    m[:, :, :2, :] = -1
    r = np.where(m == 1, rng.standard_normal((n, d, h, w)), 0.0).astype(np.float32)
    return r, m


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(2, 16, 16, 16), (1, 12, 20, 28), (1, 8, 36, 44), (1, 64, 64, 64)])
def test_staged_tile_forward_matches_per_tap_gather(unet, shape):
    """The forward pass with its 3x3x3 convolutions on the staged-tile kernel
    (one input box per 8 x 16 x 1 tile, taps as descriptor offsets) against the
    per-tap gather kernel: the same accumulation order, so the same output,
    on grids whose quarter-resolution levels leave partial tiles; and both
    within the oracle's tolerance."""
    p = _random_params(31).astype(np.float32)
    unet.set_params(p, 0.5)
    r, m = _box_problem(*shape, seed=32)
    try:
        unet.set_conv(False)
        ref = unet.forward(r, m)
    finally:
        unet.set_conv(True)
    got = unet.forward(r, m)
    assert np.array_equal(got, ref), _rel(got, ref)
    if shape[1] <= 16:
        want = U.Net(p, 0.5).correction(r, m)
        assert _rel(got, want) <= 2e-2, _rel(got, want)

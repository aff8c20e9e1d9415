"""The settling surrogate's MLP: the oracle's backward pass against finite differences
(CPU), and the library's tensor-core forward / backward / training against the oracle
(GPU): predictions and every parameter gradient within the stated tolerance, and a
training run that lowers the loss."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import surrogate_oracle as so


def small_params(rng, layers, width, k0=so.N_FEAT):
    p, k = {}, k0
    for l in range(layers):
        p[f"W{l}"] = (rng.uniform(-1, 1, (width, k)) / np.sqrt(k)).astype(np.float32)
        p[f"b{l}"] = (0.1 * rng.standard_normal(width)).astype(np.float32)
        k = width
    p["Wo"] = (rng.uniform(-1, 1, (so.N_OUT, width)) / np.sqrt(width)).astype(np.float32)
    p["bo"] = (0.1 * rng.standard_normal(so.N_OUT)).astype(np.float32)
    return p


def test_bf16_rounding_known_answers():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.001953125, 1.01171875, -3.14159265],
                    np.float32)
    got = so.bf16_round(vals)
    # BF16 spacing at 1 is 2^-7: 1 + 2^-8 is a tie and goes to the even neighbour 1.0,
    # 1 + 3*2^-9 lies above the midpoint, 1 + 3*2^-8 is a tie that goes to 1 + 2^-6,
    # pi rounds to 3.140625
    want = np.array([1.0, 1.0, 1.0078125, 1.0, 1.015625, -3.140625], np.float32)
    assert np.array_equal(got, want)
    import torch
    rng = np.random.default_rng(4)
    x = (rng.standard_normal(4096) * 10.0 ** rng.uniform(-6, 6, 4096)).astype(np.float32)
    assert np.array_equal(so.bf16_round(x), torch.from_numpy(x).to(torch.bfloat16).float().numpy())


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    layers, width, bands = 2, 16, 3
    p = {k: v.astype(np.float64) for k, v in small_params(rng, layers, width).items()}
    u = rng.uniform(-1, 1, (12, so.N_IN))
    t = rng.standard_normal((12, so.N_OUT))
    loss, g, _ = so.forward_backward(p, layers, u, t, bands, bf16=False)
    eps = 1e-6
    for name in ["W0", "b0", "W1", "b1", "Wo", "bo"]:
        flat = p[name].ravel()
        for j in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[j]
            flat[j] = old + eps
            lp, _, _ = so.forward_backward(p, layers, u, t, bands, bf16=False)
            flat[j] = old - eps
            lm, _, _ = so.forward_backward(p, layers, u, t, bands, bf16=False)
            flat[j] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[name].ravel()[j]) <= 1e-6 + 1e-5 * abs(fd), (name, j)


def _rows(rng, n, nin=so.N_IN):
    u = rng.uniform(-1, 1, (n, nin)).astype(np.float32)
    t = np.stack([np.sin(2 * u[:, 0]) * u[:, 3], 0.5 * u[:, 1] * u[:, 2],
                  np.cos(u[:, 4]) - u[:, 2] ** 2 + 0.3 * u[:, nin - 1]], axis=1).astype(np.float32)
    return u, t


def test_feature_layout_and_width():
    assert so.feature_width(5, 8) == 128 and so.feature_width(5, 12) == 128
    assert so.feature_width(40, 4) == 384 and so.feature_width(82, 4) == 768
    u = np.array([[0.25, -0.5, 0.125]], np.float32)
    x = so.features(u, 2, bf16=False)
    assert x.shape == (1, 128)
    want = [0.25, -0.5, 0.125]
    for f in range(2):
        for i in range(3):
            a = np.float32(2.0 ** f * 3.14159265358979) * u[0, i]
            want += [np.sin(a), np.cos(a)]
    assert np.allclose(x[0, :15], want) and not x[0, 15:].any()


@pytest.mark.gpu
@pytest.mark.parametrize("width,nin,bands", [(256, 5, 8), (128, 5, 8), (256, 40, 4)])
def test_gpu_forward_and_gradients_match_oracle(gpu, width, nin, bands):
    """nin 40, bands 4: a 384-wide first layer, whose weight gradient takes one 256-wide
    and one 128-wide tile of columns."""
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=width, hidden_layers=4, fourier_bands=bands, batch=1024, seed=3,
                            inputs=nin)
    rng = np.random.default_rng(1)
    with sg.Surrogate(cfg) as s:
        p = small_params(rng, 4, width, so.feature_width(nin, bands))
        s.set_params(sg.flatten(p, cfg))
        assert np.array_equal(s.get_params(), sg.flatten(p, cfg))
        u, t = _rows(rng, 512, nin)
        y = s.predict(u)
        _, _, y_ref = so.forward_backward(p, 4, u, t, bands)
        # BF16 activations: a relative error of a few 1e-3 of the output scale
        assert np.max(np.abs(y - y_ref)) <= 2e-2 * (np.max(np.abs(y_ref)) + 1e-3)
        g, loss = s.gradients(u, t)
        loss_ref, g_ref, _ = so.forward_backward(p, 4, u, t, bands)
        assert abs(loss - loss_ref) <= 1e-2 * loss_ref
        gg = sg.unflatten(g, cfg)
        for name, _ in sg.param_shapes(cfg):
            a, b = gg[name].astype(np.float64), g_ref[name]
            rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
            assert rel < 2e-2, (name, rel)
        # predictions of rows that are not a multiple of 128, split over batches
        u2, _ = _rows(rng, 1500, nin)
        y2 = s.predict(u2)
        _, _, y2_ref = so.forward_backward(p, 4, u2, np.zeros((1500, 3), np.float32), bands)
        assert np.max(np.abs(y2 - y2_ref)) <= 2e-2 * (np.max(np.abs(y2_ref)) + 1e-3)


@pytest.mark.gpu
def test_gpu_predict_from_device_memory_equals_host_predict(gpu):
    import torch
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=256, hidden_layers=4, fourier_bands=4, batch=1024, seed=7, inputs=40)
    rng = np.random.default_rng(8)
    u, _ = _rows(rng, 300000, 40)  # one full 262,144-row chunk and a ragged one
    with sg.Surrogate(cfg) as s:
        y = s.predict(u)
        du = torch.from_numpy(u).cuda()
        dy = torch.empty((u.shape[0], 3), dtype=torch.float32, device="cuda")
        s.predict_device(du.data_ptr(), u.shape[0], dy.data_ptr())
        assert s.stream_handle != 0
    assert np.array_equal(dy.cpu().numpy(), y)


@pytest.mark.gpu
def test_gpu_training_lowers_the_loss(gpu):
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=256, hidden_layers=4, fourier_bands=6, batch=4096, seed=5,
                            learning_rate=2e-3)
    rng = np.random.default_rng(2)
    u, t = _rows(rng, 50000)
    with sg.Surrogate(cfg) as s:
        s.set_data(u, t)
        first = s.train(1)
        s.train(300)
        last = s.train(1)
        uv, tv = _rows(rng, 4096)
        mse = float(np.mean((s.predict(uv) - tv) ** 2))
    assert last < 0.1 * first
    assert mse < 0.1 * float(np.mean(tv ** 2))


@pytest.mark.gpu
def test_gpu_training_with_cosine_decay_and_wide_inputs(gpu):
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=256, hidden_layers=4, fourier_bands=4, batch=4096, seed=6,
                            learning_rate=2e-3, inputs=40, cosine_decay=1)
    rng = np.random.default_rng(3)
    u, t = _rows(rng, 50000, 40)
    with sg.Surrogate(cfg) as s:
        s.set_data(u, t)
        first = s.train(1)
        s.train(300)
        uv, tv = _rows(rng, 4096, 40)
        mse = float(np.mean((s.predict(uv) - tv) ** 2))
    assert mse < 0.2 * float(np.mean(tv ** 2)) and mse < first


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [128, 384, 1500, 37888 + 256, 300000])
def test_gpu_pingpong_forward_equals_block_forward(gpu, rows):
    """The persistent ping-pong forward pass against the one-CTA-per-block pass: one block,
    an odd number of blocks (the last pair's second block empty), a ragged row count, more
    pairs than SMs (each CTA takes several), and a full predict chunk plus a ragged one.
    The hidden layers are the same arithmetic; the output layer's FP32 sums are added in
    another order, so the outputs agree to FP32 rounding of the 256-term sums."""
    from hidem_b200 import abi
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=256, hidden_layers=4, fourier_bands=4, batch=1024, seed=9, inputs=82)
    rng = np.random.default_rng(rows)
    u, t = _rows(rng, rows, 82)
    with sg.Surrogate(cfg) as s:
        p = small_params(rng, 4, 256, so.feature_width(82, 4))
        s.set_params(sg.flatten(p, cfg))
        s.set_forward(abi.SURROGATE_FORWARD_BLOCK)
        y_block = s.predict(u)
        s.set_forward(abi.SURROGATE_FORWARD_PINGPONG)
        y_pp = s.predict(u)
        scale = np.abs(y_block).max() + 1e-6
        assert np.max(np.abs(y_pp - y_block)) <= 1e-5 * scale
        assert not np.array_equal(y_pp, np.zeros_like(y_pp))
        if rows % 128 == 0 and rows <= 1024:
            # training's forward pass too: the gradients agree to FP32 rounding of the loss
            g_pp, l_pp = s.gradients(u, t)
            s.set_forward(abi.SURROGATE_FORWARD_BLOCK)
            g_bl, l_bl = s.gradients(u, t)
            assert abs(l_pp - l_bl) <= 1e-5 * l_bl
            assert np.linalg.norm(g_pp - g_bl) <= 1e-4 * np.linalg.norm(g_bl)


@pytest.mark.gpu
def test_gpu_pingpong_forward_is_refused_for_width_128(gpu):
    from hidem_b200 import abi
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=128, hidden_layers=2, fourier_bands=2, batch=1024, seed=1)
    with sg.Surrogate(cfg) as s:
        with pytest.raises(abi.HidemError):
            s.set_forward(abi.SURROGATE_FORWARD_PINGPONG)
        s.set_forward(abi.SURROGATE_FORWARD_AUTO)
        with pytest.raises(abi.HidemError):
            s.set_forward(7)


@pytest.mark.gpu
@pytest.mark.parametrize("layers,nin,bands", [(1, 5, 8), (8, 5, 8), (2, 40, 4)])
def test_gpu_pingpong_forward_other_depths_and_widths(gpu, layers, nin, bands):
    """One hidden layer (the output layer's partial sums share the activation tile with the
    feature slots), the deepest network, and a 384-wide first layer, against the
    one-CTA-per-block pass and the oracle."""
    from hidem_b200 import abi
    from hidem_b200 import surrogate as sg
    cfg = sg.default_config(width=256, hidden_layers=layers, fourier_bands=bands, batch=1024, seed=4,
                            inputs=nin)
    rng = np.random.default_rng(10 + layers)
    u, t = _rows(rng, 1500, nin)
    with sg.Surrogate(cfg) as s:
        p = small_params(rng, layers, 256, so.feature_width(nin, bands))
        s.set_params(sg.flatten(p, cfg))
        y_pp = s.predict(u)
        s.set_forward(abi.SURROGATE_FORWARD_BLOCK)
        y_block = s.predict(u)
    assert np.max(np.abs(y_pp - y_block)) <= 1e-5 * (np.abs(y_block).max() + 1e-6)
    _, _, y_ref = so.forward_backward(p, layers, u, t, bands)
    assert np.max(np.abs(y_pp - y_ref)) <= 2e-2 * (np.max(np.abs(y_ref)) + 1e-3)

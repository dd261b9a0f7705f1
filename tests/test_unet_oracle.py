"""CPU checks of the U-Net oracle (the specification the GPU kernels are
tested against) and of the network's parameter layout in the library."""
import numpy as np
import pytest

import unet_oracle as U


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-8, 8, 4000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, -3.5e-39]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    assert np.array_equal(U.bf16(x), ref)


def test_prolongation_adjoint():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(3, 5, 4, 2))
    b = rng.normal(size=(5, 9, 7, 2))
    assert abs(np.sum(U.prolong(a) * b) - np.sum(a * U.prolong_t(b))) < 1e-12 * np.sum(np.abs(a)) * 10
    # vertex-centred: coarse values are kept at even fine nodes, odd nodes average
    p = U.prolong(a)
    assert np.allclose(p[::2, ::2, ::2], a)
    assert np.allclose(p[1, 0, 0], 0.5 * (a[0, 0, 0] + a[1, 0, 0]))


@pytest.mark.parametrize("stride", [1, 2])
def test_conv_backward_adjoint(stride):
    rng = np.random.default_rng(stride)
    x = rng.normal(size=(5, 9, 7, 3))
    W = rng.normal(size=(27, 3, 4))
    out_shape = (5, 9, 7) if stride == 1 else (3, 5, 4)
    g = rng.normal(size=out_shape + (4,))
    y = U.conv(x, W, np.zeros(4), stride, out_shape)
    dx, dW, db = U.conv_backward(x, W, g, stride)
    # linearity in x and in W: <conv(x), g> = <x, dx> = <W, dW>
    s = np.sum(y * g)
    assert abs(s - np.sum(x * dx)) < 1e-9 * abs(s) + 1e-9
    assert abs(s - np.sum(W * dW)) < 1e-9 * abs(s) + 1e-9
    assert np.allclose(db, g.reshape(-1, 4).sum(0))


@pytest.mark.parametrize("w_h1", [0.0, 0.7])
def test_oracle_gradient_matches_finite_differences(w_h1):
    """Pins the oracle's reverse-mode gradient: central differences of the
    unrounded FP64 network at randomly chosen parameters of every layer."""
    theta = U.init_params(11).astype(np.float64)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(9, 5, 13))
    y, t = U.forward_plain(theta, x)
    target = rng.normal(size=y.shape) * 0.1
    loss, g = U.backward_plain(theta, t, target, 1.0, w_h1)
    offs = np.cumsum([0] + [a + b for (a, b, _, _) in U.layer_shapes()])
    h = 1e-6
    for layer in range(len(U.CONVS)):
        for idx in rng.integers(offs[layer], offs[layer + 1], size=3):
            tp, tm = theta.copy(), theta.copy()
            tp[idx] += h
            tm[idx] -= h
            lp = U.loss_and_grad(U.forward_plain(tp, x)[0], target, 1.0, w_h1)[0]
            lm = U.loss_and_grad(U.forward_plain(tm, x)[0], target, 1.0, w_h1)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-5 * max(abs(fd), abs(g[idx])) + 1e-10, (layer, idx, fd, g[idx])


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(4)
    out = rng.normal(size=(5, 5, 9))
    tgt = rng.normal(size=out.shape)
    _, g = U.loss_and_grad(out, tgt, 0.3, 1.3)
    for idx in [(0, 0, 0), (2, 3, 4), (4, 4, 8), (1, 0, 5)]:
        e = np.zeros_like(out)
        e[idx] = 1e-6
        fd = (U.loss_and_grad(out + e, tgt, 0.3, 1.3)[0] - U.loss_and_grad(out - e, tgt, 0.3, 1.3)[0]) / 2e-6
        assert abs(fd - g[idx]) < 1e-6 * max(1.0, abs(fd))


def test_rounded_network_close_to_plain():
    theta = U.init_params(5)
    x = np.random.default_rng(6).normal(size=(9, 9, 9))
    y16, _ = U.forward(theta, x)
    y64, _ = U.forward_plain(U.bf16(theta), x)
    rel = np.linalg.norm(y16 - y64) / np.linalg.norm(y64)
    assert rel < 3e-2  # BF16 activations: ~2^-9 relative per layer


def test_library_param_layout_matches_oracle():
    import cfdfs
    assert cfdfs.UNet.param_count() == U.param_count()


def test_grid_rule():
    with pytest.raises(ValueError):
        U.level_dims((8, 9, 9))
    assert U.level_dims((65, 25, 161)) == [(65, 25, 161), (33, 13, 81), (17, 7, 41)]

"""The U-Net oracle pinned on the CPU.

The learned preconditioner has no counterpart in the reference. The oracle's
float64 gradient is pinned against central finite differences of its own
loss, and its bf16 mode is checked for rounding at the stated points only.
"""
import numpy as np
import pytest


def _scene(U, D=8, H=8, W=12, seed=1):
    rng = np.random.default_rng(seed)
    lab = np.full((D, H, W), U.FLUID, np.uint8)
    lab[0] = U.SOLID
    lab[:, 0] = U.SOLID
    lab[:, :, 0] = U.SOLID
    lab[:, -2:] = U.AIR
    lab[3, 3, 3] = U.BODY
    rhs = rng.standard_normal((D, H, W)).astype(np.float32)
    p = rng.standard_normal((D, H, W)).astype(np.float32)
    return lab, rhs, p


def test_param_count_and_layout():
    from oracle import unet_oracle as U
    assert U.n_params() == 27 * (256 + 256 + 512 + 1024 + 2048 + 4096 + 3072 + 1024 + 768 + 256) + 16 == 359440
    ws, wh = U.split(np.arange(U.n_params(), dtype=np.float64))
    assert [w.shape for w in ws][6] == (27, 32, 96) and wh.shape == (16,)
    assert ws[0][0, 0, 1] == 1 and ws[1][0, 0, 0] == 27 * 16 * 16


def test_bf16_rounding():
    from oracle import unet_oracle as U
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -3.14159, 0.0], np.float32)
    r = U.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 4 * 2 ** -8    # tie to even (up)
    assert r[3] == 1.0
    assert r[4] == -3.140625 and r[5] == 0.0


def test_float64_gradient_matches_finite_differences():
    from oracle import unet_oracle as U
    lab, rhs, p = _scene(U)
    th = U.init_params(3).astype(np.float64)
    _, g = U.loss_grad(th, lab, rhs, p, bf=False)
    rng = np.random.default_rng(5)
    sizes = np.cumsum([0] + U.layer_sizes())
    # a few parameters of every layer plus the head
    idx = [int(rng.integers(sizes[i], sizes[i + 1])) for i in range(10) for _ in range(3)]
    idx += [U.n_params() - 1, U.n_params() - 9]
    h = 1e-6
    for i in idx:
        e = np.zeros_like(th)
        e[i] = h
        fd = (U.loss_grad(th + e, lab, rhs, p, bf=False)[0] - U.loss_grad(th - e, lab, rhs, p, bf=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * (abs(fd) + abs(g[i])) + 1e-10, (i, fd, g[i])


def test_bf16_mode_is_close_to_float64():
    from oracle import unet_oracle as U
    lab, rhs, p = _scene(U)
    th = U.init_params(4)
    l64, g64 = U.loss_grad(th, lab, rhs, p, bf=False)
    l16, g16 = U.loss_grad(th, lab, rhs, p, bf=True)
    assert abs(l16 - l64) <= 2e-2 * l64
    # bf16 storage of activations and their gradients costs about 10% of the
    # gradient's norm at random initialisation; its direction is kept
    cos = float(g16 @ g64) / (np.linalg.norm(g16) * np.linalg.norm(g64))
    assert cos >= 0.99 and np.linalg.norm(g16 - g64) <= 0.15 * np.linalg.norm(g64)


def test_padding_and_scale():
    from oracle import unet_oracle as U
    lab, rhs, _ = _scene(U, D=6, H=9, W=10)
    x, s, inv_s, f = U.make_input(lab, rhs, bf=False)
    assert x.shape == (8, 12, 12, 16)
    assert np.all(x[6:, :, :, 3] == 1) and np.all(x[:, 9:, :, 3] == 1)
    fl = lab == U.FLUID
    assert s == pytest.approx(np.sqrt(np.mean(rhs[fl].astype(np.float64) ** 2)))
    assert np.all(x[:6, :9, :10, 0][~fl] == 0)
    out, xd, _ = U.forward(U.init_params(0), lab, rhs)
    assert out.shape == (8, 12, 12) and xd.shape == lab.shape and np.all(xd[~fl] == 0)

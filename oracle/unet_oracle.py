"""CPU oracle of the learned pressure preconditioner (test infrastructure only).

The reference has no learned component. Its pressure solve is the cuDSS call
at FluidSolver3D.cu:1930-2008, and this network is an addition beside it. So
this module is the arbiter of the CUDA network in fluidprjct_b200/csrc/
kernels_unet.cu and unet.cu. It restates the same forward pass, loss and
backward pass in float64 numpy. With ``bf16=True`` it rounds to bfloat16
(round to nearest even) at exactly the points where the CUDA path stores
bf16: the weights, the input tensor, every stored activation and every
stored activation gradient. Only accumulation order and FP32 arithmetic are
then left to differ. With ``bf16=False`` it is plain float64, and the tests
pin its gradient against central finite differences.

Network (3 levels, 16/32/64 channels, 3x3x3 convolutions, zero padding, no
bias, ReLU after every 3x3x3 convolution):

    X0 (16 ch: rhs/s on FLUID, FLUID, AIR, SOLID-or-BODY-or-padding, 12 zeros)
    L0 16->16, L1 16->16 = e0 -> avgpool2 -> q0
    L2 16->32, L3 32->32 = e1 -> avgpool2 -> q1
    L4 32->64, L5 64->64 = e2
    L6 [up2(e2) | e1] 96->32, L7 32->32 = d1
    L8 [up2(d1) | e0] 48->16, L9 16->16 = d0
    out = d0 . wh (16 FP32 weights);  x0 = s * out on FLUID cells

s is the RMS of the right-hand side over FLUID cells. Grid dims are padded
up to multiples of 4, and the padding counts as SOLID. The loss is
sum_F (out - p/s)^2 / sum_F (p/s)^2 over FLUID cells F.

Weights are flattened layer by layer as [27][COUT][CIN] (tap = (dz+1)*9 +
(dy+1)*3 + (dx+1)), followed by the 16 head weights.
"""
import numpy as np

SOLID, FLUID, AIR, BODY = 0, 1, 2, 3

# (name, level, CA = channels of the upsampled coarse input, CB = same-level input channels, COUT)
LAYERS = [
    ("L0", 0, 0, 16, 16),
    ("L1", 0, 0, 16, 16),
    ("L2", 1, 0, 16, 32),
    ("L3", 1, 0, 32, 32),
    ("L4", 2, 0, 32, 64),
    ("L5", 2, 0, 64, 64),
    ("L6", 1, 64, 32, 32),
    ("L7", 1, 0, 32, 32),
    ("L8", 0, 32, 16, 16),
    ("L9", 0, 0, 16, 16),
]
HEAD = 16
IN_CH = 16


def layer_sizes():
    return [27 * cout * (ca + cb) for _, _, ca, cb, cout in LAYERS]


def n_params():
    return sum(layer_sizes()) + HEAD


def split(params):
    """Flat parameter vector -> list of (27, COUT, CIN) arrays and the head."""
    params = np.asarray(params, np.float64)
    out, o = [], 0
    for (_, _, ca, cb, cout), n in zip(LAYERS, layer_sizes()):
        out.append(params[o:o + n].reshape(27, cout, ca + cb))
        o += n
    return out, params[o:o + HEAD]


def init_params(seed=0):
    """He-normal 3x3x3 weights and a small head (numpy RNG; for tests)."""
    rng = np.random.default_rng(seed)
    parts = []
    for _, _, ca, cb, cout in LAYERS:
        cin = ca + cb
        parts.append(rng.standard_normal(27 * cout * cin) * np.sqrt(2.0 / (27 * cin)))
    parts.append(rng.standard_normal(HEAD) * 0.25)
    return np.concatenate(parts).astype(np.float32)


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    x32 = np.ascontiguousarray(x, np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    b = (b + (((b >> 16) & 1) + 0x7FFF)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _tap_offsets():
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                yield dz, dy, dx


def _pad(x):
    return np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))


def conv(x, w):
    """y[v, co] = sum_t sum_ci x[v + off(t), ci] * w[t, co, ci] (zero padding)."""
    D, H, W, _ = x.shape
    xp = _pad(x)
    y = np.zeros((D, H, W, w.shape[1]))
    for t, (dz, dy, dx) in enumerate(_tap_offsets()):
        y += xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] @ w[t].T
    return y


def conv_t(g, w):
    """dx[v, ci] = sum_t sum_co g[v - off(t), co] * w[t, co, ci]."""
    D, H, W, _ = g.shape
    gp = _pad(g)
    y = np.zeros((D, H, W, w.shape[2]))
    for t, (dz, dy, dx) in enumerate(_tap_offsets()):
        y += gp[1 - dz:1 - dz + D, 1 - dy:1 - dy + H, 1 - dx:1 - dx + W] @ w[t]
    return y


def corr(x, g):
    """dw[t, co, ci] = sum_v g[v, co] * x[v + off(t), ci]."""
    D, H, W, cin = x.shape
    xp = _pad(x)
    gm = g.reshape(-1, g.shape[-1]).T
    out = np.zeros((27, g.shape[-1], cin))
    for t, (dz, dy, dx) in enumerate(_tap_offsets()):
        out[t] = gm @ xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W].reshape(-1, cin)
    return out


def pool(x):
    D, H, W, C = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def sum_children(x):
    D, H, W, C = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(1, 3, 5))


def net_dims(D, H, W):
    r = lambda n: (n + 3) // 4 * 4
    return r(D), r(H), r(W)


def scale_of(labels, rhs):
    """(s, 1/s as float32) with s the RMS of rhs over FLUID cells (1 if none)."""
    f = labels == FLUID
    n = int(f.sum())
    ss = float(np.sum(np.asarray(rhs, np.float64)[f] ** 2))
    s = np.sqrt(ss / n) if n > 0 and ss > 0 else 1.0
    return s, np.float32(1.0 / s)


def make_input(labels, rhs, bf=True):
    """The 16-channel input tensor on the padded grid, and (s, inv_s)."""
    D, H, W = labels.shape
    Dn, Hn, Wn = net_dims(D, H, W)
    s, inv_s = scale_of(labels, rhs)
    lab = np.full((Dn, Hn, Wn), SOLID, np.uint8)
    lab[:D, :H, :W] = labels
    r = np.zeros((Dn, Hn, Wn), np.float32)
    r[:D, :H, :W] = np.asarray(rhs, np.float32)
    x = np.zeros((Dn, Hn, Wn, IN_CH))
    f = lab == FLUID
    c0 = np.where(f, r * inv_s, np.float32(0)).astype(np.float32)
    x[..., 0] = c0
    x[..., 1] = f
    x[..., 2] = lab == AIR
    x[..., 3] = (lab == SOLID) | (lab == BODY)
    return (bf16(x) if bf else x), s, inv_s, f


def forward(params, labels, rhs, bf=True):
    """Returns (out on the padded grid, x0 on the real grid, cache)."""
    rnd = bf16 if bf else (lambda a: a)
    relu = lambda a: np.maximum(a, 0.0)
    ws, wh = split(params)
    if bf:
        ws = [bf16(w) for w in ws]
        wh = np.asarray(wh, np.float32).astype(np.float64)
    x0, s, inv_s, f = make_input(labels, rhs, bf)
    c = {"X0": x0, "s": s, "inv_s": inv_s, "fluid": f, "ws": ws, "wh": wh}
    c["a0"] = rnd(relu(conv(x0, ws[0])))
    c["e0"] = rnd(relu(conv(c["a0"], ws[1])))
    c["q0"] = rnd(pool(c["e0"]))
    c["a1"] = rnd(relu(conv(c["q0"], ws[2])))
    c["e1"] = rnd(relu(conv(c["a1"], ws[3])))
    c["q1"] = rnd(pool(c["e1"]))
    c["a2"] = rnd(relu(conv(c["q1"], ws[4])))
    c["e2"] = rnd(relu(conv(c["a2"], ws[5])))
    c["in6"] = np.concatenate([up(c["e2"]), c["e1"]], axis=-1)
    c["d1a"] = rnd(relu(conv(c["in6"], ws[6])))
    c["d1"] = rnd(relu(conv(c["d1a"], ws[7])))
    c["in8"] = np.concatenate([up(c["d1"]), c["e0"]], axis=-1)
    c["d0a"] = rnd(relu(conv(c["in8"], ws[8])))
    c["d0"] = rnd(relu(conv(c["d0a"], ws[9])))
    out = c["d0"] @ wh
    c["out"] = out
    D, H, W = labels.shape
    xd = np.where(labels == FLUID, out[:D, :H, :W] * s, 0.0)
    return out, xd, c


def loss_grad(params, labels, rhs, p, bf=True):
    """(loss, flat gradient) of the relative L2 loss against the pressure p."""
    rnd = bf16 if bf else (lambda a: a)
    out, _, c = forward(params, labels, rhs, bf)
    ws, wh, f = c["ws"], c["wh"], c["fluid"]
    D, H, W = labels.shape
    t = np.zeros(out.shape)
    t[:D, :H, :W] = (np.asarray(p, np.float32) * c["inv_s"]).astype(np.float32)
    t = np.where(f, t, 0.0)
    err = np.where(f, out - t, 0.0)
    tt = float(np.sum(t * t))
    tt = tt if tt > 0 else 1.0
    loss = float(np.sum(err * err)) / tt
    g_out = 2.0 * err / tt
    gh = np.einsum("zyx,zyxc->c", g_out, c["d0"])
    dw = [None] * 10
    g9 = rnd(g_out[..., None] * wh * (c["d0"] > 0))
    dw[9] = corr(c["d0a"], g9)
    g8 = rnd(conv_t(g9, ws[9]) * (c["d0a"] > 0))
    dw[8] = corr(c["in8"], g8)
    raw8 = rnd(conv_t(g8, ws[8]))
    g7 = rnd(sum_children(raw8[..., :32]) * (c["d1"] > 0))
    dw[7] = corr(c["d1a"], g7)
    g6 = rnd(conv_t(g7, ws[7]) * (c["d1a"] > 0))
    dw[6] = corr(c["in6"], g6)
    raw6 = rnd(conv_t(g6, ws[6]))
    g5 = rnd(sum_children(raw6[..., :64]) * (c["e2"] > 0))
    dw[5] = corr(c["a2"], g5)
    g4 = rnd(conv_t(g5, ws[5]) * (c["a2"] > 0))
    dw[4] = corr(c["q1"], g4)
    gq1 = rnd(conv_t(g4, ws[4]))
    g3 = rnd((raw6[..., 64:] + up(gq1) * 0.125) * (c["e1"] > 0))
    dw[3] = corr(c["a1"], g3)
    g2 = rnd(conv_t(g3, ws[3]) * (c["a1"] > 0))
    dw[2] = corr(c["q0"], g2)
    gq0 = rnd(conv_t(g2, ws[2]))
    g1 = rnd((raw8[..., 32:] + up(gq0) * 0.125) * (c["e0"] > 0))
    dw[1] = corr(c["a0"], g1)
    g0 = rnd(conv_t(g1, ws[1]) * (c["a0"] > 0))
    dw[0] = corr(c["X0"], g0)
    grad = np.concatenate([d.ravel() for d in dw] + [gh])
    return loss, grad

"""Test infrastructure only: float64 numpy restatement of the learned channel estimator's
network (ocudu-dapp-platform_b200/csrc/learned_est.cu and tc_conv1d.cu), used to check the GPU
forward pass, the GPU gradients and the feature construction.

The reference has no learned estimator (its estimator is
lib/phy/upper/signal_processors/channel_estimator/port_channel_estimator_average_impl.cpp), so
there is nothing of the reference to pin here: the checker is exact arithmetic. With
``bf16=True`` the restatement rounds to bf16 exactly where the GPU stores bf16 (weights,
activations, output and input gradients), so that the remaining difference is FP32 accumulation
order; with ``bf16=False`` it is the exact float64 network.

Parameter layout (the C ABI's): per layer, weights [5][cin][cout] then bias [cout]; layers in
network order: 16->64, 6 x (64->64, 64->64 + residual), 64->16.
"""
import numpy as np

TAPS = 5
BLOCKS = 6
LAYERS = [(16, 64)] + [(64, 64)] * (2 * BLOCKS) + [(64, 16)]


def layer_offsets():
    offs, o = [], 0
    for cin, cout in LAYERS:
        offs.append(o)
        o += TAPS * cin * cout + cout
    return offs, o


def bf16(x):
    """Round to bf16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32).astype(np.float64)


def unpack(params):
    offs, total = layer_offsets()
    assert params.size == total
    out = []
    for (cin, cout), o in zip(LAYERS, offs):
        w = params[o:o + TAPS * cin * cout].reshape(TAPS, cin, cout).astype(np.float64)
        b = params[o + TAPS * cin * cout:o + TAPS * cin * cout + cout].astype(np.float64)
        out.append((w, b))
    return out


def conv(x, w):
    """y[r][co] = sum_t sum_ci x[r + t - 2][ci] w[t][ci][co], zero outside the buffer."""
    rows = x.shape[0]
    xp = np.zeros((rows + 4, x.shape[1]))
    xp[2:2 + rows] = x
    return sum(xp[t:t + rows] @ w[t] for t in range(TAPS))


def conv_t(dy, w):
    """Input gradient of conv: dx[q][ci] = sum_t sum_co dy[q - t + 2][co] w[t][ci][co]."""
    rows = dy.shape[0]
    dp = np.zeros((rows + 4, dy.shape[1]))
    dp[2:2 + rows] = dy
    return sum(dp[4 - t:4 - t + rows] @ w[t].T for t in range(TAPS))


def wgrad(x, dy):
    rows = x.shape[0]
    xp = np.zeros((rows + 4, x.shape[1]))
    xp[2:2 + rows] = x
    return np.stack([xp[t:t + rows].T @ dy for t in range(TAPS)]), dy.sum(0)


def forward(params, x, valid, bf16_acts=True):
    """Network output [rows][16] and the activations needed by backward."""
    R = (lambda a: bf16(a) * valid[:, None]) if bf16_acts else (lambda a: a * valid[:, None])
    lay = unpack(params)
    if bf16_acts:
        lay = [(bf16(w), b) for w, b in lay]
    x = R(x)
    a = [x]
    h = R(np.maximum(conv(x, lay[0][0]) + lay[0][1], 0))
    a.append(h)
    mids = []
    for k in range(BLOCKS):
        w1, b1 = lay[1 + 2 * k]
        w2, b2 = lay[2 + 2 * k]
        m = R(np.maximum(conv(h, w1) + b1, 0))
        mids.append(m)
        h = R(np.maximum(conv(m, w2) + b2 + h, 0))
        a.append(h)
    y = R(conv(h, lay[-1][0]) + lay[-1][1])
    return y, dict(a=a, mids=mids, lay=lay, valid=valid, bf16=bf16_acts)


def backward(cache, dy):
    """Gradients in the parameter layout for the output gradient dy [rows][16]."""
    valid, lay, a, mids = cache["valid"], cache["lay"], cache["a"], cache["mids"]
    R = (lambda v: bf16(v) * valid[:, None]) if cache["bf16"] else (lambda v: v * valid[:, None])
    dy = R(dy)
    grads = [None] * len(LAYERS)
    grads[-1] = wgrad(a[-1], dy)
    G = R(conv_t(dy, lay[-1][0]) * (a[-1] > 0))
    for k in range(BLOCKS - 1, -1, -1):
        l1, l2 = 1 + 2 * k, 2 + 2 * k
        grads[l2] = wgrad(mids[k], G)
        H = R(conv_t(G, lay[l2][0]) * (mids[k] > 0))
        grads[l1] = wgrad(a[k + 1], H)
        G = R((conv_t(H, lay[l1][0]) + G) * (a[k + 1] > 0))
    grads[0] = wgrad(a[0], G)
    return np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])


# ----------------------------------------------------------------------------------------------
# Features and refinement (learned_est.cu le_features_kernel / le_apply_kernel).

def sequences(ues, est_offsets):
    """(row0, len, est0, dstride, u, port, layer, nd) per allocation, rows as the GPU lays them out
    (two zero rows before each); ues: dicts with nof_rb, nof_layers, nof_rx_ports, nd."""
    out, row = [], 0
    for u, ue in enumerate(ues):
        nsc = 12 * ue["nof_rb"]
        nl, nd = ue["nof_layers"], ue["nd"]
        for p in range(ue["nof_rx_ports"]):
            for l in range(nl):
                row += 2
                out.append((row, nsc, est_offsets[u] + (p * nd * nl + l) * nsc, nl * nsc, u, p, l, nd))
                row += nsc
    return out, row


def features(seqs, rows, est, ls, noise_var, rsrp, beta):
    """[rows][16] features and the per-sequence gain g (est, ls: complex arrays in the
    frequency-response layout; noise_var[u][p], rsrp[u][p][l], beta[u])."""
    x = np.zeros((rows, 16))
    valid = np.zeros(rows, bool)
    gains = []
    for (r0, n, e0, ds, u, p, l, nd) in seqs:
        r = rsrp[u][p][l]
        g = beta[u] / np.sqrt(r) if r > 0 else 0.0
        gains.append(g)
        k = np.arange(n)
        valid[r0:r0 + n] = True
        if g == 0:
            continue
        p0 = est[e0 + k]
        p1 = est[e0 + (ds if nd > 1 else 0) + k]
        l0 = ls[e0 + k]
        l1 = ls[e0 + (ds if nd > 1 else 0) + k]
        nf = np.clip(np.log10(max(noise_var[u][p] * g * g / beta[u] ** 2, 1e-12)) * 0.5, -4, 4)
        blk = np.zeros((n, 16))
        blk[:, 0], blk[:, 1] = g * p0.real, g * p0.imag
        blk[:, 2], blk[:, 3] = g * p1.real, g * p1.imag
        blk[:, 4], blk[:, 5] = g * l0.real, g * l0.imag
        blk[:, 6], blk[:, 7] = g * l1.real, g * l1.imag
        blk[:, 8] = nf
        blk[:, 9] = (k % 2 == 0)
        blk[:, 10] = np.maximum(0, 1 - k / 8)
        blk[:, 11] = np.maximum(0, 1 - (n - 1 - k) / 8)
        blk[:, 12] = 1.0 if ds // n > 1 else 0.0
        blk[:, 13] = 1.0 if nd > 1 else 0.0
        x[r0:r0 + n] = blk
    return x, valid, np.array(gains)


def refine(seqs, est, y, gains):
    """est + correction / g at the DM-RS symbols (a copy), and the time-basis coefficients
    a_1 / g, a_2 / g (outputs 4-7) of the sequences with two DM-RS symbols in a buffer of est's
    layout (zero elsewhere): the channel at symbol s is then h_0 + (h_1 - h_0) w + a_1 w (1 - w)
    + a_2 w (1 - w) (2 w - 1), w = (s - d0) / (d1 - d0)."""
    out = est.copy()
    basis = np.zeros_like(est)
    for (r0, n, e0, ds, u, p, l, nd), g in zip(seqs, gains):
        if g <= 0:
            continue
        for d in range(nd):
            c = (y[r0:r0 + n, 2 * d] + 1j * y[r0:r0 + n, 2 * d + 1]) / g
            out[e0 + d * ds:e0 + d * ds + n] += c
        if nd == 2:
            for b in range(2):
                basis[e0 + b * ds:e0 + b * ds + n] = (y[r0:r0 + n, 4 + 2 * b] + 1j * y[r0:r0 + n, 5 + 2 * b]) / g
    return out, basis

"""Host-side layouts of the tensor-core convolution layers (csrc/tc_conv1d.cu): activations as
[C/8][rows][8] bf16 and packed weights [5 taps][cin/8][cout][8]; conversions to and from plain
[rows][C] float arrays, and bf16 rounding (round to nearest even) in numpy."""
import numpy as np


def bf16_bits(x):
    """float32 array -> uint16 bf16 bit patterns, round to nearest even (NaN kept quiet)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    nan = (u & 0x7FFFFFFF) > 0x7F800000
    r[nan] = ((u[nan] >> 16) | 0x40).astype(np.uint16)
    return r


def bf16_round(x):
    return (bf16_bits(x).astype(np.uint32) << 16).view(np.float32)


def from_bf16_bits(b):
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def to_chunked(a):
    """[rows][C] float -> [C/8][rows][8] bf16 bits (C a multiple of 8)."""
    rows, c = a.shape
    return np.ascontiguousarray(bf16_bits(a).reshape(rows, c // 8, 8).transpose(1, 0, 2))


def from_chunked(b):
    """[C/8][rows][8] bf16 bits -> [rows][C] float."""
    c8, rows, _ = b.shape
    return from_bf16_bits(np.ascontiguousarray(b.transpose(1, 0, 2)).reshape(rows, c8 * 8))


def pack_weights(w):
    """W[co][ci][5] float -> packed [5][ci/8][co][8] bf16 bits."""
    co, ci, t = w.shape
    p = np.transpose(w, (2, 1, 0)).reshape(t, ci // 8, 8, co).transpose(0, 1, 3, 2)
    return np.ascontiguousarray(bf16_bits(p))


def conv1d_ref(x, w, b, res=None, relu=False, valid=None):
    """Float64 'same' convolution with zero padding on [rows][cin] x (already bf16-rounded):
    y[r][co] = sum_{t,ci} x[r+t-2][ci] w[co][ci][t] + b[co] (+ res) (ReLU)."""
    rows, ci = x.shape
    co = w.shape[0]
    xp = np.zeros((rows + 4, ci))
    xp[2:2 + rows] = x
    y = np.zeros((rows, co))
    for t in range(5):
        y += xp[t:t + rows] @ w[:, :, t].astype(np.float64).T
    y += b
    if res is not None:
        y += res
    if relu:
        y = np.maximum(y, 0)
    return y


def pack_weights_t(w):
    """Packed weights of the input-gradient convolution of a layer W[co][ci][5]:
    W'[ci][co][t] = W[co][ci][4 - t], packed as [5][co/8][ci][8] bf16 bits."""
    return pack_weights(np.ascontiguousarray(np.asarray(w)[:, :, ::-1].transpose(1, 0, 2)))


def conv1d_backward_ref(x, w, dy):
    """Float64 gradients of y = conv(x, W) (+ b) for 'same' zero padding on one sample:
    dx[q][ci] = sum_{t,co} dy[q - t + 2][co] W[co][ci][t], dw[t][ci][co] = sum_r x[r + t - 2][ci] dy[r][co],
    db[co] = sum_r dy[r][co]."""
    rows, ci = x.shape
    co = w.shape[0]
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    xp = np.zeros((rows + 4, ci))
    xp[2:2 + rows] = x
    dyp = np.zeros((rows + 4, co))
    dyp[2:2 + rows] = dy
    dx = np.zeros((rows, ci))
    dw = np.zeros((5, ci, co))
    for t in range(5):
        dx += dyp[4 - t:4 - t + rows] @ np.asarray(w[:, :, t], np.float64)
        dw[t] = xp[t:t + rows].T @ dy
    return dx, dw, dy.sum(axis=0)

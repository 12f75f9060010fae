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

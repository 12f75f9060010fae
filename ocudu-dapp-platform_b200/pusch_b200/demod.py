"""Equalisation and soft demapping on the B200: Python mirrors of
``ocudu::channel_equalizer`` (include/ocudu/phy/upper/equalization/channel_equalizer.h:47-76) and
``ocudu::demodulation_mapper`` (include/ocudu/phy/upper/channel_modulation/demodulation_mapper.h:48-51).
Complex bf16 inputs are carried as uint32 arrays (real part in the low 16 bits, the layout of
the reference's cbf16_t)."""
import ctypes

import numpy as np

from . import _native

ZF, MMSE = 0, 1


def to_cbf16(x):
    """complex64 array -> uint32 array of complex bf16 (round to nearest even, as
    include/ocudu/adt/bf16.h:23-40)."""
    x = np.ascontiguousarray(x, np.complex64)
    f = x.view(np.float32).reshape(x.shape + (2,))
    u = f.view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    nan = np.isnan(f)
    rounded = np.where(nan, (u >> 16) | 0x40, rounded) & 0xFFFF
    return (rounded[..., 0] | (rounded[..., 1] << 16)).astype(np.uint32)


def from_cbf16(u):
    u = np.asarray(u, np.uint32)
    re = (u << 16).view(np.float32)
    im = (u & 0xFFFF0000).view(np.float32)
    return (re + 1j * im).astype(np.complex64)


class ChannelEqualizer:
    def __init__(self, context: _native.Context, algorithm=MMSE):
        self.ctx = context
        self.algorithm = algorithm

    def is_supported(self, nof_ports, nof_layers):
        if nof_layers == 1:
            return nof_ports in (1, 2, 4, 8)
        if self.algorithm != MMSE:
            return False
        return (nof_layers == 2 and nof_ports in (2, 4, 8)) or (nof_layers == 4 and nof_ports in (4, 8))

    def equalize(self, ch_symbols, ch_estimates, noise_var_per_port, tx_scaling=1.0):
        """ch_symbols: uint32 cbf16 [port][re]; ch_estimates: uint32 cbf16 [port][layer][re].
        Returns (complex64 [re][layer], float32 [re][layer])."""
        y = np.ascontiguousarray(ch_symbols, np.uint32)
        h = np.ascontiguousarray(ch_estimates, np.uint32)
        nports, nre = y.shape
        nlayers = h.shape[1]
        nv = np.ascontiguousarray(noise_var_per_port, np.float32)
        eq = np.zeros((nre, nlayers), np.complex64)
        var = np.zeros((nre, nlayers), np.float32)
        rc = self.ctx.lib.pg_equalize_host(self.ctx.handle, self.algorithm, nre, nports, nlayers,
                                           y.ctypes.data_as(ctypes.c_void_p), h.ctypes.data_as(ctypes.c_void_p),
                                           nv.ctypes.data_as(ctypes.c_void_p), float(tx_scaling),
                                           eq.ctypes.data_as(ctypes.c_void_p), var.ctypes.data_as(ctypes.c_void_p))
        self.ctx.check(rc)
        return eq, var


class DemodulationMapper:
    def __init__(self, context: _native.Context):
        self.ctx = context

    def demodulate_soft(self, symbols, noise_vars, modulation_order):
        sym = np.ascontiguousarray(symbols, np.complex64)
        nv = np.ascontiguousarray(noise_vars, np.float32)
        out = np.zeros(sym.size * modulation_order, np.int8)
        rc = self.ctx.lib.pg_demodulate_soft_host(self.ctx.handle, modulation_order, sym.size,
                                                  sym.ctypes.data_as(ctypes.c_void_p),
                                                  nv.ctypes.data_as(ctypes.c_void_p),
                                                  out.ctypes.data_as(ctypes.c_void_p))
        self.ctx.check(rc)
        return out

"""UL-SCH receive stages on the B200: Python mirrors of the reference's interfaces.

* ``LdpcRateDematcher`` mirrors ``ocudu::ldpc_rate_dematcher``
  (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h:36-39), batched.
* ``CrcCalculatorBatch`` mirrors ``crc_calculator::calculate`` over many bit strings
  (include/ocudu/phy/upper/channel_coding/crc_calculator.h:67-77).
* ``segment`` mirrors the reference's segmentation quantities
  (include/ocudu/ran/sch/sch_segmentation.h, lib/phy/upper/channel_coding/ldpc/
  ldpc_segmenter_rx_impl.cpp:33-85).
* ``PuschDecoder`` mirrors ``ocudu::pusch_decoder`` for new transmissions
  (include/ocudu/phy/upper/channel_processors/pusch/pusch_decoder.h): codeword LLRs in,
  transport blocks and ``pusch_decoder_result``-like statistics out.
All compute runs on the GPU through the C ABI.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native
from ._native import PgCrcItem, PgRmCb, PgSchResult, PgSchSegmentation, PgSchTb


@dataclass
class RmConfig:
    """codeblock_metadata fields read by the rate dematcher."""
    base_graph: int
    lifting_size: int
    rv: int = 0
    modulation_order: int = 2
    nref: int = 0
    nof_filler_bits: int = 0


def segment(tbs_bits, base_graph, modulation_order, nof_layers, nof_ch_symbols):
    seg = PgSchSegmentation()
    rc = _native.load().pg_sch_segment(tbs_bits, base_graph, modulation_order, nof_layers, nof_ch_symbols,
                                       ctypes.byref(seg))
    if rc != _native.PG_OK:
        raise ValueError(f"invalid segmentation request (rc={rc})")
    return {name: int(getattr(seg, name)) for name, _ in PgSchSegmentation._fields_}


class LdpcRateDematcher:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def rate_dematch_batch(self, items: Sequence[tuple]):
        """items: (input LLRs [E], output buffer [N] (read when new_data is False), new_data, RmConfig).
        Output buffers are updated in place."""
        n = len(items)
        if n == 0:
            return
        descs = (PgRmCb * n)()
        in_off, out_off = 0, 0
        for i, (llrs, out, new_data, c) in enumerate(items):
            d = descs[i]
            d.in_offset, d.rm_length, d.out_offset, d.nref = in_off, llrs.size, out_off, c.nref
            d.lifting_size, d.nof_filler_bits = c.lifting_size, c.nof_filler_bits
            d.base_graph, d.rv, d.modulation_order, d.new_data = c.base_graph, c.rv, c.modulation_order, int(new_data)
            in_off += llrs.size
            out_off += out.size
        ins = np.concatenate([np.ascontiguousarray(x[0], np.int8) for x in items])
        outs = np.concatenate([np.ascontiguousarray(x[1], np.int8) for x in items])
        rc = self.lib.pg_rate_dematch_batch_host(self.ctx.handle, ctypes.addressof(descs), n,
                                                 ins.ctypes.data_as(ctypes.c_void_p), ins.size,
                                                 outs.ctypes.data_as(ctypes.c_void_p), outs.size)
        self.ctx.check(rc)
        for i, (_, out, _, _) in enumerate(items):
            out[:] = outs[descs[i].out_offset:descs[i].out_offset + out.size]

    def rate_dematch(self, output, input, new_data, cfg: RmConfig):
        self.rate_dematch_batch([(np.asarray(input, np.int8), output, new_data, cfg)])


class CrcCalculatorBatch:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def calculate(self, poly, bit_strings: Sequence[np.ndarray]) -> np.ndarray:
        """CRC remainders of unpacked bit arrays."""
        n = len(bit_strings)
        items = (PgCrcItem * max(n, 1))()
        chunks, off = [], 0
        for i, b in enumerate(bit_strings):
            b = np.asarray(b, np.uint8)
            pad = (-b.size) % 8
            items[i].bit_offset = off * 8
            items[i].nof_bits = b.size
            items[i].poly = poly
            packed = np.packbits(np.concatenate([b, np.zeros(pad, np.uint8)])) if b.size else np.zeros(0, np.uint8)
            chunks.append(packed)
            off += packed.size
        data = np.concatenate(chunks) if chunks else np.zeros(1, np.uint8)
        if data.size == 0:
            data = np.zeros(1, np.uint8)
        out = np.zeros(max(n, 1), np.uint32)
        rc = self.lib.pg_crc_calculate_host(self.ctx.handle, ctypes.addressof(items), n,
                                            data.ctypes.data_as(ctypes.c_void_p), data.size,
                                            out.ctypes.data_as(ctypes.c_void_p))
        self.ctx.check(rc)
        return out[:n]


@dataclass
class SchTransportBlock:
    """One UL-SCH codeword to decode (pusch_decoder::configuration + set_nof_softbits)."""
    llrs: np.ndarray          # G descrambled codeword LLRs (int8)
    tbs_bits: int
    base_graph: int
    modulation_order: int
    nof_layers: int
    rv: int = 0
    nref: int = 0
    max_iterations: int = 6


@dataclass
class SchResult:
    """pusch_decoder_result subset."""
    tb_crc_ok: bool
    nof_codeblocks_total: int
    nof_codeblocks_crc_ok: int
    mean_iterations: float
    max_iterations: int
    transport_block: Optional[np.ndarray]


class PuschDecoder:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def decode_batch(self, tbs: Sequence[SchTransportBlock]) -> List[SchResult]:
        n = len(tbs)
        if n == 0:
            return []
        descs = (PgSchTb * n)()
        off, out_off = 0, 0
        for i, t in enumerate(tbs):
            g = t.llrs.size
            qm = t.modulation_order
            if g % qm:
                raise ValueError("codeword length not a multiple of Qm")
            d = descs[i]
            d.llr_offset, d.nof_ch_symbols, d.tbs_bits, d.tb_out_offset, d.nref = off, g // qm, t.tbs_bits, out_off, t.nref
            d.base_graph, d.modulation_order, d.nof_layers, d.rv, d.max_iterations = (
                t.base_graph, qm, t.nof_layers, t.rv, t.max_iterations)
            off += g
            out_off += t.tbs_bits // 8
        llrs = np.concatenate([np.ascontiguousarray(t.llrs, np.int8) for t in tbs])
        out = np.zeros(max(out_off, 1), np.uint8)
        res = (PgSchResult * n)()
        rc = self.lib.pg_sch_decode_batch_host(self.ctx.handle, ctypes.addressof(descs), n,
                                               llrs.ctypes.data_as(ctypes.c_void_p), llrs.size,
                                               out.ctypes.data_as(ctypes.c_void_p), out.size,
                                               ctypes.addressof(res))
        self.ctx.check(rc)
        results = []
        for i, t in enumerate(tbs):
            r = res[i]
            o = descs[i].tb_out_offset
            results.append(SchResult(bool(r.tb_crc_ok), int(r.nof_cbs), int(r.nof_cbs_crc_ok),
                                     float(r.mean_iterations), int(r.max_iterations_run),
                                     out[o:o + t.tbs_bits // 8].copy() if r.tb_crc_ok else None))
        return results

    def decode_resident(self, tbs: Sequence[SchTransportBlock], offsets, llrs_ptr, nof_llrs, c_init=None,
                        bit_offset=None) -> List[SchResult]:
        """pg_sch_decode_batch_resident: the TBs' soft bits are already in device memory (llrs_ptr,
        TB i from offsets[i]; the llrs fields of `tbs` only give their lengths). c_init: per TB, the
        soft bits are still scrambled with that initialisation (from bit_offset[i], default 0)."""
        n = len(tbs)
        if n == 0:
            return []
        descs = (PgSchTb * n)()
        out_off = 0
        for i, t in enumerate(tbs):
            qm = t.modulation_order
            d = descs[i]
            d.llr_offset, d.nof_ch_symbols, d.tbs_bits, d.tb_out_offset, d.nref = (
                int(offsets[i]), t.llrs.size // qm, t.tbs_bits, out_off, t.nref)
            d.base_graph, d.modulation_order, d.nof_layers, d.rv, d.max_iterations = (
                t.base_graph, qm, t.nof_layers, t.rv, t.max_iterations)
            out_off += t.tbs_bits // 8
        ci = None if c_init is None else (ctypes.c_uint32 * n)(*[int(x) for x in c_init])
        bo = None if bit_offset is None else (ctypes.c_uint32 * n)(*[int(x) for x in bit_offset])
        out = np.zeros(max(out_off, 1), np.uint8)
        res = (PgSchResult * n)()
        self.ctx.check(self.lib.pg_sch_decode_batch_resident(self.ctx.handle, ctypes.addressof(descs), n, llrs_ptr,
                                                             nof_llrs, ci, bo, out.ctypes.data_as(ctypes.c_void_p),
                                                             out.size, ctypes.addressof(res)))
        results = []
        for i, t in enumerate(tbs):
            r = res[i]
            o = descs[i].tb_out_offset
            results.append(SchResult(bool(r.tb_crc_ok), int(r.nof_cbs), int(r.nof_cbs_crc_ok),
                                     float(r.mean_iterations), int(r.max_iterations_run),
                                     out[o:o + t.tbs_bits // 8].copy() if r.tb_crc_ok else None))
        return results

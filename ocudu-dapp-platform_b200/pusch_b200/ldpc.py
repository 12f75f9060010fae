"""LDPC decoding on the B200: Python mirror of the reference's decoder interfaces.

* ``LdpcDecoder`` mirrors ``ocudu::ldpc_decoder``
  (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h:19-58): ``decode(output, input,
  crc, cfg)`` returns the iteration count on success and ``None`` on failure, exactly like the
  reference's ``std::optional<unsigned>``; ``output`` receives the K*Z hard bits.
* ``LdpcBatchDecoder`` mirrors the batch entry
  ``pusch_resident_codeblock_decoder::decode_batch``
  (include/ocudu/phy/upper/channel_processors/pusch/pusch_resident_codeblock_decoder.h): many
  codeblocks with their own base graph, lifting size, fillers, CRC and iteration cap in one
  kernel launch.

Both run on the GPU through the C ABI (pg_ldpc_decode_batch_*); there is no CPU path.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native
from ._native import PG_CRC16, PG_CRC24A, PG_CRC24B, PG_CRC_NONE, PgLdpcCb

BG1, BG2 = 1, 2
LIFTING_SIZES = sorted({a * (1 << j) for a in (2, 3, 5, 7, 9, 11, 13, 15) for j in range(8) if a * (1 << j) <= 384})


def bg_k(bg):
    """Information variable nodes of the base graph (K_b)."""
    return 22 if bg == BG1 else 10


def bg_n_short(bg):
    """Variable nodes after shortening the 2 punctured systematic nodes."""
    return 66 if bg == BG1 else 50


class CrcCalculator:
    """Mirror of ocudu::crc_calculator's identity (crc_calculator.h:17-24): the decoder only needs
    the generator polynomial; the CRC itself runs inside the decoding kernel."""

    POLYS = {PG_CRC16: 0x11021, PG_CRC24A: 0x1864CFB, PG_CRC24B: 0x1800063}

    def __init__(self, poly):
        if poly not in self.POLYS:
            raise ValueError(f"unsupported CRC polynomial {poly}")
        self.poly = poly

    def get_generator_poly(self):
        return self.POLYS[self.poly]


@dataclass
class LdpcDecoderConfiguration:
    """ldpc_decoder::configuration (ldpc_decoder.h:26-38)."""
    base_graph: int = BG1
    lifting_size: int = 2
    nof_filler_bits: int = 0
    nof_crc_bits: int = 16
    max_iterations: int = 6


@dataclass
class CodeblockJob:
    """One codeblock of a batch: its rate-dematched LLRs and configuration."""
    llrs: np.ndarray
    cfg: LdpcDecoderConfiguration
    crc_poly: int = PG_CRC24B


def output_bytes(bg, z):
    return (bg_k(bg) * z + 7) // 8


def make_descriptors(jobs: Sequence[CodeblockJob]):
    """Packs jobs into (descriptor array, concatenated LLRs, total output bytes)."""
    n = len(jobs)
    descs = (PgLdpcCb * max(n, 1))()
    llr_off = 0
    out_off = 0
    for i, j in enumerate(jobs):
        d = descs[i]
        d.llr_offset = llr_off
        d.nof_llrs = int(j.llrs.size)
        d.out_offset = out_off
        d.lifting_size = j.cfg.lifting_size
        d.nof_filler_bits = j.cfg.nof_filler_bits
        d.base_graph = j.cfg.base_graph
        d.crc_poly = j.crc_poly
        d.max_iterations = j.cfg.max_iterations
        llr_off += int(j.llrs.size)
        out_off += output_bytes(j.cfg.base_graph, j.cfg.lifting_size)
    llrs = np.concatenate([np.ascontiguousarray(j.llrs, dtype=np.int8) for j in jobs]) if n else np.zeros(1, np.int8)
    return descs, llrs, out_off


class LdpcBatchDecoder:
    """Batched decoder (pusch_resident_codeblock_decoder::decode_batch)."""

    def __init__(self, device=0, max_codeblocks=1024, context: Optional[_native.Context] = None):
        self.ctx = context or _native.Context(device=device, max_codeblocks=max_codeblocks)
        self.lib = self.ctx.lib

    def decode_batch(self, jobs: Sequence[CodeblockJob]):
        """Decodes host-resident codeblocks. Returns (list of packed-bit arrays, iterations array)
        where iterations[i] == 0 means failure (the reference's empty optional)."""
        n = len(jobs)
        if n == 0:
            return [], np.zeros(0, np.int32)
        descs, llrs, out_bytes = make_descriptors(jobs)
        bits = np.zeros(max(out_bytes, 1), np.uint8)
        iters = np.zeros(n, np.int32)
        rc = self.lib.pg_ldpc_decode_batch_host(self.ctx.handle, ctypes.addressof(descs), n,
                                                llrs.ctypes.data_as(ctypes.c_void_p), llrs.size,
                                                bits.ctypes.data_as(ctypes.c_void_p), bits.size,
                                                iters.ctypes.data_as(ctypes.c_void_p))
        self.ctx.check(rc)
        outs = []
        for i in range(n):
            off = descs[i].out_offset
            outs.append(bits[off:off + output_bytes(jobs[i].cfg.base_graph, jobs[i].cfg.lifting_size)].copy())
        return outs, iters

    def decode_device(self, descs, n, llrs_ptr, bits_ptr, iters_ptr, stream_ptr=0):
        """Enqueues a decode of device-resident buffers (raw device pointers) on a CUDA stream;
        descriptors are host-side (staged by the library)."""
        rc = self.lib.pg_ldpc_decode_batch_device(self.ctx.handle, ctypes.addressof(descs), n, llrs_ptr, bits_ptr,
                                                  iters_ptr, stream_ptr)
        self.ctx.check(rc)

    def decode_resident(self, descs_ptr, n, llrs_ptr, bits_ptr, iters_ptr, stream_ptr=0):
        """Enqueues a decode whose descriptors are already in device memory."""
        rc = self.lib.pg_ldpc_decode_batch_resident(self.ctx.handle, descs_ptr, n, llrs_ptr, bits_ptr, iters_ptr,
                                                    stream_ptr)
        self.ctx.check(rc)

    def set_kernel(self, kernel: int):
        """Selects the decoding kernel (_native.PG_LDPC_KERNEL_*); results do not depend on it."""
        self.ctx.check(self.lib.pg_set_ldpc_kernel(self.ctx.handle, int(kernel)))

    def set_order(self, mode: int):
        """Work order of the batch decodes (_native.PG_LDPC_ORDER_*); results do not depend on it."""
        self.ctx.check(self.lib.pg_set_ldpc_order(self.ctx.handle, int(mode)))

    def set_ctas_per_sm(self, ctas_per_sm: int):
        """Resident CTAs per SM of the batch decodes (0: the kernel's limit); results do not depend on it."""
        self.ctx.check(self.lib.pg_set_ldpc_ctas_per_sm(self.ctx.handle, int(ctas_per_sm)))

    def set_kernel_timing(self, enabled: bool):
        self.ctx.check(self.lib.pg_set_kernel_timing(self.ctx.handle, int(enabled)))

    def last_kernel_ms(self) -> float:
        return float(self.lib.pg_last_kernel_ms(self.ctx.handle))


class LdpcDecoder:
    """Single-codeblock decoder with the reference's ldpc_decoder::decode contract."""

    def __init__(self, device=0, batch: Optional[LdpcBatchDecoder] = None):
        self.batch = batch or LdpcBatchDecoder(device=device, max_codeblocks=64)

    def decode(self, output: np.ndarray, input: np.ndarray, crc: Optional[CrcCalculator],
               cfg: LdpcDecoderConfiguration) -> Optional[int]:
        """output: uint8 array of ceil(K*Z/8) bytes (packed MSB first), written in place."""
        poly = PG_CRC_NONE if crc is None else crc.poly
        if crc is not None and cfg.nof_crc_bits not in (16, 24):
            raise ValueError("nof_crc_bits must be 16 or 24")
        outs, iters = self.batch.decode_batch([CodeblockJob(np.asarray(input, np.int8), cfg, poly)])
        output[:outs[0].size] = outs[0]
        return int(iters[0]) if iters[0] > 0 else None

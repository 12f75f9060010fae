"""UCI on PUSCH: UL-SCH demultiplexing of HARQ-ACK and CSI Part 1 and short-block detection,
mirroring the reference's ulsch_demultiplex
(include/ocudu/phy/upper/channel_processors/pusch/ulsch_demultiplex.h:31-90) and
short_block_detector (include/ocudu/phy/upper/channel_coding/short/short_block_detector.h) over
the library's GPU entries."""
import ctypes
from typing import List, Sequence, Tuple

import numpy as np

from . import _native
from ._native import PgUciShortBlock, PgUlschDemuxConfig

CONFIG_FIELDS = [f for f, _ in PgUlschDemuxConfig._fields_]


def make_config(**fields) -> PgUlschDemuxConfig:
    """A pg_ulsch_demux_config from keyword fields (missing ones are zero)."""
    c = PgUlschDemuxConfig()
    for k, v in fields.items():
        if k not in CONFIG_FIELDS:
            raise KeyError(k)
        setattr(c, k, int(v))
    return c


class UlschDemultiplexer:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def sizes(self, cfg: PgUlschDemuxConfig) -> Tuple[int, int, int]:
        """Soft bits of the UL-SCH, HARQ-ACK and CSI Part 1 streams (host computation)."""
        out = (ctypes.c_uint32 * 3)()
        rc = self.lib.pg_ulsch_demultiplex_sizes(ctypes.byref(cfg), out)
        if rc:
            raise _native.PgError(rc, "inconsistent or unsupported UL-SCH demultiplexing configuration")
        return tuple(int(x) for x in out)

    def demultiplex_device(self, cfgs: Sequence[PgUlschDemuxConfig], llrs_ptr, sch_ptr, ack_ptr, csi_ptr,
                           stream_ptr=0):
        arr = (PgUlschDemuxConfig * max(1, len(cfgs)))(*cfgs)
        self.ctx.check(self.lib.pg_ulsch_demultiplex_device(self.ctx.handle, ctypes.addressof(arr), len(cfgs),
                                                            llrs_ptr, sch_ptr, ack_ptr, csi_ptr, stream_ptr))

    def demultiplex(self, cfgs: Sequence[PgUlschDemuxConfig], llrs: Sequence[np.ndarray]):
        """Host soft bits in, [(sch, harq_ack, csi_part1)] out (offsets are assigned here)."""
        import torch
        cfgs = [PgUlschDemuxConfig.from_buffer_copy(c) for c in cfgs]
        off_in, offs, spans = 0, [0, 0, 0], []
        for c, x in zip(cfgs, llrs):
            s = self.sizes(c)
            c.llr_offset = off_in
            c.sch_offset, c.harq_ack_offset, c.csi_part1_offset = offs
            spans.append([(offs[k], s[k]) for k in range(3)])
            off_in += int(np.asarray(x).size)
            offs = [offs[k] + s[k] for k in range(3)]
        d_in = torch.from_numpy(np.ascontiguousarray(np.concatenate(llrs), dtype=np.int8)).cuda()
        outs = [torch.zeros(max(1, offs[k]), dtype=torch.int8, device="cuda") for k in range(3)]
        st = torch.cuda.current_stream()
        self.demultiplex_device(cfgs, d_in.data_ptr(), outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                st.cuda_stream)
        st.synchronize()
        host = [o.cpu().numpy() for o in outs]
        return [tuple(host[k][o:o + n] for k, (o, n) in enumerate(sp)) for sp in spans]


class ShortBlockDetector:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def detect(self, messages: Sequence[Tuple[int, int, np.ndarray]]) -> List[Tuple[np.ndarray, bool]]:
        """messages: (nof_bits, modulation_order, soft bits); returns (bits, valid) per message."""
        import torch
        n = len(messages)
        if n == 0:
            return []
        items = (PgUciShortBlock * n)()
        off, out_off = 0, 0
        for i, (K, qm, llr) in enumerate(messages):
            items[i].llr_offset, items[i].nof_llrs, items[i].out_offset = off, int(np.asarray(llr).size), out_off
            items[i].nof_bits, items[i].modulation_order = K, qm
            off += int(np.asarray(llr).size)
            out_off += K
        d_in = torch.from_numpy(np.ascontiguousarray(np.concatenate([m[2] for m in messages]), dtype=np.int8)).cuda()
        d_bits = torch.zeros(out_off, dtype=torch.uint8, device="cuda")
        d_valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
        st = torch.cuda.current_stream()
        self.ctx.check(self.lib.pg_uci_short_block_detect_device(self.ctx.handle, ctypes.addressof(items), n,
                                                                 d_in.data_ptr(), d_bits.data_ptr(),
                                                                 d_valid.data_ptr(), st.cuda_stream))
        st.synchronize()
        bits, valid = d_bits.cpu().numpy(), d_valid.cpu().numpy()
        out, o = [], 0
        for i, (K, _, _) in enumerate(messages):
            out.append((bits[o:o + K].copy(), bool(valid[i])))
            o += K
        return out


class PolarUciDecoder:
    """Polar-coded UCI messages of 12 to 1706 bits (pg_uci_polar_decode_device): the reference's
    uci_decoder::decode above 11 bits (lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:25-111)."""

    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def decode(self, messages: Sequence[Tuple[int, np.ndarray]]) -> List[Tuple[np.ndarray, bool]]:
        """messages: (nof_bits, soft bits); returns (bits, valid) per message."""
        import torch
        n = len(messages)
        if n == 0:
            return []
        items = (_native.PgUciPolar * n)()
        off, out_off = 0, 0
        for i, (A, llr) in enumerate(messages):
            items[i].llr_offset, items[i].nof_llrs, items[i].out_offset = off, int(np.asarray(llr).size), out_off
            items[i].nof_bits = A
            off += int(np.asarray(llr).size)
            out_off += A
        d_in = torch.from_numpy(np.ascontiguousarray(np.concatenate([m[1] for m in messages]), dtype=np.int8)).cuda()
        d_bits = torch.zeros(out_off, dtype=torch.uint8, device="cuda")
        d_valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
        st = torch.cuda.current_stream()
        self.ctx.check(self.lib.pg_uci_polar_decode_device(self.ctx.handle, ctypes.addressof(items), n,
                                                           d_in.data_ptr(), d_bits.data_ptr(), d_valid.data_ptr(),
                                                           st.cuda_stream))
        st.synchronize()
        bits, valid = d_bits.cpu().numpy(), d_valid.cpu().numpy()
        out, o = [], 0
        for i, (A, _) in enumerate(messages):
            out.append((bits[o:o + A].copy(), bool(valid[i])))
            o += A
        return out


def polar_code(K, E):
    """The polar code pg_uci_polar_decode_device builds for one codeblock (pg_polar_code; host only):
    dict with n, N, nPC, nWmPC, k_set (0/1 per sub-channel), pc_set and subblock (N entries), or
    None when the reference's polar_code_impl rejects (K, E)."""
    info = _native.PgPolarCodeInfo()
    if _native.load().pg_polar_code(K, E, ctypes.byref(info)) != 0:
        return None
    N = info.N
    kset = np.array([(info.k_set[i >> 5] >> (i & 31)) & 1 for i in range(N)], np.uint8)
    return dict(n=info.n, N=N, nPC=info.nPC, nWmPC=info.nWmPC, k_set=kset, pc_set=list(info.pc_set),
                subblock=np.array(info.subblock[:N], np.uint16))


def ulsch_information(tbs_bits, base_graph, modulation_order, nof_layers, nof_rb, start_symbol, nof_symbols,
                      dmrs_symbol_mask, nof_harq_ack_bits=0, nof_csi_part1_bits=0, nof_csi_part2_bits=0,
                      alpha_scaling=1.0, beta_offset_harq_ack=20.0, beta_offset_csi_part1=6.25,
                      beta_offset_csi_part2=6.25, nof_cdm_groups_without_data=2, target_code_rate=0.5,
                      contains_dc=False) -> dict:
    """pg_ulsch_information: the encoded soft-bit counts of UCI multiplexed on a PUSCH (the
    reference's get_ulsch_information, include/ocudu/ran/pusch/ulsch_info.h:144)."""
    from ._native import PgUlschInfo, PgUlschInfoConfig
    c = PgUlschInfoConfig()
    c.tbs_bits, c.target_code_rate, c.alpha_scaling = tbs_bits, target_code_rate, alpha_scaling
    c.beta_offset_harq_ack, c.beta_offset_csi_part1, c.beta_offset_csi_part2 = (
        beta_offset_harq_ack, beta_offset_csi_part1, beta_offset_csi_part2)
    c.nof_harq_ack_bits, c.nof_csi_part1_bits, c.nof_csi_part2_bits = (
        nof_harq_ack_bits, nof_csi_part1_bits, nof_csi_part2_bits)
    c.nof_rb, c.dmrs_symbol_mask, c.base_graph = nof_rb, dmrs_symbol_mask, base_graph
    c.modulation_order, c.nof_layers, c.start_symbol, c.nof_symbols = (
        modulation_order, nof_layers, start_symbol, nof_symbols)
    c.nof_cdm_groups_without_data, c.contains_dc = nof_cdm_groups_without_data, int(bool(contains_dc))
    out = PgUlschInfo()
    rc = _native.load().pg_ulsch_information(ctypes.byref(c), ctypes.byref(out))
    if rc:
        raise _native.PgError(rc, "invalid UL-SCH information request")
    return {n: int(getattr(out, n)) for n, _ in PgUlschInfo._fields_}

"""PUSCH slot processing on the B200: Python mirror of ``ocudu::pusch_processor::process``
(include/ocudu/phy/upper/channel_processors/pusch/pusch_processor.h:199-203) for batches of UEs,
and access to the individual stages (DM-RS channel estimation, demodulation) on device buffers.
All compute runs on the GPU through the C ABI; torch tensors are only device-memory plumbing."""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native
from ._native import PgPuschPlanInfo, PgSchResult
from .sim import PuschSlot, PuschUe, nof_ch_symbols


class PgPuschUe(ctypes.Structure):
    _fields_ = [("grid_offset", ctypes.c_uint32), ("grid_nof_subc", ctypes.c_uint32), ("llr_offset", ctypes.c_uint32),
                ("est_offset", ctypes.c_uint32), ("tbs_bits", ctypes.c_uint32), ("tb_out_offset", ctypes.c_uint32),
                ("nref", ctypes.c_uint32), ("dmrs_scaling", ctypes.c_float), ("rb_start", ctypes.c_uint16),
                ("nof_rb", ctypes.c_uint16), ("dmrs_symbol_mask", ctypes.c_uint16), ("n_id", ctypes.c_uint16),
                ("rnti", ctypes.c_uint16), ("n_id_data", ctypes.c_uint16), ("dc_subcarrier", ctypes.c_int16),
                ("slot", ctypes.c_uint8), ("n_scid", ctypes.c_uint8), ("first_symbol", ctypes.c_uint8),
                ("nof_symbols", ctypes.c_uint8), ("nof_rx_ports", ctypes.c_uint8), ("nof_layers", ctypes.c_uint8),
                ("modulation_order", ctypes.c_uint8), ("base_graph", ctypes.c_uint8), ("rv", ctypes.c_uint8),
                ("max_iterations", ctypes.c_uint8)]


class PgPortResult(ctypes.Structure):
    _fields_ = [("noise_var", ctypes.c_float), ("epre", ctypes.c_float), ("snr", ctypes.c_float),
                ("rsrp", ctypes.c_float * 2)]


def make_ue_descriptors(slot: PuschSlot, max_iterations=6, grid_offset=0, dc_subcarrier=-1, tb_offset=0):
    """pg_pusch_ue array for the UEs of one simulated slot (grid at grid_offset words)."""
    n = len(slot.ues)
    arr = (PgPuschUe * n)()
    llr, est, tbo = 0, 0, tb_offset
    for i, ue in enumerate(slot.ues):
        d = arr[i]
        d.grid_offset = grid_offset
        d.grid_nof_subc = 12 * slot.nof_prb_grid
        d.llr_offset = llr
        d.est_offset = est
        d.tbs_bits = ue.tbs_bits
        d.tb_out_offset = tbo
        d.nref = 0
        d.dmrs_scaling = slot.dmrs_scaling
        d.rb_start, d.nof_rb = ue.rb_start, ue.nof_rb
        d.dmrs_symbol_mask = sum(1 << s for s in ue.dmrs_symbols)
        d.n_id, d.rnti, d.n_id_data = ue.n_id, ue.rnti, ue.n_id_data
        d.dc_subcarrier = dc_subcarrier
        d.slot, d.n_scid, d.first_symbol, d.nof_symbols = slot.slot, 0, ue.first_symbol, ue.nof_symbols
        d.nof_rx_ports, d.nof_layers, d.modulation_order = slot.nof_ports, ue.nof_layers, ue.modulation_order
        d.base_graph, d.rv, d.max_iterations = ue.base_graph, ue.rv, max_iterations
        llr += nof_ch_symbols(ue) * ue.modulation_order
        est += slot.nof_ports * len(ue.dmrs_symbols) * ue.nof_layers * 12 * ue.nof_rb
        tbo += ue.tbs_bits // 8
    return arr, llr, est, tbo


@dataclass
class PuschResult:
    tb_crc_ok: bool
    transport_block: Optional[np.ndarray]
    nof_codeblocks: int
    nof_codeblocks_crc_ok: int
    mean_iterations: float
    noise_var: np.ndarray
    rsrp: np.ndarray
    snr: np.ndarray


class PuschProcessor:
    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = _native.load()

    def process_slots(self, slots: Sequence[PuschSlot], max_iterations=6, dc_subcarrier=-1) -> List[PuschResult]:
        """Decodes every UE of every slot (one cell per slot) in one batched call."""
        descs, grids, off_words, tb_off, ue_list = [], [], 0, 0, []
        for sl in slots:
            arr, _, _, tbo = make_ue_descriptors(sl, max_iterations, off_words, dc_subcarrier, tb_off)
            descs.extend(arr[i] for i in range(len(sl.ues)))
            grids.append(np.ascontiguousarray(sl.grid, np.uint32).ravel())
            off_words += grids[-1].size
            tb_off = tbo
            ue_list.extend(sl.ues)
        n = len(descs)
        arr = (PgPuschUe * n)(*descs)
        grid = np.concatenate(grids)
        tb = np.zeros(max(tb_off, 1), np.uint8)
        pr = (PgPortResult * (4 * n))()
        res = (PgSchResult * n)()
        rc = self.lib.pg_pusch_process_host(self.ctx.handle, ctypes.addressof(arr), n,
                                            grid.ctypes.data_as(ctypes.c_void_p), grid.size,
                                            tb.ctypes.data_as(ctypes.c_void_p), tb.size, ctypes.addressof(pr),
                                            ctypes.addressof(res))
        self.ctx.check(rc)
        out = []
        for i in range(n):
            r = res[i]
            p = [pr[4 * i + k] for k in range(descs[i].nof_rx_ports)]
            o = descs[i].tb_out_offset
            out.append(PuschResult(bool(r.tb_crc_ok),
                                   tb[o:o + descs[i].tbs_bits // 8].copy() if r.tb_crc_ok else None,
                                   int(r.nof_cbs), int(r.nof_cbs_crc_ok), float(r.mean_iterations),
                                   np.array([q.noise_var for q in p]), np.array([[q.rsrp[0], q.rsrp[1]] for q in p]),
                                   np.array([q.snr for q in p])))
        return out


@dataclass
class PortEstimate:
    """port_channel_estimator_results of one receive port."""
    freq_response: np.ndarray      # complex64 [dmrs symbol][layer][12 nof_rb], FP32
    symbol_estimates: np.ndarray   # uint32 cbf16 [14][layer][12 nof_rb]
    noise_var: float
    epre: float
    snr: float
    rsrp: np.ndarray
    cfo_hz: Optional[float]
    time_alignment_s: float


class PortChannelEstimator:
    """Mirror of ``port_channel_estimator::compute`` (port_channel_estimator.h:86-89) for one port,
    FD "filter", TD "interpolate": the caller gives that port's grid and the DM-RS pilots."""

    def __init__(self, context: _native.Context):
        self.ctx = context
        self.lib = context.lib

    def compute(self, grid_port, pilots, rb_start, nof_rb, dmrs_symbols, scaling, first_symbol=0, nof_symbols=14,
                scs_khz=30) -> PortEstimate:
        """grid_port: uint32 cbf16 [14][nsubc]; pilots: complex64 [dmrs symbol][layer][6 nof_rb]."""
        g = np.ascontiguousarray(grid_port, np.uint32)
        pil = np.ascontiguousarray(pilots, np.complex64)
        nd, nl = pil.shape[0], pil.shape[1]
        cfg = _native.PgPortEstimateCfg()
        cfg.grid_nof_subc, cfg.scaling, cfg.rb_start, cfg.nof_rb = g.shape[1], scaling, rb_start, nof_rb
        cfg.dmrs_symbol_mask = sum(1 << s for s in dmrs_symbols)
        cfg.first_symbol, cfg.nof_symbols, cfg.nof_layers, cfg.scs_khz = first_symbol, nof_symbols, nl, scs_khz
        freq = np.zeros((nd, nl, 12 * nof_rb), np.complex64)
        sym = np.zeros((14, nl, 12 * nof_rb), np.uint32)
        res = _native.PgPortEstimateResult()
        self.ctx.check(self.lib.pg_port_channel_estimate_host(
            self.ctx.handle, ctypes.byref(cfg), g.ctypes.data_as(ctypes.c_void_p), pil.ctypes.data_as(ctypes.c_void_p),
            freq.ctypes.data_as(ctypes.c_void_p), sym.ctypes.data_as(ctypes.c_void_p), ctypes.byref(res)))
        cfo = None if np.isnan(res.cfo_hz) else float(res.cfo_hz)
        return PortEstimate(freq, sym, float(res.noise_var), float(res.epre), float(res.snr),
                            np.array(res.rsrp[:nl], np.float64), cfo, float(res.time_alignment_s))


def batch_descriptors(slots: Sequence[PuschSlot], max_iterations=6, dc_subcarrier=-1):
    """pg_pusch_ue array of every UE of every slot (one cell per slot), grids concatenated in slot
    order, TBs packed back to back. Returns (descriptors, grid words, TB bytes, UE list)."""
    descs, grids, off_words, tb_off, ue_list = [], [], 0, 0, []
    for sl in slots:
        arr, _, _, tbo = make_ue_descriptors(sl, max_iterations, off_words, dc_subcarrier, tb_off)
        descs.extend(arr[i] for i in range(len(sl.ues)))
        grids.append(np.ascontiguousarray(sl.grid, np.uint32).ravel())
        off_words += grids[-1].size
        tb_off = tbo
        ue_list.extend(sl.ues)
    arr = (PgPuschUe * len(descs))(*descs)
    return arr, np.concatenate(grids), tb_off, ue_list


class PuschSlotPlan:
    """A pg_pusch_plan: the PDUs of one slot batch prepared once (segmentation, work lists,
    workspace, descrambling sequences) and executed per slot - the batched form of
    pusch_processor::process (pusch_processor.h:199-203)."""

    def __init__(self, context: _native.Context, slots: Sequence[PuschSlot], max_iterations=6, dc_subcarrier=-1,
                 graph=False, uci=None):
        """uci: None, or one _native.PgPuschUci per UE (UCI multiplexed on the UE's PUSCH; all-zero
        entries carry none)."""
        self.ctx = context
        self.lib = _native.load()
        self.descs, self.grid, self.tb_bytes, self.ues = batch_descriptors(slots, max_iterations, dc_subcarrier)
        self.n = len(self.ues)
        h = ctypes.c_void_p()
        if uci is None:
            self.ctx.check(self.lib.pg_pusch_plan_create(self.ctx.handle, ctypes.addressof(self.descs), self.n,
                                                         self.grid.size, ctypes.byref(h)))
        else:
            arr = (_native.PgPuschUci * self.n)(*uci)
            self.ctx.check(self.lib.pg_pusch_plan_create_uci(self.ctx.handle, ctypes.addressof(self.descs),
                                                             ctypes.addressof(arr), self.n, self.grid.size,
                                                             ctypes.byref(h)))
        self.handle = h
        info = PgPuschPlanInfo()
        self.ctx.check(self.lib.pg_pusch_plan_info(self.handle, ctypes.byref(info)))
        self.info = info
        self.set_graph(graph)

    def set_graph(self, enabled: bool):
        self.ctx.check(self.lib.pg_pusch_plan_set_graph(self.handle, int(bool(enabled))))

    def uci_results(self):
        """UCI of the last execution per UE: (harq_ack bits, valid, csi_part1 bits, valid), the bit
        arrays of each message's length (empty when the UE carries no such field)."""
        res = (_native.PgPuschUciResult * self.n)()
        self.ctx.check(self.lib.pg_pusch_plan_uci_results(self.handle, ctypes.addressof(res)))
        return res

    def uci_message(self, ue, field, nbits):
        """One UCI message of the last execution (field 0 HARQ-ACK, 1 CSI Part 1; any size, polar-coded
        ones included): (bits, valid)."""
        import numpy as np
        buf = np.zeros(max(1, nbits), np.uint8)
        valid = ctypes.c_uint8(0)
        self.ctx.check(self.lib.pg_pusch_plan_uci_message(self.handle, ue, field, buf.ctypes.data_as(ctypes.c_void_p),
                                                          buf.size, ctypes.byref(valid)))
        return buf[:nbits].copy(), bool(valid.value)

    def set_learned(self, net, use=None):
        """Refines the channel estimates with a LearnedEstimator (None: the plain estimator only)
        for the UEs with use[u] true (all when use is None)."""
        u = None if use is None else (ctypes.c_uint8 * self.n)(*[int(bool(v)) for v in use])
        self.ctx.check(self.lib.pg_pusch_plan_set_learned(self.handle, net.handle if net is not None else None, u))

    def set_harq(self, new_data=None, rv=None):
        """HARQ: for UEs with new_data[u] false the next execution soft-combines into the codeblock
        buffers the plan kept from the previous one, with redundancy version rv[u]."""
        nd = None if new_data is None else (ctypes.c_uint8 * self.n)(*[int(bool(v)) for v in new_data])
        r = None if rv is None else (ctypes.c_uint8 * self.n)(*[int(v) for v in rv])
        self.ctx.check(self.lib.pg_pusch_plan_set_harq(self.handle, nd, r))

    def tuning(self):
        t = _native.PgPuschPlanTuning()
        self.ctx.check(self.lib.pg_pusch_plan_get_tuning(self.handle, ctypes.byref(t)))
        return t

    def set_tuning(self, t):
        self.ctx.check(self.lib.pg_pusch_plan_set_tuning(self.handle, ctypes.byref(t)))

    def autotune(self, grid_ptr, reps=5):
        """Picks the fastest launch shapes for this plan's slot (pg_pusch_plan_autotune); returns
        (PgPuschPlanTuning, best ms)."""
        t = _native.PgPuschPlanTuning()
        ms = ctypes.c_float()
        self.ctx.check(self.lib.pg_pusch_plan_autotune(self.handle, grid_ptr, reps, ctypes.byref(t), ctypes.byref(ms)))
        return t, ms.value

    def le_rows(self, use=None):
        """Rows a LearnedEstimator needs for this plan."""
        if use is None:
            return int(self.lib.pg_le_rows(ctypes.addressof(self.descs), self.n))
        sel = [self.descs[i] for i in range(self.n) if use[i]]
        arr = (PgPuschUe * len(sel))(*sel)
        return int(self.lib.pg_le_rows(ctypes.addressof(arr), len(sel))) if sel else 0

    def execute_device(self, grid_ptr, tb_ptr, results_ptr, port_results_ptr=None, stream_ptr=0):
        self.ctx.check(self.lib.pg_pusch_plan_execute_device(self.handle, grid_ptr, tb_ptr, results_ptr,
                                                             port_results_ptr, stream_ptr))

    def execute_host(self, grid: Optional[np.ndarray] = None, with_port_results=True) -> List[PuschResult]:
        grid = self.grid if grid is None else grid
        tb = np.zeros(max(self.tb_bytes, 1), np.uint8)
        res = (PgSchResult * self.n)()
        pr = (PgPortResult * (4 * self.n))() if with_port_results else None
        self.ctx.check(self.lib.pg_pusch_plan_execute_host(self.handle, grid.ctypes.data_as(ctypes.c_void_p),
                                                           tb.ctypes.data_as(ctypes.c_void_p), tb.size,
                                                           ctypes.addressof(res),
                                                           ctypes.addressof(pr) if pr is not None else None))
        return results_from(self.descs, res, pr, tb)

    def submit_host(self, grid: np.ndarray):
        """Pipelined execution: enqueues one slot (pg_pusch_plan_submit_host). The grid array must stay
        alive and unchanged until the matching collect_host returns."""
        grid = np.ascontiguousarray(grid, dtype=np.uint32)
        self._inflight = getattr(self, "_inflight", []) + [grid]
        self.ctx.check(self.lib.pg_pusch_plan_submit_host(self.handle, grid.ctypes.data_as(ctypes.c_void_p)))

    def collect_host(self, with_port_results=True) -> List[PuschResult]:
        """Results of the oldest submitted slot (pg_pusch_plan_collect_host)."""
        tb = np.zeros(max(self.tb_bytes, 1), np.uint8)
        res = (PgSchResult * self.n)()
        pr = (PgPortResult * (4 * self.n))() if with_port_results else None
        self.ctx.check(self.lib.pg_pusch_plan_collect_host(self.handle, tb.ctypes.data_as(ctypes.c_void_p), tb.size,
                                                           ctypes.addressof(res),
                                                           ctypes.addressof(pr) if pr is not None else None))
        self._inflight = self._inflight[1:]
        return results_from(self.descs, res, pr, tb)

    def execute_host_bfp(self, compressed: np.ndarray, data_width: int, with_port_results=True) -> List[PuschResult]:
        """execute_host with the grids as O-RAN BFP-compressed PRBs (pg_pusch_plan_execute_host_bfp)."""
        compressed = np.ascontiguousarray(compressed, dtype=np.uint8)
        n = self.n
        res = (PgSchResult * n)()
        pr = (PgPortResult * (4 * n))() if with_port_results else None
        tb = np.zeros(max(self.tb_bytes, 1), np.uint8)
        self.ctx.check(self.lib.pg_pusch_plan_execute_host_bfp(
            self.handle, compressed.ctypes.data_as(ctypes.c_void_p), compressed.size, data_width,
            tb.ctypes.data_as(ctypes.c_void_p), tb.size, ctypes.addressof(res),
            ctypes.addressof(pr) if pr is not None else None))
        return results_from(self.descs, res, pr, tb)

    def close(self):
        # A plan outlived by its context (closed first, e.g. at interpreter exit) is not destroyed:
        # the plan refers to the context's stream.
        if getattr(self, "handle", None) and getattr(self.ctx, "handle", None):
            self.lib.pg_pusch_plan_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def results_from(descs, res, pr, tb) -> List[PuschResult]:
    out = []
    for i in range(len(descs)):
        r = res[i]
        p = [pr[4 * i + k] for k in range(descs[i].nof_rx_ports)] if pr is not None else []
        o = descs[i].tb_out_offset
        out.append(PuschResult(bool(r.tb_crc_ok), tb[o:o + descs[i].tbs_bits // 8].copy() if r.tb_crc_ok else None,
                               int(r.nof_cbs), int(r.nof_cbs_crc_ok), float(r.mean_iterations),
                               np.array([q.noise_var for q in p]), np.array([[q.rsrp[0], q.rsrp[1]] for q in p]),
                               np.array([q.snr for q in p])))
    return out

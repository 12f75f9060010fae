"""Seeded synthetic workloads (the project's own simulator; inputs only, never the measured path).

``ldpc_batch``: the LDPC decoder batch workload - codeblocks of random bits with CRC24B attached,
LDPC-encoded (this project's encoder, pusch_b200.codec), BPSK over AWGN at an Eb/N0 drawn per
codeblock, and LLRs 2y/sigma^2 scaled by ``llr_scale`` (LLR units per LSB = 1/llr_scale),
rounded and saturated to int8 +-127. The code rate used for Eb/N0 is R = K/N (CRC included).
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import codec
from .ldpc import BG1, BG2, CodeblockJob, LdpcDecoderConfiguration, bg_k, bg_n_short
from ._native import PG_CRC24B


@dataclass
class LdpcBatch:
    jobs: List[CodeblockJob]
    truth: List[np.ndarray]          # K_b*Z transmitted message bits per codeblock (unpacked)
    ebn0_db: np.ndarray
    base_graphs: np.ndarray
    info_bits: np.ndarray            # information bits per codeblock (K - F - 24)
    params: dict = field(default_factory=dict)


def ldpc_batch(seed=0, n=512, z=384, ebn0_range=(1.0, 3.0), llr_scale=4.0, max_iterations=10, bg_mix=0.5,
               bgs=None):
    """Codeblocks of BG1 (E = N = 66Z, rate 1/3) or BG2 (E = N = 50Z, rate 1/5) mixed by seed."""
    rng = np.random.default_rng(seed)
    if bgs is None:
        bgs = np.where(rng.random(n) < bg_mix, BG1, BG2).astype(np.int32)
    ebn0 = rng.uniform(ebn0_range[0], ebn0_range[1], n)
    jobs, truth = [None] * n, [None] * n
    info = np.zeros(n, np.int64)
    for bg in (BG1, BG2):
        idx = np.nonzero(bgs == bg)[0]
        if idx.size == 0:
            continue
        k = bg_k(bg) * z
        nn = bg_n_short(bg) * z
        msg = codec.attach_crc(PG_CRC24B, rng.integers(0, 2, (idx.size, k - 24), dtype=np.uint8))
        cw = codec.ldpc_encode(bg, z, msg)
        rate = k / nn
        sigma = np.sqrt(1.0 / (2.0 * rate * 10.0 ** (ebn0[idx] / 10.0)))
        y = (1.0 - 2.0 * cw.astype(np.float32)) + sigma[:, None].astype(np.float32) * rng.standard_normal(
            cw.shape, dtype=np.float32)
        llr = np.clip(np.rint(2.0 * y / (sigma[:, None] ** 2) * llr_scale), -127, 127).astype(np.int8)
        cfg = LdpcDecoderConfiguration(base_graph=bg, lifting_size=z, nof_filler_bits=0, nof_crc_bits=24,
                                       max_iterations=max_iterations)
        for t, i in enumerate(idx):
            jobs[i] = CodeblockJob(llr[t], cfg, PG_CRC24B)
            truth[i] = msg[t]
            info[i] = k - 24
    return LdpcBatch(jobs, truth, ebn0, bgs, info,
                     dict(seed=seed, n=n, z=z, ebn0_range=ebn0_range, llr_scale=llr_scale,
                          max_iterations=max_iterations))


# ----------------------------------------------------------------------------------------------
# PUSCH slots.

@dataclass
class PuschUe:
    """One UE's PUSCH PDU in a slot (the fields the receive path needs)."""
    rb_start: int
    nof_rb: int
    nof_layers: int
    modulation_order: int
    tbs_bits: int
    base_graph: int = 1
    rnti: int = 0x4601
    n_id: int = 0           # DM-RS scrambling identity
    n_id_data: int = 0      # data scrambling identity
    rv: int = 0
    dmrs_symbols: tuple = (2,)
    first_symbol: int = 0
    nof_symbols: int = 14
    snr_db: float = 10.0
    channel: str = "flat"   # "flat": one CN(0,1) coefficient per (port, layer); "pdp": exponential PDP
    rms_delay_ns: float = 100.0
    nof_taps: int = 8
    doppler_hz: float = 0.0  # maximum Doppler shift of the "pdp" taps (0: constant in time)


@dataclass
class PuschSlot:
    grid: np.ndarray                 # uint32 complex bf16 [port][14][12*nof_prb_grid]
    ues: list
    truth: list                      # transport-block bits per UE
    nof_ports: int
    nof_prb_grid: int
    slot: int
    scs_khz: int = 30
    dmrs_scaling: float = float(np.float32(10 ** (3 / 20)))  # two CDM groups without data: +3 dB DM-RS
    channels: list = field(default_factory=list)      # per UE: [P][L][nsc] or [P][L][14][nsc]
    noise_vars: list = field(default_factory=list)
    symbols: list = field(default_factory=list)       # per UE: transmitted data symbols [RE][layer]


def data_symbol_list(ue):
    return [s for s in range(ue.first_symbol, ue.first_symbol + ue.nof_symbols) if s not in ue.dmrs_symbols]


def nof_ch_symbols(ue):
    """Channel symbols of the codeword over all layers (no data on DM-RS symbols)."""
    return len(data_symbol_list(ue)) * 12 * ue.nof_rb * ue.nof_layers


def symbol_start_s(scs_khz=30):
    """Start time of each of the 14 OFDM symbols of a slot (normal cyclic prefix, equal symbols)."""
    return np.arange(14) * (1e-3 / (scs_khz / 15) / 14)


def channel_response(rng, ue, nof_ports, scs_khz):
    """Frequency response over the allocation: H [port][layer][12*nof_rb], constant in time, or
    [port][layer][14][12*nof_rb] for exponential-PDP taps with a Doppler shift (each tap a sum of
    16 sinusoids with random arrival angles and phases: Rayleigh fading with Jakes' spectrum)."""
    nsc = 12 * ue.nof_rb
    if ue.channel == "flat":
        h = (rng.standard_normal((nof_ports, ue.nof_layers)) + 1j * rng.standard_normal((nof_ports, ue.nof_layers)))
        return np.repeat((h / np.sqrt(2))[..., None], nsc, axis=-1)
    # Exponential power-delay profile with the given RMS delay spread, nof_taps equally spaced taps
    # up to 3 RMS delays, unit total power, independent Rayleigh taps per (port, layer).
    tau = np.linspace(0, 3 * ue.rms_delay_ns * 1e-9, ue.nof_taps)
    p = np.exp(-tau / (ue.rms_delay_ns * 1e-9))
    p /= p.sum()
    f = (np.arange(nsc) + 12 * ue.rb_start) * scs_khz * 1e3
    steer = np.exp(-2j * np.pi * tau[:, None] * f[None, :])
    if ue.doppler_hz > 0:
        m = 16
        ang = rng.uniform(0, 2 * np.pi, (nof_ports, ue.nof_layers, ue.nof_taps, m))
        ph = rng.uniform(0, 2 * np.pi, (nof_ports, ue.nof_layers, ue.nof_taps, m))
        t = symbol_start_s(scs_khz)
        a = np.exp(1j * (2 * np.pi * ue.doppler_hz * np.cos(ang)[..., None] * t + ph[..., None])).sum(3) / np.sqrt(m)
        return np.einsum("plts,tf->plsf", a * np.sqrt(p)[None, None, :, None], steer)
    taps = (rng.standard_normal((nof_ports, ue.nof_layers, ue.nof_taps))
            + 1j * rng.standard_normal((nof_ports, ue.nof_layers, ue.nof_taps))) * np.sqrt(p / 2)
    return np.einsum("plt,tf->plf", taps, steer)


def make_pusch_slot(ues, nof_ports, nof_prb_grid=273, slot=0, seed=0, scs_khz=30, tb_bits=None):
    """Seeded uplink slot: for each UE, random TB -> UL-SCH coding -> scrambling -> modulation ->
    layer mapping -> RE mapping with DM-RS (type 1, amplitude +3 dB) -> channel -> AWGN; the
    grid is rounded to complex bf16 (the reference's resource-grid storage). tb_bits (one array per
    UE) transmits given transport blocks instead, e.g. a HARQ retransmission with another rv."""
    from . import prg
    from .demod import to_cbf16

    rng = np.random.default_rng(seed)
    nsc_grid = 12 * nof_prb_grid
    grid = np.zeros((nof_ports, 14, nsc_grid), np.complex128)
    truth, chans, nvs, syms = [], [], [], []
    beta = float(np.float32(10 ** (3 / 20)))
    for ue in ues:
        ncs = nof_ch_symbols(ue)
        seg = codec.segment_tx(ue.tbs_bits, ue.base_graph, ue.modulation_order, ue.nof_layers, ncs)
        tb = rng.integers(0, 2, ue.tbs_bits, dtype=np.uint8)
        if tb_bits is not None:
            tb = np.asarray(tb_bits[len(truth)], np.uint8)
        cw = codec.ulsch_encode(tb, ue.base_graph, ue.modulation_order, ue.nof_layers, ncs, seg, rv=ue.rv)
        cw = cw ^ prg.scrambling(ue.rnti, ue.n_id_data, cw.size)
        d = codec.modulate(cw, ue.modulation_order)              # [ncs]
        nre_sym = 12 * ue.nof_rb
        x = d.reshape(-1, ue.nof_layers)                          # [RE][layer]
        h = channel_response(rng, ue, nof_ports, scs_khz)         # [P][L][nsc]
        sc = slice(12 * ue.rb_start, 12 * (ue.rb_start + ue.nof_rb))
        r = 0
        for s in range(ue.first_symbol, ue.first_symbol + ue.nof_symbols):
            if s in ue.dmrs_symbols:
                pil = prg.dmrs_type1(slot, s, ue.n_id, ue.rb_start, ue.nof_rb, ue.nof_layers) * beta
                tx = np.zeros((ue.nof_layers, nre_sym), np.complex128)
                tx[:, 0::2] = pil
            else:
                tx = x[r:r + nre_sym].T
                r += nre_sym
            hs = h[:, :, s, :] if h.ndim == 4 else h
            grid[:, s, sc] += np.einsum("plf,lf->pf", hs, tx)
        # Noise: SNR per receive port relative to unit per-layer signal power.
        nv = 10 ** (-ue.snr_db / 10)
        for s in range(ue.first_symbol, ue.first_symbol + ue.nof_symbols):
            grid[:, s, sc] += np.sqrt(nv / 2) * (rng.standard_normal((nof_ports, nre_sym))
                                                + 1j * rng.standard_normal((nof_ports, nre_sym)))
        truth.append(tb)
        chans.append(h)
        nvs.append(nv)
        syms.append(x)
    return PuschSlot(to_cbf16(grid.astype(np.complex64)), list(ues), truth, nof_ports, nof_prb_grid, slot, scs_khz,
                     beta, chans, nvs, syms)


# ----------------------------------------------------------------------------------------------
# Slot workloads of the benchmark configurations.

def required_snr_db(qm, rate_x1024, nof_layers, nof_ports):
    """Per-port SNR at which a PDU is expected to decode with BLER <= 10 %: the Shannon SNR of its
    spectral efficiency per layer, less the combining gain of nof_ports receive ports over
    nof_layers layers, plus an implementation gap of 8 dB (one layer) or 9 dB (two layers). The gap
    is where this simulator's slots (exponential-PDP Rayleigh channels, DM-RS estimation, 6 LDPC
    iterations, no HARQ) reached 10 % BLER in a sweep of 3,072 UEs over MCS table 2."""
    se = qm * rate_x1024 / 1024.0
    gap = 8.0 + (nof_layers - 1) * 1.0
    return 10 * np.log10(2.0 ** se - 1.0) + gap - 10 * np.log10(nof_ports - nof_layers + 1)


def ue_from_mcs(rb_start, nof_rb, nof_layers, table, index, dmrs_symbols, **kw):
    """A PDU whose TBS and base graph follow TS 38.214 / TS 38.212 from (MCS table, index)."""
    from . import mcs as mcs_tables
    qm, r = mcs_tables.mcs(table, index)
    a = mcs_tables.tbs(14, 12 * len(dmrs_symbols), 0, qm, r, nof_layers, nof_rb)
    return PuschUe(rb_start=rb_start, nof_rb=nof_rb, nof_layers=nof_layers, modulation_order=qm, tbs_bits=a,
                   base_graph=mcs_tables.base_graph(r, a), dmrs_symbols=tuple(dmrs_symbols), **kw)


def single_ue_slot(seed=0):
    """20 MHz / 30 kHz, 51 PRB, DM-RS symbol 2, 1 layer, 2 rx, QPSK (MCS table 1 index 5),
    flat Rayleigh per rx port, 10 dB."""
    ue = ue_from_mcs(0, 51, 1, 1, 5, (2,), snr_db=10.0, channel="flat")
    return make_pusch_slot([ue], 2, nof_prb_grid=51, seed=seed)


def full_cell_slot(seed=0, slot=0):
    """100 MHz / 30 kHz, 273 PRB, DM-RS symbols 2 and 11, 2 layers, 4 rx, 256QAM (MCS table 2
    index 20), exponential PDP (100 ns RMS, 8 taps), 25 dB."""
    ue = ue_from_mcs(0, 273, 2, 2, 20, (2, 11), snr_db=25.0, channel="pdp")
    return make_pusch_slot([ue], 4, nof_prb_grid=273, seed=seed, slot=slot)


def uneven_cells(seed=0, nof_cells=16, nof_ports=4, snr_range=(0.0, 30.0), max_ues=16, delay_range_ns=None,
                 doppler_range_hz=None, la_margin_db=0.0):
    """The batched uneven slot: nof_cells cells of 273 PRB, each with 1..max_ues UEs on contiguous
    PRB allocations that tile at most 273 PRB, 1 or 2 layers, per-UE SNR uniform in snr_range,
    exponential-PDP channels. The MCS (table 2) of each UE is drawn among the indices its SNR
    supports (required_snr_db), the highest few favoured; TBS and base graph follow from it.
    With delay_range_ns / doppler_range_hz, each UE's RMS delay spread and maximum Doppler shift
    are drawn uniformly from them (from a second generator, so the rest of the slot is the same);
    otherwise 100 ns and no Doppler. la_margin_db raises every link-adaptation threshold."""
    from . import mcs as mcs_tables
    rng = np.random.default_rng(seed)
    rng_ch = np.random.default_rng([seed, 1])
    slots = []
    for cell in range(nof_cells):
        n_ues = int(rng.integers(1, max_ues + 1))
        used = int(rng.integers(max(n_ues, 200), 274))
        cuts = np.sort(rng.choice(np.arange(1, used), size=n_ues - 1, replace=False)) if n_ues > 1 else []
        edges = [0, *[int(c) for c in cuts], used]
        ues = []
        for u in range(n_ues):
            nof_rb = edges[u + 1] - edges[u]
            layers = int(rng.integers(1, 3))
            snr = float(rng.uniform(*snr_range))
            ok = [i for i, (qm, r) in enumerate(mcs_tables.MCS_TABLE_2)
                  if required_snr_db(qm, r, layers, nof_ports) + la_margin_db <= snr]
            if not ok and layers == 2:
                layers = 1
                ok = [i for i, (qm, r) in enumerate(mcs_tables.MCS_TABLE_2)
                      if required_snr_db(qm, r, layers, nof_ports) + la_margin_db <= snr]
            top = max(ok) if ok else 0
            index = int(rng.integers(max(0, top - 3), top + 1))
            ch = {}
            if delay_range_ns is not None:
                ch["rms_delay_ns"] = float(rng_ch.uniform(*delay_range_ns))
            if doppler_range_hz is not None:
                ch["doppler_hz"] = float(rng_ch.uniform(*doppler_range_hz))
            ues.append(ue_from_mcs(edges[u], nof_rb, layers, 2, index, (2, 11), snr_db=snr, channel="pdp",
                                   rnti=0x4000 + 16 * cell + u, n_id=cell, n_id_data=cell, **ch))
        slots.append(make_pusch_slot(ues, nof_ports, nof_prb_grid=273, slot=cell % 20,
                                     seed=int(rng.integers(0, 2 ** 31))))
    return slots


# ----------------------------------------------------------------------------------------------
# Open Fronthaul block floating point (O-RAN.WG4.CUS Annex A.1.2), the uplink U-plane payload a
# radio unit sends: per PRB an exponent byte, then the 24 samples of `width` bits, big-endian.


def bfp_compress(words, width):
    """Compresses complex bf16 grid words (12 per PRB, real in the low half) to BFP bytes: samples
    quantised to 16-bit fixed point (gain 2^15 - 1, rounded to nearest, saturated to int16), the
    PRB's exponent the smallest right shift that fits every sample in `width` signed bits."""
    w = np.ascontiguousarray(words, np.uint32).reshape(-1, 12)
    nprb = w.shape[0]
    f = np.stack([(w & 0xFFFF) << 16, w & 0xFFFF0000], axis=-1).astype(np.uint32).view(np.float32).reshape(nprb, 24)
    q = np.clip(np.rint(f.astype(np.float64) * np.float32(32767.0)), -32768, 32767).astype(np.int32)
    mag = np.max(np.where(q < 0, -q - 1, q), axis=1)          # largest magnitude of the signed values
    need = np.where(mag > 0, np.floor(np.log2(np.maximum(mag, 1))).astype(np.int32) + 2, 1)
    e = np.clip(need - width, 0, 15).astype(np.int32)
    v = (q >> e[:, None]) & ((1 << width) - 1)
    bits = ((v[:, :, None] >> np.arange(width - 1, -1, -1)) & 1).astype(np.uint8).reshape(nprb, 24 * width)
    out = np.zeros((nprb, 1 + 3 * width), np.uint8)
    out[:, 0] = e
    out[:, 1:] = np.packbits(bits, axis=1)
    return out.ravel()


def scale_grid_words(words, factor):
    """Complex bf16 grid words multiplied by a power of two (exact): the radio unit's gain that
    brings the received signal into the fixed-point range before BFP compression."""
    w = np.asarray(words, np.uint32)
    f = np.stack([(w & 0xFFFF) << 16, w & 0xFFFF0000], axis=-1).astype(np.uint32).view(np.float32) * np.float32(factor)
    h = (f.view(np.uint32) >> 16).astype(np.uint32)
    return (h[..., 0] | (h[..., 1] << 16)).astype(np.uint32)


# ----------------------------------------------------------------------------------------------
# Replay bursts (the E3 pusch.symbols recording format of the reference's ocudu-pusch-replay).

def synthetic_burst(seed=0, nof_prb=52, mcs_table=2, mcs_index=10, nof_layers=1, sinr_db=20.0, rv=0,
                    crc_ok_reported=True, nof_dmrs=2, nof_harq_ack_bits=0, nof_csi_part1_bits=0):
    """A recorded PUSCH burst in the form the reference's replay tool reads
    (apps/tools/pusch_replay/ocudu_pusch_replay.cpp:93-137): the grant of one UE with 14 OFDM
    symbols and DM-RS type 1 at symbols 2 (and 11), and its equalised data symbols - the scrambled
    UL-SCH codeword of a random TB, QAM-modulated with unit energy, plus complex white noise of
    variance 10^(-SINR/10). With UCI bits in the grant the symbols are random QPSK-scaled noise of
    the same length (this simulator has no UCI transmit multiplexer), a burst for the replay's
    accounting and demultiplexing, not for decoding. Returns (replay.Burst, transmitted TB bits)."""
    from . import mcs as mcs_tables
    from . import prg
    from .replay import Burst

    rng = np.random.default_rng(seed)
    dmrs = (2, 11)[:nof_dmrs]
    qm, r = mcs_tables.mcs(mcs_table, mcs_index)
    tbs = mcs_tables.tbs(14, 12 * len(dmrs), 0, qm, r, nof_layers, nof_prb)
    bg = mcs_tables.base_graph(r, tbs)
    ncs = (14 - len(dmrs)) * 12 * nof_prb * nof_layers
    seg = codec.segment_tx(tbs, bg, qm, nof_layers, ncs)
    tb = rng.integers(0, 2, tbs, dtype=np.uint8)
    # TBS_LBRM of TS 38.212 Section 5.4.2.1 for a 273-PRB, 4-layer, 256QAM carrier.
    lbrm_bits = mcs_tables.tbs(14, 12, 0, 8, 948, 4, 273)
    c = seg["nof_cbs"]
    nref = min(lbrm_bits * 3 // (2 * c), 25344)
    rnti, n_id = int(rng.integers(1, 0xFFEF)), int(rng.integers(0, 1024))
    cw = codec.ulsch_encode(tb, bg, qm, nof_layers, ncs, seg, rv=rv, nref=nref)
    cw = cw ^ prg.scrambling(rnti, n_id, cw.size)
    x = codec.modulate(cw, qm)
    if nof_harq_ack_bits or nof_csi_part1_bits:
        x = codec.modulate(rng.integers(0, 2, cw.size, dtype=np.uint8), qm)
    nv = 10 ** (-sinr_db / 10)
    y = x + np.sqrt(nv / 2) * (rng.standard_normal(x.size) + 1j * rng.standard_normal(x.size))
    mask = 0
    for s in dmrs:
        mask |= 1 << s
    grant = {"tbs_bytes": tbs // 8, "tbs_lbrm_bytes": lbrm_bits // 8, "ldpc_base_graph": bg, "rv": rv,
             "harq_id": 0, "n_id": n_id, "mcs_index": mcs_index, "mcs_table": mcs_table,
             "nof_harq_ack_bits": nof_harq_ack_bits, "nof_csi_part1_bits": nof_csi_part1_bits, "alpha_scaling": 1.0,
             "beta_offset_harq_ack": 20.0,
             "beta_offset_csi_part1": 6.25, "beta_offset_csi_part2": 6.25, "start_symbol": 0, "nof_symbols": 14,
             "dmrs_type": 1, "dmrs_symbol_mask": mask, "nof_cdm_groups_without_data": 2, "dc_position": None,
             "prb_mask": "ff" * ((nof_prb + 7) // 8)}
    burst = Burst(rnti=rnti, numerology=1, sfn=int(rng.integers(0, 1024)), slot=int(rng.integers(0, 20)),
                  modulation_bits=qm, sinr_db=float(sinr_db), nof_prb=nof_prb, nof_layers=nof_layers,
                  crc_known=crc_ok_reported is not None, crc_ok_reported=bool(crc_ok_reported),
                  symbols_truncated=False, grant=grant, symbols=y.astype(np.complex64))
    return burst, tb

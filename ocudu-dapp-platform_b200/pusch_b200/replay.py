"""Offline PUSCH burst replay on the B200: the counterpart of the reference's ocudu-pusch-replay
(apps/tools/pusch_replay/ocudu_pusch_replay.cpp). A burst is one recorded PUSCH transmission as the
E3 ``pusch.symbols`` stream publishes it: a JSON file with the grant parameters and a ``samples_file``
of complex64 equalised data symbols ([OFDM symbol][RE][layer], the exporter's order). The burst
runs through the receiver chain the gNB runs after equalisation - soft demapping with a flat noise
variance from the reported post-equalisation SINR, descrambling, UL-SCH demultiplexing, rate
dematching, LDPC decoding, TB CRC - here on the GPU (pg_demodulate_soft_host,
pg_descramble_host, pg_ulsch_demultiplex_device for bursts that carry UCI with the sizes of
pg_ulsch_information, pg_sch_decode_batch_host),
and the TB CRC is printed next to the one the gNB reported, so recordings can be validated and other
front ends (channel estimation, equalisation) scored by writing their output as the same JSON + cf32
pair.

    python -m pusch_b200.replay burst.json [--iterations N] [--verbose]

Exit status as the reference tool: 0 when the replayed CRC passes, 1 when it fails, 2 on errors.
"""
import argparse
import ctypes
import json
import math
import os
import sys
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native, uci
from .demod import DemodulationMapper
from .sch import PuschDecoder, SchTransportBlock

# ldpc::MAX_CODEBLOCK_SIZE (include/ocudu/phy/upper/channel_coding/ldpc/ldpc.h): 66 * 384.
MAX_CODEBLOCK_SIZE = 25344


@dataclass
class Burst:
    """The fields ocudu_pusch_replay.cpp:93-137 reads from the exporter's JSON."""
    rnti: int
    numerology: int
    sfn: int
    slot: int
    modulation_bits: int
    sinr_db: float
    nof_prb: int
    nof_layers: int
    crc_known: bool
    crc_ok_reported: bool
    symbols_truncated: bool
    grant: dict
    symbols: np.ndarray  # complex64


def load_burst(path) -> Burst:
    """Reads a burst JSON and its sample file (a bare file name is taken relative to the JSON's
    directory). Values the gNB did not report are JSON null: sinr_db then defaults to 20 dB and the
    reported CRC is unknown, as in the reference tool."""
    with open(path) as f:
        root = json.load(f)
    slot = root["radio_slot"]
    sinr = root.get("sinr_db")
    crc = root.get("crc_ok")
    trunc = root.get("symbols_truncated")
    samples = root["samples_file"]
    if "/" not in samples:
        samples = os.path.join(os.path.dirname(os.path.abspath(path)), samples)
    raw = np.fromfile(samples, np.uint8)
    if raw.size % 8:
        raise ValueError("sample file is not whole complex64 values")
    return Burst(rnti=int(root["rnti"]), numerology=int(slot["numerology"]), sfn=int(slot["sfn"]),
                 slot=int(slot["slot"]), modulation_bits=int(root["modulation_bits"]),
                 sinr_db=float(sinr) if isinstance(sinr, (int, float)) and not isinstance(sinr, bool) else 20.0,
                 nof_prb=int(root["nof_prb"]), nof_layers=int(root["nof_layers"]),
                 crc_known=crc is not None, crc_ok_reported=bool(crc) if crc is not None else False,
                 symbols_truncated=trunc is True, grant=root["grant"], symbols=raw.view(np.complex64))


def write_burst(path, burst: Burst, samples_name=None):
    """Writes a burst in the exporter's format (JSON + cf32), e.g. to score another front end."""
    samples_name = samples_name or os.path.splitext(os.path.basename(path))[0] + ".cf32"
    root = {"rnti": burst.rnti, "radio_slot": {"numerology": burst.numerology, "sfn": burst.sfn, "slot": burst.slot},
            "modulation_bits": burst.modulation_bits, "sinr_db": burst.sinr_db, "nof_prb": burst.nof_prb,
            "nof_layers": burst.nof_layers, "crc_ok": burst.crc_ok_reported if burst.crc_known else None,
            "symbols_truncated": burst.symbols_truncated, "grant": burst.grant, "samples_file": samples_name}
    with open(path, "w") as f:
        json.dump(root, f, indent=1)
    np.ascontiguousarray(burst.symbols, np.complex64).tofile(os.path.join(os.path.dirname(os.path.abspath(path)),
                                                                          samples_name))


@dataclass
class ReplayResult:
    crc_ok: bool
    tbs_bytes: int
    nof_codeblocks: int
    ulsch_bits: int
    mean_iterations: float
    transport_block: Optional[np.ndarray]
    llrs: np.ndarray  # the descrambled codeword soft bits


def nof_codeblocks(tbs_bits, base_graph):
    """compute_nof_codeblocks (include/ocudu/ran/sch/sch_segmentation.h:52): the TB with its CRC over
    the largest codeblock payload of the base graph."""
    crc = 16 if tbs_bits <= 3824 else 24
    b = tbs_bits + crc
    kcb = 8448 if base_graph == 1 else 3840
    return 1 if b <= kcb else math.ceil(b / (kcb - 24))


def replay(ctx: _native.Context, burst: Burst, iterations=10) -> ReplayResult:
    g = burst.grant
    qm, nl = burst.modulation_bits, burst.nof_layers
    nre_symbol = 12 * burst.nof_prb
    if burst.symbols.size % (nre_symbol * nl):
        raise ValueError(f"sample count {burst.symbols.size} is not a whole number of OFDM symbols")
    tbs_bits = 8 * int(g["tbs_bytes"])
    bg = 2 if int(g["ldpc_base_graph"]) == 2 else 1
    c = nof_codeblocks(tbs_bits, bg)
    nref = min(8 * int(g["tbs_lbrm_bytes"]) * 3 // (2 * c), MAX_CODEBLOCK_SIZE)
    # Soft demapping with the flat post-equalisation noise of the reported SINR, then descrambling
    # with c_init = RNTI 2^15 + n_ID (TS 38.211 Section 6.3.1.1).
    noise = np.full(burst.symbols.size, 10.0 ** (-burst.sinr_db / 10.0), np.float32)
    llrs = DemodulationMapper(ctx).demodulate_soft(burst.symbols, noise, qm)
    c_init = ((burst.rnti << 15) + int(g["n_id"])) & 0xFFFFFFFF
    ctx.check(ctx.lib.pg_descramble_host(ctx.handle, c_init, llrs.ctypes.data_as(ctypes.c_void_p),
                                         llrs.ctypes.data_as(ctypes.c_void_p), llrs.size))
    # UL-SCH information: how many soft bits carry data and how many UCI (TS 38.212 6.3.2.4), then the
    # UL-SCH stream out of the codeword when UCI is multiplexed (ocudu_pusch_replay.cpp:152-188,255-263).
    ack, csi1 = int(g.get("nof_harq_ack_bits") or 0), int(g.get("nof_csi_part1_bits") or 0)
    mask = int(g["dmrs_symbol_mask"])
    contains_dc = False
    if g.get("dc_position") is not None:
        dc_prb = int(g["dc_position"]) // 12
        prb_mask = str(g["prb_mask"])
        contains_dc = bool((int(prb_mask[2 * (dc_prb // 8):2 * (dc_prb // 8) + 2], 16) >> (dc_prb % 8)) & 1)
    info = uci.ulsch_information(tbs_bits, bg, qm, nl, burst.nof_prb, int(g["start_symbol"]), int(g["nof_symbols"]),
                                 mask, ack, csi1, 0, float(g["alpha_scaling"]), float(g["beta_offset_harq_ack"]),
                                 float(g["beta_offset_csi_part1"]), float(g["beta_offset_csi_part2"]),
                                 int(g["nof_cdm_groups_without_data"]), contains_dc=contains_dc)
    sch_llrs = llrs
    if ack or csi1:
        cfg = uci.make_config(nof_llrs=llrs.size, c_init=c_init, nof_harq_ack_rvd=info["nof_harq_ack_rvd"],
                              nof_enc_harq_ack_bits=info["nof_harq_ack_bits"],
                              nof_enc_csi_part1_bits=info["nof_csi_part1_bits"], nof_prb=burst.nof_prb,
                              dmrs_symbol_mask=mask, modulation_order=qm, nof_layers=nl,
                              start_symbol_index=int(g["start_symbol"]), nof_symbols=int(g["nof_symbols"]),
                              dmrs_type=int(g["dmrs_type"]),
                              nof_cdm_groups_without_data=int(g["nof_cdm_groups_without_data"]),
                              nof_harq_ack_bits=ack, nof_csi_part1_bits=csi1)
        sch_llrs = uci.UlschDemultiplexer(ctx).demultiplex([cfg], [llrs])[0][0]
    if sch_llrs.size != info["nof_ul_sch_bits"]:
        raise ValueError(f"{llrs.size} soft bits for a grant of {info['nof_ul_sch_bits']} UL-SCH bits")
    res = PuschDecoder(ctx).decode_batch([SchTransportBlock(llrs=sch_llrs, tbs_bits=tbs_bits, base_graph=bg,
                                                            modulation_order=qm, nof_layers=nl, rv=int(g["rv"]),
                                                            nref=nref, max_iterations=iterations)])[0]
    return ReplayResult(res.tb_crc_ok, tbs_bits // 8, res.nof_codeblocks_total, info["nof_ul_sch_bits"],
                        res.mean_iterations, res.transport_block, llrs)


def main(argv=None):
    p = argparse.ArgumentParser(description="Replays a PUSCH burst captured over E3 through the GPU receiver chain "
                                            "and compares the transport-block CRC with the recorded verdict.")
    p.add_argument("burst")
    p.add_argument("--iterations", type=int, default=10)
    p.add_argument("--verbose", action="store_true")
    a = p.parse_args(argv)
    if not 1 <= a.iterations <= 10000:
        print("error: --iterations out of range", file=sys.stderr)
        return 2
    try:
        b = load_burst(a.burst)
        ctx = _native.Context(max_codeblocks=160)
        r = replay(ctx, b, a.iterations)
    except (OSError, ValueError, KeyError, _native.PgError) as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    g = b.grant
    mcs = (f"{g['mcs_index']}/table{g.get('mcs_table') if isinstance(g.get('mcs_table'), int) else 0}"
           if g.get("mcs_index") is not None else "unknown")
    print(f"rnti=0x{b.rnti:04x} sfn={b.sfn} slot={b.slot} tbs={r.tbs_bytes} B mcs={mcs} bg={g['ldpc_base_graph']} "
          f"rv={g['rv']} prb={b.nof_prb} Qm={b.modulation_bits} layers={b.nof_layers} ulsch_bits={r.ulsch_bits} "
          f"codeblocks={r.nof_codeblocks}")
    reported = ("OK" if b.crc_ok_reported else "FAIL") if b.crc_known else "unknown"
    print(f"replay CRC: {'OK' if r.crc_ok else 'FAIL'} | gNB CRC: {reported}"
          f"{' | capture incomplete' if b.symbols_truncated else ''}"
          f"{' | MISMATCH' if b.crc_known and r.crc_ok != b.crc_ok_reported else ''}")
    if a.verbose:
        print(f"ldpc iterations: mean {r.mean_iterations:.1f} over {r.nof_codeblocks} codeblocks")
        if r.crc_ok:
            print("transport block (first 16 bytes): " + " ".join(f"{x:02x}" for x in r.transport_block[:16]))
    return 0 if r.crc_ok else 1


if __name__ == "__main__":
    sys.exit(main())

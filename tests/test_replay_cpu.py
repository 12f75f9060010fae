"""Replay bursts (the E3 pusch.symbols recording of the reference's ocudu-pusch-replay): the
project's writer and synthetic bursts checked against the reference's own replay tool, compiled
from its source into oracle/_ref (oracle/Makefile), and the JSON reader's handling of the
exporter's null values."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from pusch_b200 import replay, sim

REF_REPLAY = os.path.join(ROOT, "oracle", "_ref", "ocudu_pusch_replay")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_REPLAY), reason="oracle/_ref/ocudu_pusch_replay not built")

# (SINR dB, MCS table, MCS index, layers, PRBs, rv): 16QAM, a failing low-SINR burst, the 100 MHz
# 256QAM two-layer grant (65 codeblocks), a BG2 QPSK retransmission version.
CASES = [(20.0, 2, 10, 1, 52, 0), (-3.0, 2, 10, 1, 52, 0), (30.0, 2, 25, 2, 273, 0), (15.0, 1, 5, 1, 20, 2)]


def write_cases(tmp_path, uci=False):
    out = []
    for i, (sinr, table, index, nl, prb, rv) in enumerate(CASES):
        ack, csi = ((0, 0), (2, 0), (5, 8), (1, 11))[i] if uci else (0, 0)
        b, tb = sim.synthetic_burst(seed=i, nof_prb=prb, mcs_table=table, mcs_index=index, nof_layers=nl,
                                    sinr_db=sinr, rv=rv, nof_harq_ack_bits=ack, nof_csi_part1_bits=csi)
        path = os.path.join(str(tmp_path), f"burst{i}.json")
        replay.write_burst(path, b)
        out.append((path, b, tb))
    return out


@needs_ref
def test_reference_tool_replays_synthetic_bursts(tmp_path):
    for (path, b, tb), case in zip(write_cases(tmp_path), CASES):
        r = subprocess.run([REF_REPLAY, path, "--verbose"], capture_output=True, text=True, timeout=300)
        lines = r.stdout.splitlines()
        if case[0] > 0:
            assert r.returncode == 0, r.stdout + r.stderr
            assert lines[1] == "replay CRC: OK | gNB CRC: OK"
            want = " ".join(f"{x:02x}" for x in np.packbits(tb)[:16])
            assert lines[3] == "transport block (first 16 bytes): " + want
        else:
            assert r.returncode == 1
            assert lines[1] == "replay CRC: FAIL | gNB CRC: OK | MISMATCH"


def test_burst_json_round_trip_and_nulls(tmp_path):
    b, _ = sim.synthetic_burst(seed=5, nof_prb=6, mcs_table=1, mcs_index=3)
    path = os.path.join(str(tmp_path), "b.json")
    replay.write_burst(path, b)
    got = replay.load_burst(path)
    assert (got.rnti, got.sfn, got.slot, got.modulation_bits, got.nof_prb, got.nof_layers) == \
        (b.rnti, b.sfn, b.slot, b.modulation_bits, b.nof_prb, b.nof_layers)
    assert got.grant == b.grant and np.array_equal(got.symbols, b.symbols)
    # Values the gNB did not report are JSON null: SINR then defaults to 20 dB, the CRC is unknown.
    root = json.load(open(path))
    root["sinr_db"], root["crc_ok"] = None, None
    json.dump(root, open(path, "w"))
    got = replay.load_burst(path)
    assert got.sinr_db == 20.0 and not got.crc_known
    # A sample file that is not whole complex64 values is refused.
    with open(os.path.join(str(tmp_path), root["samples_file"]), "ab") as f:
        f.write(b"\0")
    with pytest.raises(ValueError):
        replay.load_burst(path)

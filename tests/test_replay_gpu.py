"""The GPU replay chain (pusch_b200.replay: pg_demodulate_soft_host, pg_descramble_host,
pg_sch_decode_batch_host) against the reference's own replay tool on the same bursts: identical
output (grant line, CRC verdicts, mean LDPC iterations, TB bytes) and exit status."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from pusch_b200 import _native, prg, replay, sim
from test_replay_cpu import REF_REPLAY, needs_ref, write_cases

pytestmark = pytest.mark.gpu


@needs_ref
@pytest.mark.parametrize("uci", [False, True])
def test_replay_matches_reference_tool(tmp_path, uci):
    """uci: the grants carry HARQ-ACK / CSI Part 1 (the UL-SCH bit count and demultiplexing follow the
    UCI sizes; the symbols are noise, so both tools report the same failing CRC and iterations)."""
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "ocudu-dapp-platform_b200"))
    for path, b, tb in write_cases(tmp_path, uci):
        ref = subprocess.run([REF_REPLAY, path, "--verbose"], capture_output=True, text=True, timeout=300)
        got = subprocess.run([sys.executable, "-m", "pusch_b200.replay", path, "--verbose"], capture_output=True,
                             text=True, timeout=300, env=env)
        assert got.returncode == ref.returncode, got.stdout + got.stderr
        assert got.stdout == ref.stdout


def test_descramble_matches_gold_sequence():
    ctx = _native.Context(max_codeblocks=4)
    rng = np.random.default_rng(3)
    for n in (1, 31, 32, 33, 1000, 628992):
        x = rng.integers(-127, 128, n).astype(np.int8)
        c_init = int(rng.integers(0, 1 << 31))
        out = np.empty_like(x)
        ctx.check(ctx.lib.pg_descramble_host(ctx.handle, c_init, x.ctypes.data, out.ctypes.data, n))
        c = prg.gold(c_init, n)
        assert np.array_equal(out, np.where(c == 1, -x.astype(np.int16), x).astype(np.int8))


@needs_ref
def test_replay_decodes_transmitted_tb(tmp_path):
    ctx = _native.Context(max_codeblocks=160)
    b, tb = sim.synthetic_burst(seed=11, nof_prb=106, mcs_table=2, mcs_index=19, nof_layers=2, sinr_db=28.0)
    r = replay.replay(ctx, b, iterations=10)
    assert r.crc_ok and np.array_equal(np.unpackbits(r.transport_block), tb)

"""UCI on PUSCH without a GPU: the Reed-Muller basis table of the library against the reference's
encoder, the demultiplexer's stream sizes (host layout, pg_ulsch_demultiplex_sizes) against the
reference's ulsch_demultiplex on the same configurations, and the checker's own encode/detect round
trip."""
import ctypes
import os
import re

import numpy as np
import pytest

import uci_cases
from pusch_b200 import _native

SRC = os.path.join(os.path.dirname(__file__), "..", "ocudu-dapp-platform_b200", "csrc", "uci_rm_basis.inc")


@pytest.fixture(scope="module")
def lib():
    return _native.load()


def sizes_fn(lib):
    def f(c):
        s = uci_cases.to_struct(c)
        out = (ctypes.c_uint32 * 3)()
        rc = lib.pg_ulsch_demultiplex_sizes(ctypes.byref(s), out)
        return None if rc else tuple(out)
    return f


def test_rm_basis_matches_reference_encoder(ref):
    words = [int(w, 16) for w in re.findall(r"0x([0-9a-f]+)", open(SRC).read().split("{", 1)[1])]
    assert len(words) == 32
    for n in range(11):
        msg = np.zeros(11, np.uint8)
        msg[n] = 1
        cw = ref.short_block_encode(msg, 32, 2)
        assert [(w >> n) & 1 for w in words] == list(cw)


def test_demux_sizes_match_reference(lib, ref):
    rng = np.random.default_rng(71)
    f = sizes_fn(lib)
    for _ in range(150):
        c, sizes = uci_cases.random_config(rng, f)
        llr = uci_cases.random_llrs(rng, c["nof_llrs"])
        sch, ack, csi, complete = ref.ulsch_demultiplex(c, llr, block_size=int(rng.integers(50, 5000)))
        assert complete
        assert sizes == (sch.size, ack.size, csi.size), c


def test_demux_rejects_unsupported(lib):
    f = sizes_fn(lib)
    base = dict(c_init=1, nof_harq_ack_rvd=0, nof_enc_harq_ack_bits=240, nof_enc_csi_part1_bits=0, nof_prb=10,
                dmrs_symbol_mask=1 << 2, modulation_order=2, nof_layers=1, start_symbol_index=0, nof_symbols=14,
                dmrs_type=1, nof_cdm_groups_without_data=2, nof_harq_ack_bits=5, nof_csi_part1_bits=0)
    base["nof_llrs"] = uci_cases.codeword_size(base)
    assert f(base) is not None
    # Polar-coded messages demultiplex as the short-block ones of 3 to 11 bits.
    assert f(dict(base, nof_harq_ack_bits=12)) == f(base) == f(dict(base, nof_harq_ack_bits=1706))
    for bad in (dict(nof_harq_ack_bits=1707), dict(nof_enc_harq_ack_bits=241), dict(nof_llrs=base["nof_llrs"] + 2),
                dict(nof_harq_ack_rvd=4), dict(nof_enc_harq_ack_bits=10 ** 6), dict(dmrs_symbol_mask=0),
                dict(modulation_order=3)):
        assert f(dict(base, **bad)) is None, bad


def test_reference_short_block_round_trip(ref):
    """Noiseless codewords decode to their messages through the reference's detector (the checker
    the GPU detector is compared with)."""
    rng = np.random.default_rng(5)
    for K in range(1, 12):
        for qm in (1, 2, 4, 6, 8):
            msg = rng.integers(0, 2, K, dtype=np.uint8)
            E = max(ref.uci_min_encoded_bits(K), qm) * 3
            E = (E + qm - 1) // qm * qm
            cw = ref.short_block_encode(msg, E, qm)
            llr = np.where(cw == 0, 60, np.where(cw == 1, -60, 0)).astype(np.int8)
            bits, ok = ref.short_block_detect(K, llr, qm)
            assert ok and (bits == msg).all(), (K, qm)

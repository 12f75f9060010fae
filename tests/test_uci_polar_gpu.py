"""Polar-coded UCI (12 to 1706 bits) on the GPU (pg_uci_polar_decode_device) against the
reference's uci_decoder::decode (oracle._ref): equal validity on every message and equal bits on
every valid one, over the shared cases (CRC6 and CRC11, parity-check bits, shortening, puncturing,
repetition, one and two codeblocks, failures at low SNR) decoded in one batch; and the host's
rejection of messages without a polar code."""
import numpy as np
import pytest

import polar_cases
from pusch_b200 import uci
from pusch_b200._native import PgError

pytestmark = pytest.mark.gpu


def test_polar_decoder_matches_reference(ctx, ref):
    cs = polar_cases.cases(ref, seed=0) + polar_cases.cases(ref, seed=1)
    got = uci.PolarUciDecoder(ctx).decode([(A, llr) for A, llr, _ in cs])
    nvalid = 0
    for (A, llr, msg), (bits, ok) in zip(cs, got):
        want_bits, want_ok = ref.uci_polar_decode(A, llr)
        assert ok == want_ok, A
        if want_ok:
            nvalid += 1
            assert np.array_equal(bits, want_bits), A
            assert np.array_equal(bits, msg), A
    assert nvalid >= 2 * len(polar_cases.SIZES)


def test_polar_decoder_rejects_messages_without_code(ctx):
    dec = uci.PolarUciDecoder(ctx)
    with pytest.raises(PgError):
        dec.decode([(11, np.zeros(40, np.int8))])  # a short-block message
    with pytest.raises(PgError):
        dec.decode([(12, np.zeros(20, np.int8))])  # E = 20 is not above K + nPC = 21
    with pytest.raises(PgError):
        dec.decode([(1707, np.zeros(9000, np.int8))])

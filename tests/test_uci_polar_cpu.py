"""Polar-coded UCI (12 to 1706 bits), CPU side:
- the library's code construction (pg_polar_code: N, K_set, PC_set, sub-block interleaver) equals
  the reference's polar_code_impl::set over the uplink range of (K, E);
- the oracle's restatement of the decoder (oracle/polar_oracle.py) gives the reference's
  uci_decoder::decode output (bits and validity) on the shared cases, including failures;
- the encoder of the test vectors round-trips through the reference decoder at high SNR."""
import numpy as np

import polar_cases
import polar_oracle
from pusch_b200 import uci


def test_code_construction_matches_reference(ref):
    checked = 0
    for K in list(range(18, 26)) + list(range(31, 1024, 11)):
        for E in sorted({K + 4, K + 30, int(K * 1.2) + 4, int(K * 2.2), K + 190, 600, 1088, 4000, 8192}):
            a, b = ref.polar_code(K, E), uci.polar_code(K, E)
            assert (a is None) == (b is None), (K, E)
            if a is None:
                continue
            assert a["N"] == b["N"] and a["nPC"] == b["nPC"], (K, E)
            assert np.array_equal(a["k_set"], b["k_set"]), (K, E)
            assert a["pc_set"][:a["nPC"]] == b["pc_set"][:b["nPC"]], (K, E)
            assert np.array_equal(a["subblock"], b["subblock"]), (K, E)
            checked += 1
    assert checked > 800
    # The reference's range checks: K 26..30, E not above K + nPC, E above 8192.
    assert uci.polar_code(28, 200) is None and uci.polar_code(18, 21) is None and uci.polar_code(40, 8193) is None


def test_oracle_decoder_matches_reference(ref):
    nvalid = 0
    for A, llr, msg in polar_cases.cases(ref):
        want_bits, want_ok = ref.uci_polar_decode(A, llr)
        got_bits, got_ok = polar_oracle.uci_polar_decode(A, llr, ref.polar_code)
        assert got_ok == want_ok, A
        if want_ok:
            nvalid += 1
            assert np.array_equal(got_bits, want_bits), A
            assert np.array_equal(want_bits, msg), A
    assert nvalid >= len(polar_cases.SIZES)  # every size decodes at the higher SNR


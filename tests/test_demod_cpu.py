"""Demapper restatement and FP64 equaliser against the reference's outputs (no GPU)."""
import numpy as np

import golden_io
from fp64 import equalize_fp64, rel_err

# The reference's one-layer equaliser multiplies by the approximate reciprocal (rcp14 on
# AVX-512, 2^-14 relative error) and its noise variance by its square; MMSE uses an exact
# reciprocal. Bound of the reference's own error against exact arithmetic:
REF_EQ_REL_BOUND = 2.5e-4


def test_port_demapper_matches_golden(port):
    for c in golden_io.demap_cases():
        got = port.demodulate_soft(c["qm"], c["symbols"], c["noise"])
        assert (got == c["llrs"]).all(), c["qm"]


def test_fp64_equalizer_vs_reference_golden():
    for c in golden_io.eq_cases():
        eq, var = equalize_fp64(c["y"], c["h"], c["nv"], c["tx"])
        assert np.array_equal(np.isinf(var), np.isinf(c["var"]))
        assert rel_err(c["eq"], eq).max() < REF_EQ_REL_BOUND, (c["ports"], c["layers"])
        assert rel_err(c["var"], var).max() < REF_EQ_REL_BOUND, (c["ports"], c["layers"])

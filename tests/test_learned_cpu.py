"""Learned channel estimator, host side and checker (no GPU): the float64 network restatement
against finite differences, and the parameter layout against the library's."""
import numpy as np

import learned_ref as lr
from pusch_b200 import _native
from pusch_b200 import learned


def test_parameter_layout_matches_library():
    assert _native.load().pg_le_nof_params() == lr.layer_offsets()[1] == learned.nof_params() == 256848


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    rows = 40
    valid = np.ones(rows, bool)
    valid[:2] = valid[20:22] = False
    params = learned.init_params(3).astype(np.float64)
    params[-16 - 5 * 64 * 16:] *= 50  # a visible output layer
    x = rng.standard_normal((rows, 16)) * valid[:, None]
    dy = rng.standard_normal((rows, 16)) * valid[:, None]
    y, cache = lr.forward(params, x, valid, bf16_acts=False)
    g = lr.backward(cache, dy)
    offs, _ = lr.layer_offsets()
    for layer, idx in [(0, 7), (5, 1234), (13, 100), (13, 5 * 64 * 16 + 3), (2, 5 * 64 * 64 + 10)]:
        i = offs[layer] + idx
        e = 1e-6
        p2 = params.copy()
        p2[i] += e
        y2, _ = lr.forward(p2, x, valid, bf16_acts=False)
        fd = ((y2 - y) * dy).sum() / e
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(fd)), (layer, idx, fd, g[i])


def test_initial_network_is_close_to_identity():
    """The untrained network's corrections are small: the plain estimate is the starting point."""
    rng = np.random.default_rng(1)
    rows = 300
    valid = np.ones(rows, bool)
    x = rng.standard_normal((rows, 16))
    y, _ = lr.forward(learned.init_params(0).astype(np.float64), x, valid, bf16_acts=False)
    assert np.abs(y).mean() < 0.1

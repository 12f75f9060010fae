"""port_channel_estimator on the GPU through pg_port_channel_estimate_host (the drop-in adapter's
entry), given the reference's own pilots: frequency response, noise, EPRE, SNR and RSRP within 1e-4
of the reference's estimator, per-symbol bf16 estimates equal or one unit apart, and the reference's
CFO and time alignment, on the golden cases (1 to 273 PRB) and on every UE and port of a 16-cell
slot."""
import math

import numpy as np
import pytest

import golden_io
from fp64 import rel_err
from pusch_b200 import sim
from pusch_b200.pusch import PortChannelEstimator

pytestmark = pytest.mark.gpu
BETA = float(np.float32(10 ** (3 / 20)))
TOL = 1e-4
TC = 1.0 / (480e3 * 4096)  # NR basic time unit


def from_seconds(s):
    """phy_time_unit::from_seconds of the reference's float seconds (include/ocudu/ran/phy_time_unit.h:
    ten times the Tc count truncated toward zero, then rounded to the nearest Tc)."""
    t = math.trunc(float(np.float32(s)) / TC * 10.0)
    return math.trunc(t / 10) + math.trunc(math.fmod(t, 10) / 5)


def cbf16_parts(w):
    w = np.asarray(w).astype(np.uint32)
    return (w << 16).view(np.float32).astype(np.float64), (w & 0xFFFF0000).view(np.float32).astype(np.float64)


def check_bf16_estimates(got, want, what):
    """Per-symbol bf16 estimates: 99 % of the components bit-equal; every component within one bf16
    unit of its own magnitude plus TOL of the coefficient's magnitude (a component much smaller than
    its coefficient carries the FP32 difference of the whole coefficient in many of its own units)."""
    g_re, g_im = cbf16_parts(got)
    r_re, r_im = cbf16_parts(want)
    mag = np.hypot(r_re, r_im)
    for g, r in ((g_re, r_re), (g_im, r_im)):
        top = np.maximum(np.abs(g), np.abs(r))
        ulp = np.where(top > 0, 2.0 ** (np.floor(np.log2(np.where(top > 0, top, 1.0))) - 7), 0.0)
        assert (np.abs(g - r) <= ulp + TOL * mag).all(), (what, float(np.max(np.abs(g - r) - ulp - TOL * mag)))
    for part in (0, 16):
        d = ((got >> part) & 0xFFFF).astype(np.int32) - ((want >> part) & 0xFFFF).astype(np.int32)
        assert (d == 0).mean() > 0.99, what


def check_port(est, ref, grid, port, slot, n_id, rb_start, nof_rb, nof_layers, dmrs, what):
    freq, sym, sc = ref.port_estimate_full(grid, port, slot, n_id, rb_start, nof_rb, nof_layers, dmrs, BETA)
    got = est.compute(grid[port], sc["pilots"], rb_start, nof_rb, dmrs, BETA)
    assert rel_err(got.freq_response, freq).max() < TOL, what
    for g, w in ((got.noise_var, sc["noise_var"]), (got.epre, sc["epre"]), (got.snr, sc["snr"])):
        assert abs(g - w) <= TOL * abs(w), what
    assert np.allclose(got.rsrp, sc["rsrp"], rtol=TOL), what
    check_bf16_estimates(got.symbol_estimates, sym, what)
    if np.isnan(sc["cfo_hz"]):
        assert got.cfo_hz is None, what
    else:
        # The CFO is the phase of a sum of products; FP32 summation order moves it by a few ulp of the
        # phase: 1e-3 Hz absolute or 1e-3 relative.
        assert abs(got.cfo_hz - sc["cfo_hz"]) <= max(1e-3, 1e-3 * abs(sc["cfo_hz"])), (what, got.cfo_hz, sc["cfo_hz"])
    # Time alignment: the reference reports whole Tc (phy_time_unit::from_seconds of the curve-fitted
    # correlation peak). The same Tc, or the neighbouring one where this inverse DFT's raw value lies
    # within 1 % of a correlation sample (1 / (N x SCS x 2) seconds, N <= 4096) of a rounding boundary.
    n_dft = max(128, 1 << int(np.ceil(np.log2(max(1, 6 * nof_rb * 4096 // 3300)))))
    fs = n_dft * 30e3 * 2
    got_tc, ref_tc = from_seconds(got.time_alignment_s), round(sc["ta_s"] / TC)
    raw = got.time_alignment_s / TC
    near = abs(abs(raw - math.trunc(raw)) - 0.5) <= 0.01 / fs / TC
    assert got_tc == ref_tc or (abs(got_tc - ref_tc) == 1 and near), (what, got.time_alignment_s, sc["ta_s"])
    return got


def test_port_estimator_golden_cases(ctx, ref):
    est = PortChannelEstimator(ctx)
    for c in golden_io.est_cases():
        for p in range(c["ports"]):
            check_port(est, ref, c["grid"], p, c["slot"], c["n_id"], c["rb_start"], c["nof_rb"], c["nof_layers"],
                       c["dmrs"], (c["nof_rb"], p))


def test_port_estimator_16cell_slot(ctx, ref):
    est = PortChannelEstimator(ctx)
    for cell in sim.uneven_cells(seed=5, nof_cells=16)[::3]:
        for ue in cell.ues:
            for p in range(cell.nof_ports):
                check_port(est, ref, cell.grid, p, cell.slot, ue.n_id, ue.rb_start, ue.nof_rb, ue.nof_layers,
                           list(ue.dmrs_symbols), (ue.rb_start, ue.nof_rb, p))

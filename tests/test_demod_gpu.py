"""GPU equaliser and demapper against the reference (golden fixtures), the restated demapper and
the FP64 equaliser."""
import numpy as np
import pytest

import golden_io
from fp64 import equalize_fp64, rel_err
from pusch_b200.demod import MMSE, ZF, ChannelEqualizer, DemodulationMapper

pytestmark = pytest.mark.gpu

# Float32 kernels against exact arithmetic (the north-star bound for equalised symbols and noise
# variances), and against the reference's own float32 outputs (which carry rcp14 error).
EQ_REL_TOL_FP64 = 1e-4
EQ_REL_TOL_REF = 2.5e-4


def test_demapper_golden_within_one_lsb(ctx):
    dm = DemodulationMapper(ctx)
    for c in golden_io.demap_cases():
        got = dm.demodulate_soft(c["symbols"], c["noise"], c["qm"]).astype(int)
        d = np.abs(got - c["llrs"].astype(int))
        assert d.max() <= 1, c["qm"]
        assert (d == 0).mean() > 0.999, c["qm"]


def test_demapper_random_vs_port(ctx, port):
    dm = DemodulationMapper(ctx)
    rng = np.random.default_rng(5)
    for qm in (2, 4, 6, 8):
        n = 50000
        s = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.9).astype(np.complex64)
        nv = rng.uniform(1e-3, 2.0, n).astype(np.float32)
        d = np.abs(dm.demodulate_soft(s, nv, qm).astype(int) - port.demodulate_soft(qm, s, nv).astype(int))
        assert d.max() <= 1
        assert (d == 0).mean() > 0.999


def test_equalizer_golden(ctx):
    for c in golden_io.eq_cases():
        eqz = ChannelEqualizer(ctx, algorithm=c["alg"])
        eq, var = eqz.equalize(c["y"], c["h"], c["nv"], c["tx"])
        e64, v64 = equalize_fp64(c["y"], c["h"], c["nv"], c["tx"])
        assert np.array_equal(np.isinf(var), np.isinf(c["var"]))
        assert np.array_equal(eq == 0, c["eq"] == 0)
        assert rel_err(eq, e64).max() < EQ_REL_TOL_FP64, (c["ports"], c["layers"])
        assert rel_err(var, v64).max() < EQ_REL_TOL_FP64, (c["ports"], c["layers"])
        assert rel_err(eq, c["eq"]).max() < EQ_REL_TOL_REF
        assert rel_err(var, c["var"]).max() < EQ_REL_TOL_REF


def test_equalizer_rejects_zf_multilayer(ctx):
    from pusch_b200 import _native
    eqz = ChannelEqualizer(ctx, algorithm=ZF)
    y = np.zeros((4, 8), np.uint32)
    h = np.zeros((4, 2, 8), np.uint32)
    with pytest.raises(_native.PgError):
        eqz.equalize(y, h, np.ones(4, np.float32))

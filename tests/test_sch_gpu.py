"""GPU rate dematching, CRC and transport-block decoding against the reference's outputs
(golden fixtures) and the CPU restatement."""
import numpy as np
import pytest

import golden_io
from pusch_b200 import codec, sch
from pusch_b200.sch import CrcCalculatorBatch, LdpcRateDematcher, PuschDecoder, RmConfig, SchTransportBlock

pytestmark = pytest.mark.gpu


def test_rate_dematch_golden(ctx):
    rm = LdpcRateDematcher(ctx)
    cases = golden_io.rm_cases()
    items = []
    for c in cases:
        items.append((c["llrs"], c["prev"].copy(), bool(c["new_data"]),
                      RmConfig(c["bg"], c["z"], c["rv"], c["qm"], c["nref"], c["filler"])))
    rm.rate_dematch_batch(items)
    for c, it in zip(cases, items):
        assert (it[1] == c["out"]).all(), (c["bg"], c["z"], c["qm"], c["rv"], c["new_data"])


def test_rate_dematch_random_vs_port(ctx, port):
    rm = LdpcRateDematcher(ctx)
    rng = np.random.default_rng(11)
    items, want = [], []
    for t in range(120):
        bg = 1 + t % 2
        z = [384, 288, 64, 16, 7, 2, 208, 120][t % 8]
        k = golden_io.kbits(bg, z)
        n = (66 if bg == 1 else 50) * z
        qm = [1, 2, 4, 6, 8][t % 5]
        f = int(rng.integers(0, (k - 2 * z) // 3))
        nref = 0 if t % 3 else int(rng.integers(k + 1, n + 1))
        e = qm * int(rng.integers(1, (3 * n) // qm))
        llr = rng.integers(-120, 121, e).astype(np.int8)
        prev = rng.integers(-120, 121, n).astype(np.int8)
        nd = bool(t % 4)
        cfg = RmConfig(bg, z, t % 4, qm, nref, f)
        items.append((llr, prev.copy(), nd, cfg))
        want.append(port.rate_dematch(bg, z, llr, rv=t % 4, qm=qm, Nref=nref, filler=f, new_data=nd, out=prev.copy()))
    rm.rate_dematch_batch(items)
    for it, w in zip(items, want):
        assert (it[1] == w).all()


def test_crc_golden(ctx):
    calc = CrcCalculatorBatch(ctx)
    cases = golden_io.crc_cases()
    for poly in (0, 1, 2):
        sel = [c for c in cases if c["poly"] == poly]
        got = calc.calculate(poly, [c["bits"] for c in sel])
        assert [int(x) for x in got] == [c["crc"] for c in sel]


def test_crc_long_strings_vs_port(ctx, port):
    calc = CrcCalculatorBatch(ctx)
    rng = np.random.default_rng(3)
    strings = [rng.integers(0, 2, n, dtype=np.uint8) for n in (1, 31, 32, 33, 4095, 65537, 417976 + 24, 1_000_003)]
    for poly in (0, 1, 2):
        got = calc.calculate(poly, strings)
        assert [int(x) for x in got] == [port.crc(poly, s) for s in strings]


def make_tb(rng, tbs, bg, qm, nl, nsym, snr_db=None, rv=0):
    seg = sch.segment(tbs, bg, qm, nl, nsym)
    tb = rng.integers(0, 2, tbs, dtype=np.uint8)
    g = codec.ulsch_encode(tb, bg, qm, nl, nsym, seg, rv=rv)
    x = 1.0 - 2.0 * g
    if snr_db is None:
        llr = (x * 100).astype(np.int8)
    else:
        sigma = 10 ** (-snr_db / 20)
        y = x + sigma * rng.standard_normal(g.size)
        llr = np.clip(np.rint(y * 2 / sigma ** 2 * 2), -120, 120).astype(np.int8)
    return tb, llr, seg


def oracle_tb_decode(port, llr, tbs, bg, qm, seg, max_iter, rv=0):
    """CPU chain: restated dematcher and decoder, TB CRC by the restated CRC."""
    c, z, f = seg["nof_cbs"], seg["lifting_size"], seg["nof_filler_bits"]
    k = seg["cb_length"]
    n = (66 if bg == 1 else 50) * z
    off, payload, ok_all, iters = 0, [], True, []
    for i in range(c):
        e = seg["e_short"] if i < seg["nof_short_cbs"] else seg["e_long"]
        buf = port.rate_dematch(bg, z, llr[off:off + e], rv=rv, qm=qm, filler=f, new_data=True)
        off += e
        poly = 2 if c > 1 else (0 if tbs <= 3824 else 1)
        it, bits = port.ldpc_decode(bg, z, buf, filler=f, crc_poly=poly, max_iter=max_iter)
        iters.append(it)
        ok_all &= it > 0
        kp = k - f - (24 if c > 1 else 0)
        payload.append(np.unpackbits(bits)[:kp])
    tbcat = np.concatenate(payload)
    tb_ok = ok_all and (c == 1 or port.crc(1 if tbs > 3824 else 0, tbcat) == 0)
    return tb_ok, tbcat[:tbs], iters


@pytest.mark.parametrize("tbs,bg,qm,nl,nsym,snr", [
    (5888, 1, 2, 1, 13 * 612, None),          # 20 MHz QPSK slot, one codeblock
    (5888, 1, 2, 1, 13 * 612, 1.0),
    (417976, 1, 8, 2, 2 * 12 * 3276, None),   # 100 MHz 2-layer 256QAM slot, 50 codeblocks
    (417976, 1, 8, 2, 2 * 12 * 3276, 14.0),
    (1320, 2, 4, 1, 600, 3.0),
    (3840, 2, 6, 2, 2400, None),
    (40016, 1, 4, 2, 21000, 2.0),
])
def test_sch_decode_matches_oracle(ctx, port, tbs, bg, qm, nl, nsym, snr):
    rng = np.random.default_rng(tbs + qm)
    tb, llr, seg = make_tb(rng, tbs, bg, qm, nl, nsym, snr)
    dec = PuschDecoder(ctx)
    res = dec.decode_batch([SchTransportBlock(llr, tbs, bg, qm, nl, max_iterations=6)])[0]
    want_ok, want_bits, want_it = oracle_tb_decode(port, llr, tbs, bg, qm, seg, 6)
    assert res.tb_crc_ok == want_ok
    assert res.nof_codeblocks_total == seg["nof_cbs"]
    assert res.nof_codeblocks_crc_ok == sum(1 for x in want_it if x > 0)
    if want_ok:
        assert (np.unpackbits(res.transport_block) == want_bits).all()
        assert (want_bits == tb).all()
    if snr is None:
        assert res.tb_crc_ok


def test_sch_decode_batch_mixed(ctx):
    rng = np.random.default_rng(9)
    jobs, truth = [], []
    for tbs, bg, qm, nl, nsym in [(5888, 1, 2, 1, 13 * 612), (1320, 2, 4, 1, 600), (100008, 1, 6, 2, 40000),
                                  (3840, 2, 6, 2, 2400), (24, 2, 2, 1, 48)]:
        tb, llr, _ = make_tb(rng, tbs, bg, qm, nl, nsym, None)
        jobs.append(SchTransportBlock(llr, tbs, bg, qm, nl))
        truth.append(tb)
    res = PuschDecoder(ctx).decode_batch(jobs)
    for r, tb in zip(res, truth):
        assert r.tb_crc_ok
        assert (np.unpackbits(r.transport_block) == tb).all()

"""The CPU restatement (oracle/pusch_oracle.c) pinned against the reference: golden fixtures
made by the reference's own code, plus fresh random cases when oracle/_ref is built."""
import numpy as np
import pytest

import golden_io


def unpack(b, n):
    return np.unpackbits(np.asarray(b, np.uint8))[:n]


@pytest.mark.parametrize("case", range(len(golden_io.ldpc_cases())))
def test_port_ldpc_matches_golden(port, case):
    c = golden_io.ldpc_cases()[case]
    poly = -1 if c["poly"] == 255 else c["poly"]
    it, bits = port.ldpc_decode(c["bg"], c["z"], c["llrs"], filler=c["filler"], crc_poly=poly,
                                max_iter=c["max_iter"])
    assert it == c["iterations"]
    k = golden_io.kbits(c["bg"], c["z"])
    assert (unpack(bits, k) == unpack(c["bits"], k)).all()


def test_port_rate_dematch_matches_golden(port):
    for c in golden_io.rm_cases():
        out = port.rate_dematch(c["bg"], c["z"], c["llrs"], rv=c["rv"], qm=c["qm"], Nref=c["nref"],
                                filler=c["filler"], new_data=c["new_data"], out=c["prev"].copy())
        assert (out == c["out"]).all(), c["meta"] if "meta" in c else (c["bg"], c["z"], c["qm"], c["rv"])


def test_port_crc_matches_golden(port):
    for c in golden_io.crc_cases():
        assert port.crc(c["poly"], c["bits"]) == c["crc"]


def test_port_vs_reference_random(port, ref):
    """Fresh noisy codeblocks of many shapes: bits and iteration counts identical."""
    from pusch_b200 import codec
    rng = np.random.default_rng(99)
    for t in range(24):
        bg = 1 + t % 2
        z = [384, 288, 64, 16, 2, 7, 208, 240, 13, 44, 120, 352][t % 12]
        k = golden_io.kbits(bg, z)
        n = (66 if bg == 1 else 50) * z
        f = 0 if t % 3 else min(k // 5, 60)
        msg = np.concatenate([codec.attach_crc(2, rng.integers(0, 2, k - 24 - f, dtype=np.uint8)),
                              np.zeros(f, np.uint8)])
        cw = codec.ldpc_encode(bg, z, msg)
        e = int(rng.integers(k + 2 * z, n + 1))
        sigma = np.sqrt(1 / (2 * (k / e) * 10 ** (rng.uniform(0, 3) / 10)))
        llr = np.clip(np.rint((1 - 2.0 * cw + sigma * rng.standard_normal(n)) * 2 / sigma ** 2 * 3), -120,
                      120).astype(np.int8)
        llr[e:] = 0
        if f:
            llr[k - 2 * z - f:k - 2 * z] = 127
        a = ref.ldpc_decode(bg, z, llr, filler=f, max_iter=8)
        b = port.ldpc_decode(bg, z, llr, filler=f, max_iter=8)
        assert a[0] == b[0]
        assert (unpack(a[1], k) == unpack(b[1], k)).all()


def test_port_rate_dematch_vs_reference_random(port, ref):
    rng = np.random.default_rng(5)
    for t in range(60):
        bg = 1 + t % 2
        z = [384, 288, 64, 16, 7, 2][t % 6]
        k = golden_io.kbits(bg, z)
        n = (66 if bg == 1 else 50) * z
        qm = [1, 2, 4, 6, 8][t % 5]
        f = int(rng.integers(0, (k - 2 * z) // 3))
        nref = 0 if t % 3 else int(rng.integers(k, n + 1))
        e = qm * int(rng.integers(1, (2 * n) // qm))
        llr = rng.integers(-120, 121, e).astype(np.int8)
        prev = rng.integers(-120, 121, n).astype(np.int8)
        for nd in (True, False):
            a = ref.rate_dematch(bg, z, llr, rv=t % 4, qm=qm, Nref=nref, filler=f, new_data=nd, out=prev.copy())
            b = port.rate_dematch(bg, z, llr, rv=t % 4, qm=qm, Nref=nref, filler=f, new_data=nd, out=prev.copy())
            assert (a == b).all()


def test_reference_variants_agree(ref):
    """AVX-512 and AVX2 reference decoders agree bit for bit (the parity target)."""
    import os
    try:
        ref.ldpc_decode(1, 2, np.ones(132, np.int8), variant="avx512")
    except RuntimeError:
        pytest.skip("no AVX-512 on this host")
    for c in golden_io.ldpc_cases()[:8]:
        a = ref.ldpc_decode(c["bg"], c["z"], c["llrs"], max_iter=c["max_iter"], variant="avx512")
        b = ref.ldpc_decode(c["bg"], c["z"], c["llrs"], max_iter=c["max_iter"], variant="avx2")
        assert a[0] == b[0] and (a[1] == b[1]).all()

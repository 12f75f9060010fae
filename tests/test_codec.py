"""The simulator's transmit-side coding (pusch_b200.codec) against the reference's outputs."""
import numpy as np

import golden_io
from pusch_b200 import codec


def test_encoder_matches_reference_golden():
    for c in golden_io.enc_cases():
        cw = codec.ldpc_encode(c["bg"], c["z"], c["msg"])
        assert (cw == c["cw"]).all(), (c["bg"], c["z"])


def test_crc_matches_reference_golden():
    for c in golden_io.crc_cases():
        assert int(codec.crc(c["poly"], c["bits"])) == c["crc"]


def test_attach_crc_checks_to_zero():
    rng = np.random.default_rng(1)
    for poly in (0, 1, 2):
        b = codec.attach_crc(poly, rng.integers(0, 2, (5, 333), dtype=np.uint8))
        assert (codec.crc(poly, b) == 0).all()


def test_codewords_satisfy_all_parity_checks():
    rng = np.random.default_rng(2)
    for bg, z in [(1, 384), (2, 384), (1, 5), (2, 36)]:
        kb = 22 if bg == 1 else 10
        msg = rng.integers(0, 2, (2, kb * z), dtype=np.uint8)
        cw = codec.ldpc_encode(bg, z, msg)
        full = np.concatenate([msg[:, :2 * z], cw], axis=1).reshape(2, -1, z)
        for r, row in enumerate(codec.lifted_edges(bg, z)):
            acc = np.zeros((2, z), np.uint8)
            for c, s in row:
                acc ^= np.roll(full[:, c, :], -s, axis=-1)
            assert not acc.any(), (bg, z, r)

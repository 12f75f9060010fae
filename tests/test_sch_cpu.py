"""Segmentation and transmit-side rate matching against the reference (no GPU)."""
import numpy as np
import pytest

from pusch_b200 import codec, sch


@pytest.mark.parametrize("tbs,bg", [(5888, 1), (417976, 1), (100, 2), (3824, 2), (3832, 1), (1000000, 1), (24, 2),
                                    (600, 2), (8424, 1), (8448, 1), (200, 2), (1320, 2), (3840, 2), (24000, 1)])
def test_segmentation_matches_reference(ref, tbs, bg):
    r = ref.sch_segmentation(tbs, bg)
    s = sch.segment(tbs, bg, 2, 1, 6000)
    assert (r["C"], r["Z"], r["K"], r["tb_crc"]) == (s["nof_cbs"], s["lifting_size"], s["cb_length"], s["tb_crc_bits"])


def test_rate_lengths_follow_38212():
    # TS 38.212 5.4.2.1: E_r = N_L*Qm*floor(G/(N_L*Qm*C)) for the first C - mod(G/(N_L*Qm), C)
    # codeblocks, ceil for the rest; the lengths add up to G.
    for tbs, bg, qm, nl, nsym in [(417976, 1, 8, 2, 2 * 12 * 3276), (5888, 1, 2, 1, 13 * 612), (40000, 1, 4, 2, 21000)]:
        s = sch.segment(tbs, bg, qm, nl, nsym)
        c = s["nof_cbs"]
        g = nsym * qm
        per_layer = nsym // nl
        assert s["nof_short_cbs"] == c - per_layer % c
        assert s["e_short"] == nl * qm * (g // (nl * qm * c))
        assert s["nof_short_cbs"] * s["e_short"] + (c - s["nof_short_cbs"]) * s["e_long"] == g


def test_config_segmentations():
    # 20 MHz QPSK slot: TBS 5888, one BG1 codeblock, Z = 288, F = 424, E = 15912.
    s = sch.segment(5888, 1, 2, 1, 13 * 612)
    assert (s["nof_cbs"], s["lifting_size"], s["nof_filler_bits"], s["e_short"]) == (1, 288, 424, 15912)
    # 100 MHz 2-layer 256QAM slot: TBS 417976 -> 50 BG1 codeblocks with Z = 384.
    s = sch.segment(417976, 1, 8, 2, 2 * 12 * 3276)
    assert (s["nof_cbs"], s["lifting_size"]) == (50, 384)


def test_rate_match_matches_reference(ref):
    rng = np.random.default_rng(4)
    for t in range(30):
        bg = 1 + t % 2
        z = [384, 288, 64, 16, 7, 2][t % 6]
        k = (22 if bg == 1 else 10) * z
        n = (66 if bg == 1 else 50) * z
        qm = [1, 2, 4, 6, 8][t % 5]
        f = int(rng.integers(0, (k - 2 * z) // 3))
        nref = 0 if t % 3 else int(rng.integers(k + 1, n + 1))
        e = qm * int(rng.integers(1, (2 * n) // qm))
        msg = rng.integers(0, 2, k).astype(np.uint8)
        msg[k - f:] = 0
        a = ref.ldpc_encode_rm(bg, z, msg, e, rv=t % 4, qm=qm, Nref=nref, filler=f)
        b = codec.rate_match(bg, z, codec.ldpc_encode(bg, z, msg), e, rv=t % 4, qm=qm, nref=nref, nof_filler_bits=f)
        assert (a == b).all()


def test_transmit_segmentation_matches_library_and_reference(ref):
    """The simulator's own segmentation (codec.segment_tx, transmit side) equals the receive
    library's (pg_sch_segment) and the reference's for random transport blocks and allocations."""
    rng = np.random.default_rng(21)
    for _ in range(400):
        bg = int(rng.integers(1, 3))
        tbs = 8 * int(rng.integers(3, 60000 if bg == 1 else 500))
        qm = int(rng.choice([1, 2, 4, 6, 8]))
        nl = int(rng.integers(1, 3))
        nsym = nl * int(rng.integers(1, 40000))
        a = codec.segment_tx(tbs, bg, qm, nl, nsym)
        b = sch.segment(tbs, bg, qm, nl, nsym)
        assert a == b, (tbs, bg, qm, nl, nsym)
        r = ref.sch_segmentation(tbs, bg)
        assert (r["C"], r["Z"], r["K"], r["tb_crc"]) == (a["nof_cbs"], a["lifting_size"], a["cb_length"],
                                                          a["tb_crc_bits"])

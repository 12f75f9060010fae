"""pg_ulsch_information (the encoded sizes of UCI multiplexed on PUSCH, TS 38.212 Section 6.3.2.4)
against the reference's get_ulsch_information (lib/ran/pusch/ulsch_info.cpp) compiled in
oracle/_ref, over random grants with and without UL-SCH, every HARQ-ACK / CSI size class and beta
offset of TS 38.213 Tables 9.3-1/2."""
import numpy as np
import pytest

from pusch_b200 import mcs, uci

ref_mod = pytest.importorskip("oracle")

BETA_ACK = [1.0, 2.0, 2.5, 3.125, 4.0, 5.0, 6.25, 8.0, 10.0, 12.625, 15.875, 20.0, 31.0, 50.0, 80.0, 126.0]
BETA_CSI = [1.125, 1.25, 1.375, 1.625, 1.75, 2.0, 2.25, 2.5, 2.875, 3.125, 3.5, 4.0, 5.0, 6.25, 8.0, 10.0, 12.625,
            15.875, 20.0]
FIELDS = ["nof_ul_sch_bits", "nof_harq_ack_bits", "nof_harq_ack_rvd", "nof_csi_part1_bits", "nof_csi_part2_bits",
          "nof_harq_ack_re", "nof_csi_part1_re", "nof_csi_part2_re", "nof_dc_overlap_bits"]


def test_ulsch_information_matches_reference():
    try:
        ref = ref_mod.Ref()
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(9)
    checked = 0
    for _ in range(3000):
        table = int(rng.integers(1, 3))
        index = int(rng.integers(0, 28))
        qm, rate = mcs.mcs(table, index)
        nl = int(rng.integers(1, 3))
        nof_rb = int(rng.integers(1, 274))
        start = int(rng.integers(0, 3))
        nsym = int(rng.integers(4, 15 - start))
        dmrs = [start] if rng.random() < 0.3 else [start + 2, start + nsym - 2][:1 + (nsym >= 8)]
        dmrs = sorted(set(d for d in dmrs if start <= d < start + nsym))
        mask = sum(1 << d for d in dmrs)
        cdm = int(rng.integers(1, 3))
        with_sch = rng.random() < 0.85
        tbs = mcs.tbs(nsym, 6 * cdm * len(dmrs), 0, qm, rate, nl, nof_rb) if with_sch else 0
        bg = mcs.base_graph(rate, tbs) if with_sch else 1
        ack = int(rng.choice([0, 1, 2, 3, 5, 11, 12, 19, 20, 40]))
        csi1 = int(rng.choice([0, 1, 4, 11, 12, 20, 60]))
        csi2 = 0 if with_sch else int(rng.choice([0, 0, 8, 30]))
        alpha = float(rng.choice([0.5, 0.65, 0.8, 1.0]))
        b_ack, b_c1, b_c2 = float(rng.choice(BETA_ACK)), float(rng.choice(BETA_CSI)), float(rng.choice(BETA_CSI))
        dc = bool(rng.random() < 0.1)
        want = ref.ulsch_information(tbs, float(rate), qm, nl, ack, csi1, csi2, alpha, b_ack, b_c1, b_c2, nof_rb,
                                     start, nsym, mask, cdm, dc)
        got = uci.ulsch_information(tbs, bg, qm, nl, nof_rb, start, nsym, mask, ack, csi1, csi2, alpha, b_ack, b_c1,
                                    b_c2, cdm, float(np.float32(rate) * np.float32(1.0 / 1024)), dc)
        assert tuple(got[f] for f in FIELDS) == want, (tbs, qm, nl, nof_rb, start, nsym, dmrs, cdm, ack, csi1, csi2)
        checked += 1
    assert checked == 3000

"""The reference's CPU receive path as assembled in the oracle (ref_pusch_decode_mt: the
reference's estimator, equaliser, demapper, descrambler, segmenter, dematcher, decoder and TB
join, in pusch_processor's order) decodes the simulator's slots: it is the CPU baseline of the
PUSCH benchmark and the reference arm, so it must recover the transmitted transport blocks."""
import numpy as np

from pusch_b200 import sim
from pusch_b200.pusch import batch_descriptors


def test_reference_chain_decodes_simulated_slots(ref):
    slots = [sim.single_ue_slot(seed=1)] + sim.uneven_cells(seed=5, nof_cells=2, max_ues=4)
    descs, grid, tb_bytes, ues = batch_descriptors(slots, max_iterations=6)
    ok, iters, tb, dt = ref.pusch_decode_mt(descs, grid, tb_bytes, 2)
    truth = [t for sl in slots for t in sl.truth]
    assert ok[0]  # the 20 MHz single-UE slot
    assert ok.mean() >= 0.9
    for i, t in enumerate(truth):
        if ok[i]:
            o = descs[i].tb_out_offset
            assert (np.unpackbits(tb[o:o + descs[i].tbs_bits // 8]) == t).all(), i
    assert dt > 0

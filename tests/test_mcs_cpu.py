"""MCS tables, TBS and base-graph selection of the workload generator against the reference's own
pusch_mcs_get_config, tbs_calculator_calculate and get_ldpc_base_graph."""
import numpy as np

from pusch_b200 import mcs


def test_mcs_tables_match_reference(ref):
    for table, rows in ((1, mcs.MCS_TABLE_1), (2, mcs.MCS_TABLE_2)):
        for i, (qm, r) in enumerate(rows):
            assert ref.pusch_mcs(table, i) == (qm, r), (table, i)


def test_tbs_and_base_graph_match_reference(ref):
    rng = np.random.default_rng(5)
    cases = [(14, 12, 5, 1, 51), (14, 24, 20, 2, 273)]  # the 20 MHz and 100 MHz slot shapes
    for _ in range(3000):
        nd = int(rng.integers(1, 3))
        cases.append((int(rng.integers(4, 15)), 12 * nd, int(rng.integers(0, 28)), int(rng.integers(1, 3)), int(rng.integers(1, 274))))
    for table in (1, 2):
        for nsym, ndmrs, idx, layers, nprb in cases:
            rows = mcs.MCS_TABLE_1 if table == 1 else mcs.MCS_TABLE_2
            qm, r = rows[min(idx, len(rows) - 1)]
            want = ref.tbs(nsym, ndmrs, 0, qm, r, layers, nprb)
            got = mcs.tbs(nsym, ndmrs, 0, qm, r, layers, nprb)
            assert got == want, (table, nsym, ndmrs, idx, layers, nprb)
            assert mcs.base_graph(r, got) == ref.base_graph(r, got)
    # The configurations' own TBS: 51 PRB QPSK table 1 index 5 and 273 PRB 2 layers table 2 index 20.
    assert mcs.tbs(14, 12, 0, *mcs.mcs(1, 5), 1, 51) == 5888
    assert mcs.tbs(14, 24, 0, *mcs.mcs(2, 20), 2, 273) == 417976

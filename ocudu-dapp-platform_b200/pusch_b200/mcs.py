"""PUSCH MCS tables, transport block size and LDPC base graph (TS 38.214 Tables 5.1.3.1-1/-2 and
Section 5.1.3.2; TS 38.212 Section 7.2.2), used by the seeded workload generator to build PDUs the
way the reference's scheduler does (lib/ran/pusch/pusch_mcs.cpp, lib/ran/sch/tbs_calculator.cpp,
include/ocudu/ran/sch/ldpc_base_graph.h:20-31)."""
import numpy as np

# (Qm, target code rate x 1024) per MCS index; table 1 = "qam64", table 2 = "qam256".
MCS_TABLE_1 = [(2, 120), (2, 157), (2, 193), (2, 251), (2, 308), (2, 379), (2, 449), (2, 526), (2, 602), (2, 679),
               (4, 340), (4, 378), (4, 434), (4, 490), (4, 553), (4, 616), (4, 658), (6, 438), (6, 466), (6, 517),
               (6, 567), (6, 616), (6, 666), (6, 719), (6, 772), (6, 822), (6, 873), (6, 910), (6, 948)]
MCS_TABLE_2 = [(2, 120), (2, 193), (2, 308), (2, 449), (2, 602), (4, 378), (4, 434), (4, 490), (4, 553), (4, 616),
               (4, 658), (6, 466), (6, 517), (6, 567), (6, 616), (6, 666), (6, 719), (6, 772), (6, 822), (6, 873),
               (8, 682.5), (8, 711), (8, 754), (8, 797), (8, 841), (8, 885), (8, 916.5), (8, 948)]

# TBS for N'_info <= 3824 (TS 38.214 Table 5.1.3.2-1).
TBS_SMALL = [24, 32, 40, 48, 56, 64, 72, 80, 88, 96, 104, 112, 120, 128, 136, 144, 152, 160, 168, 176, 184, 192, 208,
             224, 240, 256, 272, 288, 304, 320, 336, 352, 368, 384, 408, 432, 456, 480, 504, 528, 552, 576, 608, 640,
             672, 704, 736, 768, 808, 848, 888, 928, 984, 1032, 1064, 1128, 1160, 1192, 1224, 1256, 1288, 1320, 1352,
             1416, 1480, 1544, 1608, 1672, 1736, 1800, 1864, 1928, 2024, 2088, 2152, 2216, 2280, 2408, 2472, 2536,
             2600, 2664, 2728, 2792, 2856, 2976, 3104, 3240, 3368, 3496, 3624, 3752, 3824]


def mcs(table, index):
    """(Qm, R x 1024) of MCS `index` in table 1 (qam64) or 2 (qam256)."""
    return (MCS_TABLE_1 if table == 1 else MCS_TABLE_2)[index]


def tbs(nof_symb_sh, nof_dmrs_prb, nof_oh_prb, qm, rate_x1024, nof_layers, n_prb):
    """Transport block size in bits (TS 38.214 Section 5.1.3.2, no TB scaling). nof_symb_sh counts
    every symbol of the allocation (DM-RS symbols included); nof_dmrs_prb the DM-RS REs per PRB
    including the CDM groups without data. N_info is formed in single precision, as the reference's
    calculator does, so that values at a rounding boundary give the same TBS."""
    f32 = np.float32
    n_re = min(156, 12 * nof_symb_sh - nof_dmrs_prb - nof_oh_prb) * n_prb
    tcr = f32(rate_x1024) * f32(1.0 / 1024)
    n_info = f32(f32(f32(f32(1.0) * f32(n_re)) * tcr) * f32(qm)) * f32(nof_layers)
    if n_info <= 3824:
        n = 3 if n_info <= 512 else int(np.floor(np.log2(n_info))) - 6
        n_info_p = max(24, (1 << n) * int(np.floor(n_info / f32(1 << n))))
        return next(t for t in TBS_SMALL if t >= n_info_p)
    n = int(np.floor(np.log2(f32(n_info - f32(24)))) - f32(5))
    q = f32(f32(n_info - f32(24)) / f32(1 << n))
    qd = float(q)  # std::round: half away from zero, exact on the float32 value
    n_info_p = max(3840, (1 << n) * int(np.floor(qd) + (1 if qd - np.floor(qd) >= 0.5 else 0)))
    c = 1
    if tcr <= f32(0.25):
        c = -(-(n_info_p + 24) // 3816)
    elif n_info_p > 8424:
        c = -(-(n_info_p + 24) // 8424)
    return 8 * c * -(-(n_info_p + 24) // (8 * c)) - 24


def base_graph(rate_x1024, tbs_bits):
    """LDPC base graph 1 or 2 for target code rate R and payload size A (TS 38.212 Section 7.2.2)."""
    r = np.float32(rate_x1024) * np.float32(1.0 / 1024)
    if tbs_bits <= 292 or r <= 0.25 or (tbs_bits <= 3824 and r <= 0.67):
        return 2
    return 1

"""Seeded UCI-on-PUSCH cases shared by the CPU and GPU tests: demultiplexer configurations that
fit their allocation, and short-block messages with their soft bits."""
import numpy as np

from pusch_b200._native import PgUlschDemuxConfig

FIELDS = [f for f, _ in PgUlschDemuxConfig._fields_]


def codeword_size(c):
    """Soft bits of the allocation: data REs of every symbol times Qm * layers."""
    re_dmrs = (12 - c["nof_cdm_groups_without_data"] * (6 if c["dmrs_type"] == 1 else 4)) * c["nof_prb"]
    g = 0
    for s in range(c["start_symbol_index"], c["start_symbol_index"] + c["nof_symbols"]):
        g += (re_dmrs if (c["dmrs_symbol_mask"] >> s) & 1 else 12 * c["nof_prb"])
    return g * c["modulation_order"] * c["nof_layers"]


def to_struct(c):
    s = PgUlschDemuxConfig()
    for f in FIELDS:
        setattr(s, f, int(c.get(f, 0)))
    return s


def random_config(rng, sizes_fn, tries=200):
    """A random consistent configuration (sizes_fn: the library's pg_ulsch_demultiplex_sizes)."""
    for _ in range(tries):
        qm = int(rng.choice([1, 2, 4, 6, 8]))
        L = int(rng.choice([1, 1, 2]))
        bpr = qm * L
        nof_prb = int(rng.integers(1, 25))
        start = int(rng.integers(0, 3))
        nsym = int(rng.integers(6, 15 - start))
        # DM-RS from the allocation's second symbol on: the reference's demultiplexer takes no soft
        # bits when the allocation starts with a symbol that carries none.
        dm = [start + int(rng.integers(1, 3))]
        if rng.random() < 0.5 and nsym > 8:
            dm.append(start + nsym - 1 - int(rng.integers(0, 3)))
        if rng.random() < 0.25:
            dm.append(dm[0] + 1)  # double-symbol DM-RS
        mask = 0
        for s in dm:
            mask |= 1 << s
        dmrs_type = int(rng.choice([1, 2]))
        ncdm = int(rng.integers(1, 3 if dmrs_type == 1 else 4))
        ack_bits = int(rng.choice([0, 1, 2, 3, 5, 8, 11]))
        csi_bits = int(rng.choice([0, 0, 1, 2, 4, 11]))
        # Data REs available for UCI (symbols without DM-RS) bound the random sizes.
        uci_re = sum(12 * nof_prb for s in range(start, start + nsym) if not (mask >> s) & 1)
        cap = max(1, uci_re // 3)
        rvd = ack = csi = 0
        if ack_bits:
            a = int(rng.integers(1, max(2, min(cap, 200))))
            if ack_bits <= 2:
                rvd = bpr * (a + int(rng.integers(0, 20)))
            ack = bpr * a
        if csi_bits:
            csi = bpr * int(rng.integers(1, max(2, min(cap, 300))))
        c = dict(c_init=int(rng.integers(0, 2 ** 31)), nof_harq_ack_rvd=rvd, nof_enc_harq_ack_bits=ack,
                 nof_enc_csi_part1_bits=csi, nof_prb=nof_prb, dmrs_symbol_mask=mask, modulation_order=qm,
                 nof_layers=L, start_symbol_index=start, nof_symbols=nsym, dmrs_type=dmrs_type,
                 nof_cdm_groups_without_data=ncdm, nof_harq_ack_bits=ack_bits, nof_csi_part1_bits=csi_bits)
        c["nof_llrs"] = codeword_size(c)
        sizes = sizes_fn(c)
        if sizes is not None:
            return c, sizes
    raise RuntimeError("no consistent configuration found")


def random_llrs(rng, n):
    x = rng.integers(-120, 121, n).astype(np.int8)
    sat = rng.random(n) < 0.02
    x[sat] = np.where(rng.random(sat.sum()) < 0.5, 127, -127)
    return x


def short_block_cases(rng, ref, n):
    """(K, qm, llrs) triples: encoded messages at various SNRs, pure noise, sparse and saturated
    inputs, and spans below the minimum length."""
    out = []
    for t in range(n):
        K = int(rng.integers(1, 12))
        qm = int(rng.choice([1, 2, 4, 6, 8]))
        E_min = ref.uci_min_encoded_bits(K)
        E = max(qm, E_min) + int(rng.integers(0, 150))
        E = (E + qm - 1) // qm * qm
        kind = t % 6
        if kind == 5:
            E = max(1, E_min - int(rng.integers(1, 3)))  # too short
        msg = rng.integers(0, 2, K, dtype=np.uint8)
        cw = ref.short_block_encode(msg, E, qm) if E >= qm or K > 2 else np.zeros(E, np.uint8)
        bits = np.where(cw <= 1, cw, 0).astype(np.float64)  # placeholders count as zero-valued bits
        amp = 1.0 - 2.0 * bits
        amp[cw > 1] = 0.0
        if kind == 0:
            llr = amp * 60.0
        elif kind in (1, 2):
            sigma = [0.3, 1.2][kind - 1]
            llr = (amp + sigma * rng.standard_normal(E)) * 40.0
        elif kind == 3:
            llr = rng.standard_normal(E) * 50.0
        else:
            llr = amp * 127.0
            llr[rng.random(E) < 0.5] = 0.0
        out.append((K, qm, np.clip(np.rint(llr), -127, 127).astype(np.int8)))
    return out

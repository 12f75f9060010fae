"""UCI on PUSCH on the GPU against the reference's own CPU code (oracle/_ref): the UL-SCH
demultiplexer's three streams (bit-exact, placeholders and punctured REs included), the short-block
detector's bits and validity decisions, and the two chained."""
import ctypes

import numpy as np
import pytest

import uci_cases
from pusch_b200._native import PgUciShortBlock

pytestmark = pytest.mark.gpu


def sizes_fn(ctx):
    def f(c):
        s = uci_cases.to_struct(c)
        out = (ctypes.c_uint32 * 3)()
        return None if ctx.lib.pg_ulsch_demultiplex_sizes(ctypes.byref(s), out) else tuple(out)
    return f


def demux_gpu(ctx, cfgs, llrs):
    """One call over every configuration; returns per-configuration (sch, ack, csi) arrays."""
    import torch
    n = len(cfgs)
    arr = (uci_cases.PgUlschDemuxConfig * n)()
    off_in, offs = 0, [0, 0, 0]
    spans = []
    for i, (c, sizes) in enumerate(cfgs):
        s = uci_cases.to_struct(c)
        s.llr_offset = off_in
        s.sch_offset, s.harq_ack_offset, s.csi_part1_offset = offs
        arr[i] = s
        spans.append([(offs[k], sizes[k]) for k in range(3)])
        off_in += c["nof_llrs"]
        offs = [offs[k] + sizes[k] for k in range(3)]
    d_in = torch.from_numpy(np.concatenate(llrs)).cuda()
    outs = [torch.full((max(1, offs[k]),), 99, dtype=torch.int8, device="cuda") for k in range(3)]
    st = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_ulsch_demultiplex_device(ctx.handle, ctypes.addressof(arr), n, d_in.data_ptr(),
                                                  outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                                  st.cuda_stream))
    st.synchronize()
    host = [o.cpu().numpy() for o in outs]
    return [[host[k][o:o + n_] for k, (o, n_) in enumerate(sp)] for sp in spans]


def detect_gpu(ctx, cases):
    """cases: (K, qm, llrs); returns [(bits, valid)]."""
    import torch
    n = len(cases)
    items = (PgUciShortBlock * n)()
    off, out_off = 0, 0
    for i, (K, qm, llr) in enumerate(cases):
        items[i].llr_offset, items[i].nof_llrs, items[i].out_offset = off, llr.size, out_off
        items[i].nof_bits, items[i].modulation_order = K, qm
        off += llr.size
        out_off += K
    d_in = torch.from_numpy(np.concatenate([c[2] for c in cases])).cuda()
    d_bits = torch.full((out_off,), 7, dtype=torch.uint8, device="cuda")
    d_valid = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_uci_short_block_detect_device(ctx.handle, ctypes.addressof(items), n, d_in.data_ptr(),
                                                       d_bits.data_ptr(), d_valid.data_ptr(), st.cuda_stream))
    st.synchronize()
    bits, valid = d_bits.cpu().numpy(), d_valid.cpu().numpy()
    res, o = [], 0
    for i, (K, _, _) in enumerate(cases):
        res.append((bits[o:o + K], bool(valid[i])))
        o += K
    return res


def test_demux_matches_reference(ctx, ref):
    rng = np.random.default_rng(404)
    f = sizes_fn(ctx)
    cfgs = [uci_cases.random_config(rng, f) for _ in range(60)]
    llrs = [uci_cases.random_llrs(rng, c["nof_llrs"]) for c, _ in cfgs]
    got = demux_gpu(ctx, cfgs, llrs)
    kinds = set()
    for (c, _), llr, g in zip(cfgs, llrs, got):
        want = ref.ulsch_demultiplex(c, llr, block_size=int(rng.integers(100, 4000)))
        assert want[3]
        for k in range(3):
            assert np.array_equal(g[k], want[k]), (k, c)
        kinds.add((min(c["nof_harq_ack_bits"], 3), min(c["nof_csi_part1_bits"], 3), c["modulation_order"] > 1))
    # Every placeholder case was met: one-, two- and more-bit HARQ-ACK and CSI Part 1.
    assert {a for a, _, _ in kinds} >= {0, 1, 2, 3} and {b for _, b, _ in kinds} >= {0, 1, 2, 3}


def test_short_block_matches_reference(ctx, ref):
    rng = np.random.default_rng(11)
    cases = uci_cases.short_block_cases(rng, ref, 900)
    got = detect_gpu(ctx, cases)
    nvalid = 0
    for (K, qm, llr), (bits, ok) in zip(cases, got):
        wb, wok = ref.short_block_detect(K, llr, qm)
        assert ok == wok, (K, qm, llr.size)
        assert np.array_equal(bits, wb), (K, qm, llr.size)
        nvalid += ok
    assert 0.2 * len(cases) < nvalid < 0.95 * len(cases)  # both decisions are exercised


def test_uci_chain_matches_reference(ctx, ref):
    """GPU demultiplexing then GPU detection of HARQ-ACK and CSI Part 1, against the reference's
    demultiplexer then detector, on the same seeded soft bits."""
    rng = np.random.default_rng(77)
    f = sizes_fn(ctx)
    cfgs, llrs = [], []
    while len(cfgs) < 40:
        c, sizes = uci_cases.random_config(rng, f)
        if c["nof_harq_ack_bits"] == 0 and c["nof_csi_part1_bits"] == 0:
            continue
        cfgs.append((c, sizes))
        llrs.append(uci_cases.random_llrs(rng, c["nof_llrs"]) // 3)
    got = demux_gpu(ctx, cfgs, llrs)
    cases, want = [], []
    for (c, _), llr, g in zip(cfgs, llrs, got):
        w = ref.ulsch_demultiplex(c, llr)
        for k, bits_key in ((1, "nof_harq_ack_bits"), (2, "nof_csi_part1_bits")):
            K = c[bits_key]
            if K:
                assert np.array_equal(g[k], w[k])
                cases.append((K, c["modulation_order"], g[k]))
                want.append(ref.short_block_detect(K, w[k], c["modulation_order"]))
    res = detect_gpu(ctx, cases)
    for (bits, ok), (wb, wok) in zip(res, want):
        assert ok == wok and np.array_equal(bits, wb)


def test_invalid_inputs_rejected(ctx):
    import torch
    from pusch_b200._native import PgError
    d = torch.zeros(16, dtype=torch.int8, device="cuda")
    items = (PgUciShortBlock * 1)()
    items[0].nof_bits, items[0].modulation_order, items[0].nof_llrs = 12, 2, 16
    with pytest.raises(PgError):
        ctx.check(ctx.lib.pg_uci_short_block_detect_device(ctx.handle, ctypes.addressof(items), 1, d.data_ptr(),
                                                           d.data_ptr(), d.data_ptr(), None))
    c = dict(c_init=1, nof_harq_ack_rvd=0, nof_enc_harq_ack_bits=0, nof_enc_csi_part1_bits=0, nof_prb=4,
             dmrs_symbol_mask=0, modulation_order=2, nof_layers=1, start_symbol_index=0, nof_symbols=14,
             dmrs_type=1, nof_cdm_groups_without_data=2, nof_harq_ack_bits=0, nof_csi_part1_bits=0, nof_llrs=16)
    arr = (uci_cases.PgUlschDemuxConfig * 1)(uci_cases.to_struct(c))
    with pytest.raises(PgError):
        ctx.check(ctx.lib.pg_ulsch_demultiplex_device(ctx.handle, ctypes.addressof(arr), 1, d.data_ptr(),
                                                      d.data_ptr(), d.data_ptr(), d.data_ptr(), None))

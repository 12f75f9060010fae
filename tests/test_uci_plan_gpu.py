"""UCI on PUSCH inside slot plans (pg_pusch_plan_create_uci): per UE, the plan's UL-SCH results and
its HARQ-ACK / CSI Part 1 bits and validity equal those of the stage entries chained on the same
grid - pg_pusch_demodulate_device, pg_ulsch_demultiplex_device, pg_uci_short_block_detect_device
and the UL-SCH decoder on the demultiplexed stream - which tests/test_uci_gpu.py pins to the
reference's own demultiplexer and detector. UEs without UCI decode as in a plan without it."""
import ctypes

import numpy as np
import pytest

import uci_cases
from pusch_b200 import sim
from pusch_b200._native import PgPuschUci, PgUciShortBlock
from pusch_b200.pusch import PuschSlotPlan, batch_descriptors
from pusch_b200.sch import PuschDecoder, SchTransportBlock

pytestmark = pytest.mark.gpu
MAX_ITER = 6


def demux_config(ue, d, q, llr_offset, offs):
    """The demultiplexer configuration of UE ue (descriptor d) with UCI q, as the plan forms it."""
    c = dict(llr_offset=llr_offset, nof_llrs=sim.nof_ch_symbols(ue) * ue.modulation_order,
             sch_offset=offs[0], harq_ack_offset=offs[1], csi_part1_offset=offs[2],
             c_init=(ue.rnti << 15) + ue.n_id_data, nof_harq_ack_rvd=q.nof_harq_ack_rvd,
             nof_enc_harq_ack_bits=q.nof_enc_harq_ack_bits, nof_enc_csi_part1_bits=q.nof_enc_csi_part1_bits,
             nof_prb=ue.nof_rb, dmrs_symbol_mask=d.dmrs_symbol_mask,
             modulation_order=ue.modulation_order, nof_layers=ue.nof_layers, start_symbol_index=d.first_symbol,
             nof_symbols=d.nof_symbols, dmrs_type=1, nof_cdm_groups_without_data=q.nof_cdm_groups_without_data,
             nof_harq_ack_bits=q.nof_harq_ack_bits, nof_csi_part1_bits=q.nof_csi_part1_bits)
    return c


def sizes_of(ctx, c):
    out = (ctypes.c_uint32 * 3)()
    s = uci_cases.to_struct(c)
    return None if ctx.lib.pg_ulsch_demultiplex_sizes(ctypes.byref(s), out) else tuple(out)


def random_uci(ctx, rng, ues, descs):
    """UCI for about two thirds of the UEs: HARQ-ACK of 1-11 bits (reserved REs for 1-2 bits) and CSI
    Part 1 of 0-11 bits, a few to a few tens of REs each."""
    out = []
    for ue, d in zip(ues, descs):
        q = PgPuschUci()
        if rng.random() < 0.67:
            bpr = ue.modulation_order * ue.nof_layers
            q.nof_harq_ack_bits = int(rng.choice([1, 2, 3, 5, 11]))
            q.nof_csi_part1_bits = int(rng.choice([0, 0, 4, 8, 11]))
            a = int(rng.integers(2, 40))
            q.nof_enc_harq_ack_bits = bpr * a
            q.nof_harq_ack_rvd = bpr * (a + int(rng.integers(0, 10))) if q.nof_harq_ack_bits <= 2 else 0
            q.nof_enc_csi_part1_bits = bpr * int(rng.integers(4, 80)) if q.nof_csi_part1_bits else 0
            q.nof_cdm_groups_without_data = 2
            if sizes_of(ctx, demux_config(ue, d, q, 0, (0, 0, 0))) is None:
                q = PgPuschUci()
        out.append(q)
    return out


def test_plan_uci_matches_stage_chain(ctx):
    import torch
    rng = np.random.default_rng(21)
    slots = sim.uneven_cells(seed=11, nof_cells=3)
    descs, grid, tb_bytes, ues = batch_descriptors(slots, max_iterations=MAX_ITER)
    ucis = random_uci(ctx, rng, ues, descs)
    assert sum(1 for q in ucis if q.nof_harq_ack_bits) >= 5

    plan = PuschSlotPlan(ctx, slots, max_iterations=MAX_ITER, uci=ucis)
    got = plan.execute_host()
    ures = plan.uci_results()
    plan.close()
    plain = PuschSlotPlan(ctx, slots, max_iterations=MAX_ITER)
    got_plain = plain.execute_host()
    plain.close()

    # Stage chain: codeword LLRs of every UE, then the UCI UEs' demultiplexing and detection.
    n = len(ues)
    llr_off, est_off, nllr, nest = [], [], 0, 0
    for d, ue in zip(descs, ues):
        d.llr_offset, d.est_offset = nllr, nest
        llr_off.append(nllr)
        nllr += sim.nof_ch_symbols(ue) * ue.modulation_order
        nest += d.nof_rx_ports * len(ue.dmrs_symbols) * ue.nof_layers * 12 * ue.nof_rb
    st = torch.cuda.current_stream()
    d_grid = torch.from_numpy(grid.view(np.int32)).cuda()
    d_est = torch.zeros(2 * nest, dtype=torch.float32, device="cuda")
    d_pr = torch.zeros(n * 4 * 5, dtype=torch.float32, device="cuda")
    d_llr = torch.zeros(nllr, dtype=torch.int8, device="cuda")
    ctx.check(ctx.lib.pg_pusch_estimate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                               d_est.data_ptr(), d_pr.data_ptr(), st.cuda_stream))
    ctx.check(ctx.lib.pg_pusch_demodulate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                                 d_est.data_ptr(), d_pr.data_ptr(), d_llr.data_ptr(), st.cuda_stream))
    sel = [i for i, q in enumerate(ucis) if q.nof_harq_ack_bits or q.nof_csi_part1_bits]
    cfgs, spans, offs = [], [], [0, 0, 0]
    for i in sel:
        c = demux_config(ues[i], descs[i], ucis[i], llr_off[i], tuple(offs))
        sz = sizes_of(ctx, c)
        cfgs.append(c)
        spans.append([(offs[k], sz[k]) for k in range(3)])
        offs = [offs[k] + sz[k] for k in range(3)]
    arr = (uci_cases.PgUlschDemuxConfig * len(cfgs))(*[uci_cases.to_struct(c) for c in cfgs])
    outs = [torch.zeros(max(1, offs[k]), dtype=torch.int8, device="cuda") for k in range(3)]
    ctx.check(ctx.lib.pg_ulsch_demultiplex_device(ctx.handle, ctypes.addressof(arr), len(cfgs), d_llr.data_ptr(),
                                                  outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                                  st.cuda_stream))
    msgs, keys = [], []
    for j, i in enumerate(sel):
        for k, nbits in ((1, ucis[i].nof_harq_ack_bits), (2, ucis[i].nof_csi_part1_bits)):
            if nbits:
                msgs.append((k, spans[j][k], nbits, ues[i].modulation_order))
                keys.append((i, k))
    items = (PgUciShortBlock * len(msgs))()
    stream_llr = torch.cat([outs[1], outs[2]])
    out_off = 0
    for m, (k, (o, e), nbits, qm) in enumerate(msgs):
        items[m].llr_offset = o if k == 1 else offs[1] + o
        items[m].nof_llrs, items[m].out_offset, items[m].nof_bits, items[m].modulation_order = e, out_off, nbits, qm
        out_off += nbits
    d_bits = torch.zeros(max(1, out_off), dtype=torch.uint8, device="cuda")
    d_valid = torch.zeros(max(1, len(msgs)), dtype=torch.uint8, device="cuda")
    ctx.check(ctx.lib.pg_uci_short_block_detect_device(ctx.handle, ctypes.addressof(items), len(msgs),
                                                       stream_llr.data_ptr(), d_bits.data_ptr(), d_valid.data_ptr(),
                                                       st.cuda_stream))
    st.synchronize()
    bits, valid = d_bits.cpu().numpy(), d_valid.cpu().numpy()
    sch_host = outs[0].cpu().numpy()

    o = 0
    for m, ((i, k), (_, _, nbits, _)) in enumerate(zip(keys, msgs)):
        r = ures[i]
        want = bits[o:o + nbits]
        o += nbits
        if k == 1:
            assert np.array_equal(np.array(r.harq_ack[:nbits]), want), i
            assert r.harq_ack_valid == valid[m], i
        else:
            assert np.array_equal(np.array(r.csi_part1[:nbits]), want), i
            assert r.csi_part1_valid == valid[m], i
    for i, q in enumerate(ucis):
        if not q.nof_harq_ack_bits:
            assert ures[i].harq_ack_valid == 0
        if not q.nof_csi_part1_bits:
            assert ures[i].csi_part1_valid == 0

    # UL-SCH: UCI UEs decode the demultiplexed stream, the others are unchanged by UCI elsewhere.
    tbs = [SchTransportBlock(sch_host[spans[j][0][0]:spans[j][0][0] + spans[j][0][1]].copy(), ues[i].tbs_bits,
                             ues[i].base_graph, ues[i].modulation_order, ues[i].nof_layers, rv=ues[i].rv,
                             max_iterations=MAX_ITER) for j, i in enumerate(sel)]
    res = PuschDecoder(ctx).decode_batch(tbs)
    for j, i in enumerate(sel):
        g, w = got[i], res[j]
        assert g.tb_crc_ok == w.tb_crc_ok, i
        assert g.nof_codeblocks == w.nof_codeblocks_total, i
        assert g.nof_codeblocks_crc_ok == w.nof_codeblocks_crc_ok, i
        assert g.mean_iterations == w.mean_iterations, i
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, w.transport_block), i
    for i in range(n):
        if i not in sel:
            a, b = got[i], got_plain[i]
            assert a.tb_crc_ok == b.tb_crc_ok and a.mean_iterations == b.mean_iterations, i
            if a.tb_crc_ok:
                assert np.array_equal(a.transport_block, b.transport_block), i


def test_plan_uci_rejects_inconsistent_configuration(ctx):
    slots = sim.uneven_cells(seed=12, nof_cells=1)
    _, _, _, ues = batch_descriptors(slots, max_iterations=MAX_ITER)
    ucis = [PgPuschUci() for _ in ues]
    ucis[0].nof_harq_ack_bits = 5
    ucis[0].nof_enc_harq_ack_bits = 10 ** 7  # far more soft bits than the allocation has
    ucis[0].nof_cdm_groups_without_data = 2
    from pusch_b200._native import PgError
    with pytest.raises(PgError):
        PuschSlotPlan(ctx, slots, max_iterations=MAX_ITER, uci=ucis)


def test_plan_polar_uci_matches_stage_chain(ctx):
    """Polar-coded HARQ-ACK and CSI Part 1 (12 to 200 bits) inside a plan: every message's bits and
    validity (pg_pusch_plan_uci_message) equal the stage chain's - pg_ulsch_demultiplex_device on
    the demodulated codewords, then pg_uci_polar_decode_device (tests/test_uci_polar_gpu.py pins it
    to the reference's uci_decoder)."""
    import torch
    from pusch_b200.uci import PolarUciDecoder
    rng = np.random.default_rng(5)
    slots = sim.uneven_cells(seed=13, nof_cells=2)
    descs, grid, tb_bytes, ues = batch_descriptors(slots, max_iterations=MAX_ITER)
    ucis = []
    for ue, d in zip(ues, descs):
        q = PgPuschUci()
        if rng.random() < 0.7:
            bpr = ue.modulation_order * ue.nof_layers
            q.nof_harq_ack_bits = int(rng.choice([3, 12, 20, 40]))
            q.nof_csi_part1_bits = int(rng.choice([0, 19, 64, 200]))
            enc = lambda A: 0 if A == 0 else bpr * (-(-2 * (A + 14) // bpr) + int(rng.integers(0, 20)))
            q.nof_enc_harq_ack_bits = enc(q.nof_harq_ack_bits)
            q.nof_enc_csi_part1_bits = enc(q.nof_csi_part1_bits)
            q.nof_cdm_groups_without_data = 2
            if sizes_of(ctx, demux_config(ue, d, q, 0, (0, 0, 0))) is None:
                q = PgPuschUci()
        ucis.append(q)
    plan = PuschSlotPlan(ctx, slots, max_iterations=MAX_ITER, uci=ucis)
    plan.execute_host()
    sel = [i for i, q in enumerate(ucis) if q.nof_harq_ack_bits or q.nof_csi_part1_bits]
    msgs = [(i, k, n) for i in sel for k, n in ((0, ucis[i].nof_harq_ack_bits), (1, ucis[i].nof_csi_part1_bits))
            if n > 11]
    assert len(msgs) >= 8
    plan_out = {(i, k): plan.uci_message(i, k, n) for i, k, n in msgs}
    plan.close()

    n = len(ues)
    llr_off, nllr, nest = [], 0, 0
    for d, ue in zip(descs, ues):
        d.llr_offset, d.est_offset = nllr, nest
        llr_off.append(nllr)
        nllr += sim.nof_ch_symbols(ue) * ue.modulation_order
        nest += d.nof_rx_ports * len(ue.dmrs_symbols) * ue.nof_layers * 12 * ue.nof_rb
    st = torch.cuda.current_stream()
    d_grid = torch.from_numpy(grid.view(np.int32)).cuda()
    d_est = torch.zeros(2 * nest, dtype=torch.float32, device="cuda")
    d_pr = torch.zeros(n * 4 * 5, dtype=torch.float32, device="cuda")
    d_llr = torch.zeros(nllr, dtype=torch.int8, device="cuda")
    ctx.check(ctx.lib.pg_pusch_estimate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                               d_est.data_ptr(), d_pr.data_ptr(), st.cuda_stream))
    ctx.check(ctx.lib.pg_pusch_demodulate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                                 d_est.data_ptr(), d_pr.data_ptr(), d_llr.data_ptr(), st.cuda_stream))
    cfgs, spans, offs = [], {}, [0, 0, 0]
    for i in sel:
        c = demux_config(ues[i], descs[i], ucis[i], llr_off[i], tuple(offs))
        sz = sizes_of(ctx, c)
        cfgs.append(c)
        spans[i] = [(offs[k], sz[k]) for k in range(3)]
        offs = [offs[k] + sz[k] for k in range(3)]
    arr = (uci_cases.PgUlschDemuxConfig * len(cfgs))(*[uci_cases.to_struct(c) for c in cfgs])
    outs = [torch.zeros(max(1, offs[k]), dtype=torch.int8, device="cuda") for k in range(3)]
    ctx.check(ctx.lib.pg_ulsch_demultiplex_device(ctx.handle, ctypes.addressof(arr), len(cfgs), d_llr.data_ptr(),
                                                  outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                                  st.cuda_stream))
    st.synchronize()
    streams = [outs[1].cpu().numpy(), outs[2].cpu().numpy()]
    chain = PolarUciDecoder(ctx).decode([(nb, streams[k][spans[i][1 + k][0]:spans[i][1 + k][0] + spans[i][1 + k][1]])
                                         for i, k, nb in msgs])
    # The simulator carries no UCI in these REs (their soft bits are UL-SCH data), so the CRCs fail;
    # the decoders' bits are still a function of the soft bits and must agree message by message.
    for (i, k, nb), (bits, ok) in zip(msgs, chain):
        pb, pok = plan_out[(i, k)]
        assert pok == ok, (i, k)
        assert np.array_equal(pb, bits), (i, k)

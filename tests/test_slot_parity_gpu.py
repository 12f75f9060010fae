"""Slot-level parity with the reference's CPU receive path.

The reference side is oracle/_ref's ref_pusch_decode_detail: the reference's own stage objects in
pusch_processor order (lib/phy/upper/channel_processors/pusch/pusch_processor_impl.cpp:349-900):
port_channel_estimator, get_symbol_ch_estimate, channel_equalizer, demodulation_mapper,
descrambling, ldpc_segmenter_rx, ldpc_rate_dematcher, ldpc_decoder with CRC early stop, TB join.
The GPU side is the slot plan with the plain estimator. Slots are the simulator's seed-0 slots of
the three slot configurations: 20 MHz single UE (QPSK, 1 layer, 2 rx), the 100 MHz full cell
(256QAM, 2 layers, 4 rx, 50 codeblocks) and the 16-cell uneven slot (154 UEs, QPSK-256QAM).

Checks, per configuration:
- the whole path: per UE the TB CRC flag, the codeblock count, the codeblocks that pass their
  CRC, the mean LDPC iterations (pusch_decoder_result) and the TB bits equal the reference's;
- the front end: the descrambled codeword LLRs (the soft bits pusch_processor hands to
  pusch_decoder) within +-1 LSB of the reference's;
- the fused demodulator fed the reference's own channel estimates and noise variances: LLRs
  within +-1 LSB of the reference's equaliser + demapper + descrambler for every modulation;
- the back half fed the reference's LLRs: segmentation, rate dematching, LDPC and TB assembly give
  bit-exact TBs, CRC flags and per-codeblock iteration counts, both through the TB-level entry
  (pg_sch_decode_batch_host) and through the stage entries (rate dematcher, LDPC batch decoder).
"""
import ctypes
import os

import numpy as np
import pytest

from pusch_b200 import sch, sim
from pusch_b200.ldpc import CodeblockJob, LdpcBatchDecoder, LdpcDecoderConfiguration
from pusch_b200.pusch import PgPortResult, PuschSlotPlan, batch_descriptors
from pusch_b200.sch import LdpcRateDematcher, PuschDecoder, RmConfig, SchTransportBlock

pytestmark = pytest.mark.gpu
MAX_ITER = 6
PG_CRC16, PG_CRC24A, PG_CRC24B = 0, 1, 2

CASES = {
    "c1_20mhz_qpsk_1layer_2rx": lambda: [sim.single_ue_slot(seed=0)],
    "c3_100mhz_256qam_2layer_4rx": lambda: [sim.full_cell_slot(seed=0)],
    "c4_16cell_uneven": lambda: sim.uneven_cells(seed=0, nof_cells=16),
}


def assign_offsets(descs, ues):
    """Batch-wide LLR and channel-estimate offsets (one buffer for every UE of every cell)."""
    llr, est = 0, 0
    for d, ue in zip(descs, ues):
        d.llr_offset, d.est_offset = llr, est
        llr += sim.nof_ch_symbols(ue) * ue.modulation_order
        est += d.nof_rx_ports * len(ue.dmrs_symbols) * ue.nof_layers * 12 * ue.nof_rb
    return llr, est


@pytest.fixture(scope="module", params=list(CASES))
def slot_case(request, ref):
    slots = CASES[request.param]()
    descs, grid, tb_bytes, ues = batch_descriptors(slots, max_iterations=MAX_ITER)
    nllr, nest = assign_offsets(descs, ues)
    r = ref.pusch_decode_detail(descs, grid, tb_bytes, nllr, os.cpu_count() or 1)
    return dict(name=request.param, slots=slots, descs=descs, grid=grid, tb_bytes=tb_bytes, ues=ues, nllr=nllr,
                nest=nest, ref=r)


def tb_of(buf, d):
    return buf[d.tb_out_offset:d.tb_out_offset + d.tbs_bits // 8]


def test_plan_matches_reference_chain(ctx, slot_case):
    c, r = slot_case, slot_case["ref"]
    plan = PuschSlotPlan(ctx, c["slots"], max_iterations=MAX_ITER)
    got = plan.execute_host()
    plan.close()
    truth = [t for sl in c["slots"] for t in sl.truth]
    assert len(got) == len(c["ues"])
    for u, (g, d) in enumerate(zip(got, c["descs"])):
        cb_ok = int((r["cb_iters"][u] > 0).sum())
        assert g.tb_crc_ok == bool(r["ok"][u]), (c["name"], u)
        assert g.nof_codeblocks == int(r["nof_cbs"][u]), (c["name"], u)
        assert g.nof_codeblocks_crc_ok == cb_ok, (c["name"], u)
        assert g.mean_iterations == float(r["mean_iters"][u]), (c["name"], u, g.mean_iterations, r["mean_iters"][u])
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, tb_of(r["tb"], d)), (c["name"], u)
            assert np.array_equal(np.unpackbits(g.transport_block), truth[u])
    # The configurations' slots decode (the reference decodes every UE of them).
    assert all(r["ok"])


def gpu_front_end(ctx, c, est_in=None, noise_in=None):
    """Codeword LLRs of every UE through pg_pusch_estimate_device and pg_pusch_demodulate_device
    (the plan's estimation and fused demodulation kernels). est_in / noise_in replace the GPU
    estimates and port noise variances (the reference's, to test the demodulator alone)."""
    import torch
    lib, descs = ctx.lib, c["descs"]
    n = len(descs)
    s = torch.cuda.current_stream()
    d_grid = torch.from_numpy(c["grid"].view(np.int32)).cuda()
    d_est = torch.zeros(2 * max(c["nest"], 1), dtype=torch.float32, device="cuda")
    d_pr = torch.zeros(n * 4 * 5, dtype=torch.float32, device="cuda")
    ctx.check(lib.pg_pusch_estimate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(), d_est.data_ptr(),
                                           d_pr.data_ptr(), s.cuda_stream))
    if est_in is not None:
        d_est.copy_(torch.from_numpy(est_in.view(np.float32)))
        pr = d_pr.cpu().numpy().reshape(n, 4, 5)
        pr[:, :, 0] = noise_in
        d_pr.copy_(torch.from_numpy(pr.ravel()))
    d_llr = torch.zeros(max(c["nllr"], 1), dtype=torch.int8, device="cuda")
    ctx.check(lib.pg_pusch_demodulate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                             d_est.data_ptr(), d_pr.data_ptr(), d_llr.data_ptr(), s.cuda_stream))
    s.synchronize()
    return d_llr.cpu().numpy()[:c["nllr"]].astype(np.int16)


def per_modulation(c, diff):
    out = {}
    for d, ue in zip(c["descs"], c["ues"]):
        g = sim.nof_ch_symbols(ue) * ue.modulation_order
        out.setdefault(ue.modulation_order, []).append(diff[d.llr_offset:d.llr_offset + g])
    return {qm: np.concatenate(v) for qm, v in out.items()}


# Largest LLR difference of the whole front end per modulation order. The GPU estimator's FP32
# responses differ from the reference's in the last bits (summation order), so after the bf16
# rounding of the per-symbol estimates a small fraction of the channel coefficients are one bf16
# unit (2^-8 relative) apart; an LLR that is not saturated moves with such a coefficient by a
# fraction of an LSB for QPSK and by a few LSB for the denser constellations (256QAM: slope up to
# 8/sqrt(170) per 1/noise variance at 25 dB, 6 LSB per LLR unit). With the reference's own estimates
# the demodulator is within +-1 LSB for every order (test_fused_demodulator_on_reference_estimates).
FRONT_END_MAX_DIFF = {2: 1, 4: 2, 6: 2, 8: 8}


def test_front_end_llrs_match_reference(ctx, slot_case):
    c, r = slot_case, slot_case["ref"]
    got = gpu_front_end(ctx, c)
    diff = np.abs(got - r["llrs"][:c["nllr"]].astype(np.int16))
    for qm, d in per_modulation(c, diff).items():
        stats = (c["name"], qm, int(d.max()), float((d == 0).mean()), float((d <= 1).mean()))
        assert d.max() <= FRONT_END_MAX_DIFF[qm], stats
        assert (d == 0).mean() > 0.99, stats
        assert (d <= 1).mean() > 0.9999, stats


def test_fused_demodulator_on_reference_estimates(ctx, ref, slot_case):
    """pusch_demod_kernel (time interpolation, bf16 rounding, equalisation, demapping, descrambling)
    given the reference estimator's FP32 frequency responses and noise variances: every LLR within
    +-1 LSB of the reference's chain, for every modulation of the slot."""
    c, r = slot_case, slot_case["ref"]
    est = np.zeros(max(c["nest"], 1), np.complex64)
    noise = np.zeros((len(c["descs"]), 4), np.float32)
    for u, d in enumerate(c["descs"]):
        grid = c["grid"][d.grid_offset:d.grid_offset + d.nof_rx_ports * 14 * d.grid_nof_subc].reshape(
            d.nof_rx_ports, 14, d.grid_nof_subc)
        dm = [s for s in range(14) if (d.dmrs_symbol_mask >> s) & 1]
        per_port = len(dm) * d.nof_layers * 12 * d.nof_rb
        for p in range(d.nof_rx_ports):
            freq, _, sc = ref.port_estimate(grid, p, d.slot, d.n_id, d.rb_start, d.nof_rb, d.nof_layers, dm,
                                            d.dmrs_scaling)
            est[d.est_offset + p * per_port:d.est_offset + (p + 1) * per_port] = freq.ravel()
            noise[u, p] = sc["noise_var"]
    got = gpu_front_end(ctx, c, est, noise)
    diff = np.abs(got - r["llrs"][:c["nllr"]].astype(np.int16))
    for qm, d in per_modulation(c, diff).items():
        assert d.max() <= 1, (c["name"], qm, int(d.max()))
        assert (d == 0).mean() > 0.995, (c["name"], qm, float((d == 0).mean()))


def test_back_half_bit_exact_on_reference_llrs(ctx, slot_case):
    """The reference's codeword LLRs through the GPU's UL-SCH decoder: TB, CRC flag, codeblock
    counts and mean iterations equal to the reference's (pg_sch_decode_batch_host), and every
    codeblock's iteration count equal through the stage entries."""
    c, r = slot_case, slot_case["ref"]
    llrs = r["llrs"]
    tbs = []
    for d, ue in zip(c["descs"], c["ues"]):
        g = sim.nof_ch_symbols(ue) * ue.modulation_order
        tbs.append(SchTransportBlock(llrs[d.llr_offset:d.llr_offset + g].copy(), ue.tbs_bits, ue.base_graph,
                                     ue.modulation_order, ue.nof_layers, rv=ue.rv, max_iterations=MAX_ITER))
    res = PuschDecoder(ctx).decode_batch(tbs)
    for u, (g, d) in enumerate(zip(res, c["descs"])):
        assert g.tb_crc_ok == bool(r["ok"][u]), (c["name"], u)
        assert g.nof_codeblocks_total == int(r["nof_cbs"][u])
        assert g.nof_codeblocks_crc_ok == int((r["cb_iters"][u] > 0).sum())
        assert g.mean_iterations == float(r["mean_iters"][u])
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, tb_of(r["tb"], d))

    # The same soft bits scrambled again and left in device memory: the resident entry descrambles
    # them on the device and decodes the same TBs.
    import torch
    from pusch_b200 import prg
    scrambled = llrs[:c["nllr"]].astype(np.int16).copy()
    c_init = []
    for d, ue in zip(c["descs"], c["ues"]):
        g = sim.nof_ch_symbols(ue) * ue.modulation_order
        seq = prg.scrambling(ue.rnti, ue.n_id_data, g).astype(bool)
        seg_llr = scrambled[d.llr_offset:d.llr_offset + g]
        seg_llr[seq] = -seg_llr[seq]
        c_init.append((ue.rnti << 15) + ue.n_id_data)
    d_llrs = torch.from_numpy(scrambled.astype(np.int8)).cuda()
    res_r = PuschDecoder(ctx).decode_resident(tbs, [d.llr_offset for d in c["descs"]], d_llrs.data_ptr(), c["nllr"],
                                              c_init=c_init)
    for u, (g, w) in enumerate(zip(res_r, res)):
        assert (g.tb_crc_ok, g.nof_codeblocks_crc_ok, g.mean_iterations) == (
            w.tb_crc_ok, w.nof_codeblocks_crc_ok, w.mean_iterations), (c["name"], u)
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, w.transport_block)

    # Per codeblock: segmentation (pg_sch_segment), the rate dematcher and the LDPC batch decoder.
    dem, dec = LdpcRateDematcher(ctx), LdpcBatchDecoder(context=ctx)
    jobs, want = [], []
    for u, (t, ue) in enumerate(zip(tbs, c["ues"])):
        seg = sch.segment(t.tbs_bits, t.base_graph, t.modulation_order, t.nof_layers,
                          t.llrs.size // t.modulation_order)
        z, f = seg["lifting_size"], seg["nof_filler_bits"]
        n = (66 if t.base_graph == 1 else 50) * z
        poly = PG_CRC24B if seg["nof_cbs"] > 1 else (PG_CRC16 if t.tbs_bits <= 3824 else PG_CRC24A)
        items, off = [], 0
        for k in range(seg["nof_cbs"]):
            e = seg["e_short"] if k < seg["nof_short_cbs"] else seg["e_long"]
            items.append((t.llrs[off:off + e], np.zeros(n, np.int8), True,
                          RmConfig(t.base_graph, z, t.rv, t.modulation_order, 0, f)))
            off += e
        dem.rate_dematch_batch(items)
        for buf in (x[1] for x in items):
            cfg = LdpcDecoderConfiguration(t.base_graph, z, f, 16 if poly == PG_CRC16 else 24, MAX_ITER)
            jobs.append(CodeblockJob(buf, cfg, poly))
        want.extend(int(x) for x in r["cb_iters"][u])
    _, iters = dec.decode_batch(jobs)
    assert [int(x) for x in iters] == want, c["name"]

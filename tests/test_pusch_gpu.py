"""GPU PUSCH slot stages against the reference: DM-RS channel estimation (internal FP32 response,
port scalars and the bf16 per-symbol estimates), demodulation (LLRs of the reference's equaliser,
demapper and descrambling fed with the reference's estimates) and the whole receive path."""
import ctypes

import numpy as np
import pytest

import golden_io
from fp64 import estimate_port_fp64, gold_sequence, rel_err
from pusch_b200 import sim
from pusch_b200.pusch import PuschProcessor, make_ue_descriptors

pytestmark = pytest.mark.gpu
BETA = float(np.float32(10 ** (3 / 20)))
EST_REL_TOL = 1e-4


def golden_slot(c):
    ue = sim.PuschUe(rb_start=c["rb_start"], nof_rb=c["nof_rb"], nof_layers=c["nof_layers"], modulation_order=2,
                     tbs_bits=24, base_graph=2, dmrs_symbols=tuple(c["dmrs"]), n_id=c["n_id"], rnti=c["rnti"])
    return sim.PuschSlot(c["grid"], [ue], [None], c["ports"], c["grid"].shape[2] // 12, c["slot"], 30, BETA)


def run_estimator(ctx, slot):
    import torch
    lib = ctx.lib
    descs, nllr, nest, _ = make_ue_descriptors(slot)
    n = len(slot.ues)
    d_grid = torch.from_numpy(np.ascontiguousarray(slot.grid, np.uint32).view(np.int32).ravel()).cuda()
    d_est = torch.zeros(2 * max(nest, 1), dtype=torch.float32, device="cuda")
    d_pr = torch.zeros(n * 4 * 5, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    rc = lib.pg_pusch_estimate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(), d_est.data_ptr(),
                                      d_pr.data_ptr(), s.cuda_stream)
    ctx.check(rc)
    s.synchronize()
    return descs, d_grid, d_est, d_pr


def test_estimator_matches_reference(ctx):
    for c in golden_io.est_cases():
        slot = golden_slot(c)
        descs, _, d_est, d_pr = run_estimator(ctx, slot)
        nd, nl, nsc = len(c["dmrs"]), c["nof_layers"], 12 * c["nof_rb"]
        est = d_est.cpu().numpy().view(np.complex64)[:c["ports"] * nd * nl * nsc].reshape(c["ports"], nd, nl, nsc)
        pr = d_pr.cpu().numpy().reshape(-1, 4, 5)[0]
        cfg = dict(nof_layers=nl, scaling=BETA, rb_start=c["rb_start"], nof_rb=c["nof_rb"], dmrs_symbols=c["dmrs"],
                   slot=c["slot"], n_id=c["n_id"])
        for p in range(c["ports"]):
            e64 = estimate_port_fp64(c["grid"], p, cfg)
            assert rel_err(est[p], e64["freq"]).max() < EST_REL_TOL, (c["nof_rb"], p)
            assert rel_err(est[p], c["freq"][p]).max() < EST_REL_TOL, (c["nof_rb"], p)
            nv, epre, snr, *rsrp = c["scalars"][p]
            g_nv, g_epre, g_snr, g_r0, g_r1 = pr[p]
            for got, want in ((g_nv, nv), (g_epre, epre), (g_snr, snr), (g_r0, rsrp[0])):
                assert abs(got - want) / abs(want) < EST_REL_TOL
            if nl > 1:
                assert abs(g_r1 - rsrp[1]) / abs(rsrp[1]) < EST_REL_TOL


def test_symbol_estimates_match_reference_bf16(ctx):
    import torch
    for c in golden_io.est_cases():
        slot = golden_slot(c)
        descs, _, d_est, _ = run_estimator(ctx, slot)
        nl, nsc = c["nof_layers"], 12 * c["nof_rb"]
        d_sym = torch.zeros(c["ports"] * 14 * nl * nsc, dtype=torch.int32, device="cuda")
        s = torch.cuda.current_stream()
        rc = ctx.lib.pg_pusch_symbol_estimates_device(ctx.handle, ctypes.addressof(descs), d_est.data_ptr(), None,
                                                      d_sym.data_ptr(), s.cuda_stream)
        ctx.check(rc)
        s.synchronize()
        got = d_sym.cpu().numpy().view(np.uint32).reshape(c["ports"], 14, nl, nsc)
        for p in range(c["ports"]):
            want = c["sym"][p]
            # bf16 values: equal, or one unit in the last place apart where the FP32 values straddle a
            # rounding boundary.
            for part in (0, 16):
                a = ((got[p] >> part) & 0xFFFF).astype(np.int32)
                b = ((want >> part) & 0xFFFF).astype(np.int32)
                d = np.abs(a - b)
                assert d.max() <= 1, (c["nof_rb"], p)
                assert (d == 0).mean() > 0.99


def oracle_demod(ref, c, sym_est, scalars):
    """The reference's equaliser and demapper on the reference's estimates, then descrambling."""
    nl, ports, nsc = c["nof_layers"], c["ports"], 12 * c["nof_rb"]
    noise = np.array([s[0] for s in scalars], np.float32)
    sc = slice(12 * c["rb_start"], 12 * (c["rb_start"] + c["nof_rb"]))
    llrs = []
    for s in range(14):
        if s in c["dmrs"]:
            continue
        y = np.ascontiguousarray(c["grid"][:, s, sc])
        h = np.ascontiguousarray(np.stack([sym_est[p][s] for p in range(ports)]))
        eq, var = ref.equalize(1, y, h, noise, 1.0)
        llrs.append(ref.demodulate_soft(c["qm"], eq.ravel(), var.ravel()))
    llr = np.concatenate(llrs).astype(np.int16)
    seq = gold_sequence((c["rnti"] << 15) + 0, llr.size)
    return np.where(seq == 1, -llr, llr).astype(np.int8)


@pytest.mark.parametrize("qm", [2, 4, 6, 8])
def test_demodulator_matches_reference_chain(ctx, ref, qm):
    """The fused demodulator given the reference estimator's FP32 frequency responses and noise
    variances (golden fixtures, up to 273 PRB x 4 ports x 2 layers): every LLR within +-1 LSB of
    the reference's equaliser + demapper on the reference's bf16 symbol estimates, descrambled."""
    import torch
    for c in golden_io.est_cases():
        c = dict(c, qm=qm)
        slot = golden_slot(c)
        descs, d_grid, d_est, d_pr = run_estimator(ctx, slot)
        descs[0].modulation_order = qm
        nd, nl, nsc = len(c["dmrs"]), c["nof_layers"], 12 * c["nof_rb"]
        est = np.stack([c["freq"][p] for p in range(c["ports"])]).astype(np.complex64).ravel()
        d_est[:2 * est.size] = torch.from_numpy(est.view(np.float32)).cuda()
        pr = d_pr.cpu().numpy().reshape(-1, 4, 5)
        pr[0, :c["ports"], 0] = [sc[0] for sc in c["scalars"]]
        d_pr.copy_(torch.from_numpy(pr.ravel()))
        nllr = (14 - nd) * nsc * nl * qm
        d_llr = torch.zeros(nllr, dtype=torch.int8, device="cuda")
        s = torch.cuda.current_stream()
        rc = ctx.lib.pg_pusch_demodulate_device(ctx.handle, ctypes.addressof(descs), 1, d_grid.data_ptr(),
                                                d_est.data_ptr(), d_pr.data_ptr(), d_llr.data_ptr(), s.cuda_stream)
        ctx.check(rc)
        s.synchronize()
        got = d_llr.cpu().numpy().astype(int)
        want = oracle_demod(ref, c, c["sym"], c["scalars"]).astype(int)
        d = np.abs(got - want)
        assert d.max() <= 1, (c["nof_rb"], qm, int(d.max()))
        assert (d == 0).mean() > 0.99, (c["nof_rb"], qm)


@pytest.mark.parametrize("name", ["20MHz_qpsk_1layer_2rx", "100MHz_256qam_2layer_4rx", "small_16qam"])
def test_pusch_chain_decodes(ctx, name):
    if name == "20MHz_qpsk_1layer_2rx":
        ue = sim.PuschUe(rb_start=0, nof_rb=51, nof_layers=1, modulation_order=2, tbs_bits=5888, base_graph=1,
                         dmrs_symbols=(2,), snr_db=10.0, channel="flat")
        slot = sim.make_pusch_slot([ue], 2, nof_prb_grid=51, seed=11)
    elif name == "100MHz_256qam_2layer_4rx":
        ue = sim.PuschUe(rb_start=0, nof_rb=273, nof_layers=2, modulation_order=8, tbs_bits=417976, base_graph=1,
                         dmrs_symbols=(2, 11), snr_db=30.0, channel="pdp")
        slot = sim.make_pusch_slot([ue], 4, nof_prb_grid=273, seed=12)
    else:
        ue = sim.PuschUe(rb_start=7, nof_rb=6, nof_layers=1, modulation_order=4, tbs_bits=1320, base_graph=2,
                         dmrs_symbols=(2, 11), snr_db=15.0, channel="pdp")
        slot = sim.make_pusch_slot([ue], 2, nof_prb_grid=30, seed=13)
    res = PuschProcessor(ctx).process_slots([slot], max_iterations=10)[0]
    assert res.tb_crc_ok, name
    assert (np.unpackbits(res.transport_block) == slot.truth[0]).all()


def test_pusch_multi_cell_batch(ctx):
    slots = []
    for cell in range(3):
        ues = [sim.PuschUe(rb_start=0, nof_rb=40, nof_layers=1, modulation_order=4, tbs_bits=10248,
                           base_graph=1, dmrs_symbols=(2,), snr_db=18.0, channel="flat", rnti=100 + cell),
               sim.PuschUe(rb_start=40, nof_rb=20, nof_layers=2, modulation_order=6, tbs_bits=16392, base_graph=1,
                           dmrs_symbols=(2, 11), snr_db=28.0, channel="pdp", rnti=200 + cell)]
        slots.append(sim.make_pusch_slot(ues, 4, nof_prb_grid=60, slot=cell, seed=40 + cell))
    res = PuschProcessor(ctx).process_slots(slots, max_iterations=10)
    truth = [t for sl in slots for t in sl.truth]
    for r, t in zip(res, truth):
        assert r.tb_crc_ok
        assert (np.unpackbits(r.transport_block) == t).all()

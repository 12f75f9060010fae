"""HARQ soft combining in slot plans (pg_pusch_plan_set_harq): a retransmission with another
redundancy version is combined into the codeblock buffers the plan kept from the first
transmission (the reference's rate-dematch soft buffer,
lib/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher_impl.cpp:98-194, held per HARQ process by
lib/phy/upper/rx_buffer_pool_impl.cpp). Results match the CPU chain bit for bit: the restated
dematcher combining the same LLRs (new_data false, out = the first transmission's buffer), the
restated LDPC decoder and CRC."""
import ctypes
import dataclasses

import numpy as np
import pytest

from pusch_b200 import sim
from pusch_b200.pusch import PuschSlotPlan, make_ue_descriptors
from pusch_b200.sch import segment

pytestmark = pytest.mark.gpu


def device_llrs(ctx, slot):
    """Descrambled codeword LLRs of every UE of a slot from the library's estimator and
    demodulator (the stages before rate dematching), with the descriptors' llr offsets."""
    import torch
    descs, nllr, nest, _ = make_ue_descriptors(slot)
    n = len(slot.ues)
    d_grid = torch.from_numpy(np.ascontiguousarray(slot.grid, np.uint32).view(np.int32).ravel()).cuda()
    d_est = torch.zeros(2 * max(nest, 1), dtype=torch.float32, device="cuda")
    d_pr = torch.zeros(n * 4 * 5, dtype=torch.float32, device="cuda")
    d_llr = torch.zeros(max(nllr, 1), dtype=torch.int8, device="cuda")
    s = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_pusch_estimate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                               d_est.data_ptr(), d_pr.data_ptr(), s.cuda_stream))
    ctx.check(ctx.lib.pg_pusch_demodulate_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                                 d_est.data_ptr(), d_pr.data_ptr(), d_llr.data_ptr(), s.cuda_stream))
    s.synchronize()
    llr = d_llr.cpu().numpy()
    out = []
    for i, ue in enumerate(slot.ues):
        g = sim.nof_ch_symbols(ue) * ue.modulation_order
        out.append(llr[descs[i].llr_offset:descs[i].llr_offset + g].copy())
    return out


def oracle_receive(port, ue, llr, rv, soft, max_iter):
    """CPU chain for one transmission of one UE: restated rate dematching into the UE's soft
    buffers (new data when soft is None, else combining into them), restated LDPC decoding,
    codeblock and TB CRCs. Returns (soft buffers, TB CRC ok, codeblocks ok, TB bits)."""
    seg = segment(ue.tbs_bits, ue.base_graph, ue.modulation_order, ue.nof_layers, sim.nof_ch_symbols(ue))
    c, z, f, k = seg["nof_cbs"], seg["lifting_size"], seg["nof_filler_bits"], seg["cb_length"]
    bg, qm, tbs = ue.base_graph, ue.modulation_order, ue.tbs_bits
    new = soft is None
    soft = [] if new else soft
    off, payload, ok_all, nok = 0, [], True, 0
    for i in range(c):
        e = seg["e_short"] if i < seg["nof_short_cbs"] else seg["e_long"]
        if new:
            soft.append(port.rate_dematch(bg, z, llr[off:off + e], rv=rv, qm=qm, filler=f, new_data=True))
        else:
            port.rate_dematch(bg, z, llr[off:off + e], rv=rv, qm=qm, filler=f, new_data=False, out=soft[i])
        off += e
        poly = 2 if c > 1 else (0 if tbs <= 3824 else 1)
        it, bits = port.ldpc_decode(bg, z, soft[i].copy(), filler=f, crc_poly=poly, max_iter=max_iter)
        ok_all &= it > 0
        nok += it > 0
        payload.append(np.unpackbits(bits)[:k - f - (24 if c > 1 else 0)])
    assert off == llr.size
    tbcat = np.concatenate(payload)
    tb_ok = bool(ok_all and (c == 1 or port.crc(1 if tbs > 3824 else 0, tbcat) == 0))
    return soft, tb_ok, nok, tbcat[:tbs]


def retransmission(slot, combine, seed):
    """The slot's PDUs again: UEs with combine[u] resend their TB with rv 2, the others send a
    new TB with rv 0; new channel and noise."""
    rng = np.random.default_rng(seed)
    ues, tbs = [], []
    for u, ue in enumerate(slot.ues):
        ues.append(dataclasses.replace(ue, rv=2 if combine[u] else 0))
        tbs.append(slot.truth[u] if combine[u] else rng.integers(0, 2, ue.tbs_bits, dtype=np.uint8))
    return sim.make_pusch_slot(ues, slot.nof_ports, nof_prb_grid=slot.nof_prb_grid, slot=slot.slot, seed=seed,
                               tb_bits=tbs)


def test_soft_combining_matches_oracle(ctx, port):
    base = sim.uneven_cells(seed=23, nof_cells=3, max_ues=8)

    def below_threshold(ue, nof_ports):
        # 3 dB below the SNR at which the PDU reaches 10 % BLER without HARQ: most first
        # transmissions fail, and two combined transmissions gain about 3 dB or more.
        rate = int(round(1024 * ue.tbs_bits / (sim.nof_ch_symbols(ue) * ue.modulation_order)))
        snr = sim.required_snr_db(ue.modulation_order, rate, ue.nof_layers, nof_ports) - 3.0
        return dataclasses.replace(ue, snr_db=float(snr))

    first = [sim.make_pusch_slot([below_threshold(ue, sl.nof_ports) for ue in sl.ues], sl.nof_ports,
                                 nof_prb_grid=sl.nof_prb_grid, slot=sl.slot, seed=500 + k)
             for k, sl in enumerate(base)]
    ues = [ue for sl in first for ue in sl.ues]
    n = len(ues)
    combine = [u % 3 != 2 for u in range(n)]
    second, u0 = [], 0
    for k, sl in enumerate(first):
        second.append(retransmission(sl, combine[u0:u0 + len(sl.ues)], 900 + k))
        u0 += len(sl.ues)
    plan = PuschSlotPlan(ctx, first, max_iterations=6)
    plan.set_graph(True)
    got1 = plan.execute_host()
    plan.set_harq(new_data=[not c for c in combine], rv=[2 if c else 0 for c in combine])
    got2 = plan.execute_host(np.concatenate([np.ascontiguousarray(sl.grid, np.uint32).ravel() for sl in second]))
    llr1 = [x for sl in first for x in device_llrs(ctx, sl)]
    llr2 = [x for sl in second for x in device_llrs(ctx, sl)]
    truth2 = [t for sl in second for t in sl.truth]
    ok1 = ok2 = 0
    log = []
    for u in range(n):
        soft, tb_ok, nok, bits = oracle_receive(port, ues[u], llr1[u], 0, None, 6)
        assert (got1[u].tb_crc_ok, got1[u].nof_codeblocks_crc_ok) == (tb_ok, nok), u
        if tb_ok:
            assert np.array_equal(np.unpackbits(got1[u].transport_block), bits)
        _, tb_ok2, nok2, bits2 = oracle_receive(port, ues[u], llr2[u], 2 if combine[u] else 0,
                                                soft if combine[u] else None, 6)
        assert (got2[u].tb_crc_ok, got2[u].nof_codeblocks_crc_ok) == (tb_ok2, nok2), u
        if tb_ok2:
            assert np.array_equal(np.unpackbits(got2[u].transport_block), bits2)
            assert np.array_equal(bits2, truth2[u])
        if combine[u]:
            ok1 += tb_ok
            ok2 += tb_ok2
            log.append((u, ues[u].modulation_order, round(ues[u].snr_db, 1), nok, nok2, got2[u].nof_codeblocks))
    # Combining two transmissions decodes more transport blocks than the first alone.
    assert ok2 > ok1, (ok1, ok2, log)
    plan.close()


def test_harq_rejects_bad_rv_and_autotune_keeps_soft_buffers(ctx):
    slots = sim.uneven_cells(seed=29, nof_cells=1, max_ues=4)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    with pytest.raises(Exception):
        plan.set_harq(rv=[4] * plan.n)
    ref = plan.execute_host()
    plan.set_harq(new_data=[0] * plan.n, rv=[0] * plan.n)
    # Timing executions of the autotuner leave the soft buffers as they were: a combining
    # execution after it gives what it gives without the autotuner.
    grid = np.concatenate([np.ascontiguousarray(sl.grid, np.uint32).ravel() for sl in slots])
    import torch
    d_grid = torch.from_numpy(grid.view(np.int32)).cuda()
    plan.autotune(d_grid.data_ptr(), reps=1)
    a = plan.execute_host()
    plan2 = PuschSlotPlan(ctx, slots, max_iterations=6)
    plan2.execute_host()
    plan2.set_harq(new_data=[0] * plan.n, rv=[0] * plan.n)
    b = plan2.execute_host()
    for x, y, r in zip(a, b, ref):
        assert (x.tb_crc_ok, x.nof_codeblocks_crc_ok, x.mean_iterations) == \
            (y.tb_crc_ok, y.nof_codeblocks_crc_ok, y.mean_iterations)
        assert x.tb_crc_ok or not r.tb_crc_ok
    plan.close()
    plan2.close()

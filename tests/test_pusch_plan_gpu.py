"""Slot plans (pg_pusch_plan_*): the batched receive path prepared once and executed per slot.
Every UE decodes to the transmitted bits where the per-call path does, with identical results
(CRC flags, codeblock counts, iterations, port results); graph replay and plan reuse on a new slot
with the same PDUs give the same results as direct execution."""
import ctypes

import numpy as np
import pytest

from pusch_b200 import sim
from pusch_b200._native import PgSchResult
from pusch_b200.pusch import PuschProcessor, PuschSlotPlan

pytestmark = pytest.mark.gpu


def same_config_slot(slot, seed):
    """A new slot with the PDUs of `slot` (new TB bits, channel and noise)."""
    return sim.make_pusch_slot(slot.ues, slot.nof_ports, nof_prb_grid=slot.nof_prb_grid, slot=slot.slot, seed=seed)


def check_against_truth(results, slots):
    truth = [t for sl in slots for t in sl.truth]
    for r, t in zip(results, truth):
        if r.tb_crc_ok:
            assert (np.unpackbits(r.transport_block) == t).all()
    return sum(r.tb_crc_ok for r in results)


def test_plan_matches_per_call_path(ctx):
    slots = [sim.single_ue_slot(seed=1), sim.full_cell_slot(seed=2, slot=3)]
    slots += sim.uneven_cells(seed=7, nof_cells=3)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    got = plan.execute_host()
    want = PuschProcessor(ctx).process_slots(slots, max_iterations=6)
    assert len(got) == len(want) == plan.n
    for g, w in zip(got, want):
        assert g.tb_crc_ok == w.tb_crc_ok
        assert (g.nof_codeblocks, g.nof_codeblocks_crc_ok) == (w.nof_codeblocks, w.nof_codeblocks_crc_ok)
        assert g.mean_iterations == w.mean_iterations
        assert np.array_equal(g.noise_var, w.noise_var) and np.array_equal(g.snr, w.snr)
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, w.transport_block)
    assert got[0].tb_crc_ok and got[1].tb_crc_ok  # the 20 MHz and 100 MHz configurations decode
    assert check_against_truth(got, slots) >= 0.9 * plan.n
    plan.close()


def test_graph_replay_and_plan_reuse(ctx):
    import torch
    slots = sim.uneven_cells(seed=11, nof_cells=2)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    ref = plan.execute_host()
    n = plan.n
    stream = torch.cuda.Stream()
    d_grid = torch.from_numpy(plan.grid.view(np.int32)).cuda()
    d_tb = torch.zeros(max(plan.tb_bytes, 1), dtype=torch.uint8, device="cuda")
    d_res = torch.zeros(n * ctypes.sizeof(PgSchResult), dtype=torch.uint8, device="cuda")
    for graph in (False, True, True):  # direct, capture + replay, replay
        plan.set_graph(graph)
        d_tb.zero_()
        d_res.zero_()
        plan.execute_device(d_grid.data_ptr(), d_tb.data_ptr(), d_res.data_ptr(), None, stream.cuda_stream)
        stream.synchronize()
        res = (PgSchResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
        tb = d_tb.cpu().numpy()
        for i, r in enumerate(ref):
            assert bool(res[i].tb_crc_ok) == r.tb_crc_ok
            assert res[i].mean_iterations == r.mean_iterations
            if r.tb_crc_ok:
                o = plan.descs[i].tb_out_offset
                assert np.array_equal(tb[o:o + plan.descs[i].tbs_bits // 8], r.transport_block)
    # Same PDUs, new slot data: the plan decodes the new transport blocks.
    new = [same_config_slot(sl, 100 + k) for k, sl in enumerate(slots)]
    grid = np.concatenate([np.ascontiguousarray(sl.grid, np.uint32).ravel() for sl in new])
    plan.set_graph(True)
    out = plan.execute_host(grid)
    assert check_against_truth(out, new) >= 0.9 * n
    plan.close()


def test_uneven_slot_bler(ctx):
    """The 16-cell uneven workload at its link adaptation: BLER at most 10 %."""
    slots = sim.uneven_cells(seed=0, nof_cells=16)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    res = plan.execute_host()
    ok = check_against_truth(res, slots)
    print("UEs", plan.n, "codeblocks", plan.info.nof_codeblocks, "BLER", 1 - ok / plan.n)
    assert ok >= 0.9 * plan.n
    plan.close()


def test_autotuner_keeps_results(ctx):
    """pg_pusch_plan_autotune picks valid launch shapes; every shape decodes to the same results."""
    import torch
    from pusch_b200._native import PgPuschPlanTuning
    slots = sim.uneven_cells(seed=21, nof_cells=2)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6, graph=True)
    ref = plan.execute_host()
    d_grid = torch.from_numpy(plan.grid.view(np.int32)).cuda()
    best, ms = plan.autotune(d_grid.data_ptr(), reps=3)
    assert ms > 0
    assert 1 <= best.rm_ctas_per_cb <= 32 and 1 <= best.demod_res_per_thread <= 8
    assert best.demod_block in (64, 128, 256) and best.ldpc_ctas_per_sm in (1, 2, 3, 4)
    assert plan.tuning().as_dict() == best.as_dict()
    assert best.ldpc_kernel in range(5) and best.ldpc_order in (0, 1)
    for shape in (best, PgPuschPlanTuning(3, 3, 64, 1, 0), PgPuschPlanTuning(32, 8, 128, 2, 1),
                  PgPuschPlanTuning(8, 1, 256, 4, 1), PgPuschPlanTuning(8, 1, 256, 1, 1),
                  PgPuschPlanTuning(8, 1, 256, 2, 3, 1), PgPuschPlanTuning(16, 1, 256, 2, 4, 0)):
        plan.set_tuning(shape)
        got = plan.execute_host()
        for g, r in zip(got, ref):
            assert g.tb_crc_ok == r.tb_crc_ok and g.mean_iterations == r.mean_iterations
            if r.tb_crc_ok:
                assert np.array_equal(g.transport_block, r.transport_block)
    with pytest.raises(Exception):
        plan.set_tuning(PgPuschPlanTuning(0, 1, 256, 2, 0))
    plan.close()


def test_pipelined_host_execution(ctx):
    """submit_host / collect_host over four slots with up to three in flight give, slot by slot, the
    results of execute_host on the same grids; the in-flight limit and an empty collect are errors."""
    from pusch_b200._native import PgError
    slots = sim.uneven_cells(seed=13, nof_cells=2)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    grids = [plan.grid] + [np.concatenate([np.ascontiguousarray(sl.grid, np.uint32).ravel()
                                           for sl in [same_config_slot(x, 200 + 10 * k + i) for i, x in enumerate(slots)]])
                           for k in range(3)]
    want = [plan.execute_host(g) for g in grids]
    try:
        with pytest.raises(PgError):
            plan.collect_host()
        plan.submit_host(grids[0])
        plan.submit_host(grids[1])
        plan.submit_host(grids[2])
        with pytest.raises(PgError):
            plan.submit_host(grids[3])
        got = [plan.collect_host()]
        plan.submit_host(grids[3])
        got += [plan.collect_host(), plan.collect_host(), plan.collect_host()]
        for g_slot, w_slot in zip(got, want):
            for g, w in zip(g_slot, w_slot):
                assert (g.tb_crc_ok, g.nof_codeblocks_crc_ok, g.mean_iterations) == \
                    (w.tb_crc_ok, w.nof_codeblocks_crc_ok, w.mean_iterations)
                assert np.array_equal(g.noise_var, w.noise_var)
                if g.tb_crc_ok:
                    assert np.array_equal(g.transport_block, w.transport_block)
        assert sum(r.tb_crc_ok for r in got[2]) >= 0.9 * plan.n
    finally:
        plan.close()

"""Open Fronthaul BFP decompression on the GPU against the reference's compiled decompressor
(bit-exact complex bf16 words for every width 1-16, on its own compressor's output and on random
payloads, aligned and unaligned input, a partial last CTA), and slot plans fed compressed grids:
the same results as the plan fed the reference's decompressed grids."""
import ctypes

import numpy as np
import pytest

from pusch_b200 import sim
from pusch_b200.pusch import PuschSlotPlan

from test_ofh_bfp_cpu import random_grid_words

pytestmark = pytest.mark.gpu


def gpu_decompress(ctx, width, data, nprb, shift=0):
    import torch
    d_in = torch.zeros(data.size + 16, dtype=torch.uint8, device="cuda")
    d_in[shift:shift + data.size] = torch.from_numpy(data).cuda()
    d_out = torch.full((12 * nprb,), 0x7FC07FC0, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_bfp_decompress_device(ctx.handle, d_in.data_ptr() + shift, nprb, width, d_out.data_ptr(),
                                               st.cuda_stream))
    st.synchronize()
    return d_out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("width", list(range(1, 17)))
def test_decompress_matches_reference(ctx, ref, width):
    rng = np.random.default_rng(width)
    nprb = 1000 + width  # not a multiple of the 32 PRBs of a CTA
    data = ref.bfp_compress(width, random_grid_words(rng, nprb, 0.25))
    want, _ = ref.bfp_decompress(width, data, nprb)
    for shift in (0, 3):
        assert np.array_equal(gpu_decompress(ctx, width, data, nprb, shift), want), (width, shift)
    raw = rng.integers(0, 256, nprb * (1 + 3 * width), dtype=np.uint8)
    raw[::1 + 3 * width] = rng.integers(0, 16 - width + 1, nprb)
    want, _ = ref.bfp_decompress(width, raw, nprb)
    assert np.array_equal(gpu_decompress(ctx, width, raw, nprb), want), width


def test_plan_from_compressed_grids(ctx, ref):
    slots = sim.uneven_cells(seed=31, nof_cells=2)
    # The radio unit scales the received signal into the fixed-point range (the simulated grids
    # reach several times full scale, which 16-bit quantisation would clip).
    for sl in slots:
        sl.grid = sim.scale_grid_words(sl.grid, 1.0 / 16)
    plan = PuschSlotPlan(ctx, slots, max_iterations=6)
    comp = ref.bfp_compress(9, plan.grid.ravel())
    grid_ref, _ = ref.bfp_decompress(9, comp, plan.grid.size // 12)
    got = plan.execute_host_bfp(comp, 9)
    want = plan.execute_host(grid_ref)
    for g, w in zip(got, want):
        assert (g.tb_crc_ok, g.nof_codeblocks_crc_ok, g.mean_iterations) == \
            (w.tb_crc_ok, w.nof_codeblocks_crc_ok, w.mean_iterations)
        assert np.array_equal(g.noise_var, w.noise_var) and np.array_equal(g.snr, w.snr)
        if g.tb_crc_ok:
            assert np.array_equal(g.transport_block, w.transport_block)
    truth = [t for sl in slots for t in sl.truth]
    ok = sum(1 for g, t in zip(got, truth) if g.tb_crc_ok and (np.unpackbits(g.transport_block) == t).all())
    assert ok >= 0.9 * plan.n
    try:
        with pytest.raises(Exception):
            plan.execute_host_bfp(comp[:-1], 9)
    finally:
        plan.close()

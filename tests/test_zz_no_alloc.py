"""pg_ldpc_decode_batch_static_scratch (check-to-variable scratch in a fixed device array of the
library, no allocation in the call) against pg_ldpc_decode_batch_device (the context's scratch):
bit-exact decoded bits and equal iteration counts on two calls in a row, the second running over
what the first left in the shared array; batches above the fixed limit are refused."""
import ctypes
import os
import re

import numpy as np
import pytest

from pusch_b200 import _native, sim
from pusch_b200.ldpc import make_descriptors

pytestmark = pytest.mark.gpu

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "pusch_b200.h")


def static_limit():
    with open(HEADER) as f:
        return int(re.search(r"#define PG_STATIC_SCRATCH_MAX_CODEBLOCKS (\d+)", f.read()).group(1))


def to_device(jobs):
    import torch
    descs, llrs, nbytes = make_descriptors(jobs)
    d_descs = torch.from_numpy(np.frombuffer(bytes(descs), np.uint8).copy()).cuda()
    d_llrs = torch.from_numpy(llrs).cuda()
    return descs, d_descs, d_llrs, nbytes


def decode_with_context_scratch(ctx, descs, n, d_llrs, nbytes):
    import torch
    bits = torch.zeros(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_ldpc_decode_batch_device(ctx.handle, ctypes.addressof(descs), n, d_llrs.data_ptr(),
                                                  bits.data_ptr(), it.data_ptr(), s.cuda_stream))
    s.synchronize()
    return bits.cpu().numpy(), it.cpu().numpy()


def decode_with_static_scratch(small, d_descs, n, d_llrs, nbytes):
    import torch
    bits = torch.zeros(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    small.check(small.lib.pg_ldpc_decode_batch_static_scratch(small.handle, d_descs.data_ptr(), n, d_llrs.data_ptr(),
                                                              bits.data_ptr(), it.data_ptr(), s.cuda_stream))
    s.synchronize()
    return bits.cpu().numpy(), it.cpu().numpy()


@pytest.fixture(scope="module")
def small_ctx():
    # One codeblock of context scratch: the static entry is bounded by its own array, not by this.
    c = _native.Context(device=0, max_codeblocks=1)
    yield c
    c.close()


def test_static_scratch_matches_context_scratch_twice(ctx, small_ctx):
    limit = static_limit()
    batches = [sim.ldpc_batch(seed=5, n=limit, z=384).jobs,          # the full array, BG1/BG2 at Z = 384
               sim.ldpc_batch(seed=6, n=37, z=208, bg_mix=0.3).jobs]  # smaller, over the first call's leftovers
    for jobs in batches:
        descs, d_descs, d_llrs, nbytes = to_device(jobs)
        want_bits, want_it = decode_with_context_scratch(ctx, descs, len(jobs), d_llrs, nbytes)
        got_bits, got_it = decode_with_static_scratch(small_ctx, d_descs, len(jobs), d_llrs, nbytes)
        assert (got_it == want_it).all()
        assert (got_bits == want_bits).all()
        assert (got_it > 0).any()


def test_static_scratch_rejects_oversized_batch(small_ctx):
    limit = static_limit()
    rc = small_ctx.lib.pg_ldpc_decode_batch_static_scratch(small_ctx.handle, None, limit + 1, None, None, None, None)
    assert rc == _native.PG_ERR_CAPACITY
    assert str(limit) in small_ctx.lib.pg_last_error(small_ctx.handle).decode()
    rc = small_ctx.lib.pg_ldpc_decode_batch_static_scratch(small_ctx.handle, None, -1, None, None, None, None)
    assert rc == _native.PG_ERR_INVALID

"""Tensor-core 1-D convolution (tcgen05, BF16 operands, FP32 accumulation) against a float64
convolution of the same bf16 inputs: every output within one bf16 rounding of the exact value."""
import ctypes

import numpy as np
import pytest

from pusch_b200 import tclayout as tl

pytestmark = pytest.mark.gpu


def run_conv(ctx, x, w, b, res, relu, valid):
    import torch
    rows = x.shape[0]
    cin, cout = w.shape[1], w.shape[0]
    d_x = torch.from_numpy(tl.to_chunked(x).view(np.int16)).cuda()
    d_w = torch.from_numpy(tl.pack_weights(w).view(np.int16)).cuda()
    d_b = torch.from_numpy(b.astype(np.float32)).cuda()
    d_r = torch.from_numpy(tl.to_chunked(res).view(np.int16)).cuda() if res is not None else None
    d_y = torch.zeros((cout // 8, rows, 8), dtype=torch.int16, device="cuda")
    d_v = torch.from_numpy(valid.astype(np.uint8)).cuda()
    d_e = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_conv1d_forward_device(ctx.handle, cin, cout, d_x.data_ptr(), d_w.data_ptr(), d_b.data_ptr(),
                                               d_r.data_ptr() if d_r is not None else None, d_y.data_ptr(),
                                               d_v.data_ptr(), rows, int(relu), d_e.data_ptr(), s.cuda_stream))
    s.synchronize()
    assert int(d_e.item()) == 0
    return tl.from_chunked(d_y.cpu().numpy().view(np.uint16))


@pytest.mark.parametrize("cin,cout,rows,relu,with_res", [(16, 64, 300, True, False), (64, 64, 1000, False, True),
                                                         (64, 16, 257, False, False), (64, 64, 128, True, False)])
def test_conv_matches_float64(ctx, cin, cout, rows, relu, with_res):
    rng = np.random.default_rng(cin * 7 + cout + rows)
    x = tl.bf16_round(rng.standard_normal((rows, cin)).astype(np.float32))
    w = tl.bf16_round((rng.standard_normal((cout, cin, 5)) / np.sqrt(5 * cin)).astype(np.float32))
    b = rng.standard_normal(cout).astype(np.float32) * 0.1
    res = tl.bf16_round(rng.standard_normal((rows, cout)).astype(np.float32)) if with_res else None
    valid = np.ones(rows, bool)
    valid[::37] = False  # rows that must stay untouched (zero)
    x[~valid] = 0
    got = run_conv(ctx, x, w, b, res, relu, valid)
    want = tl.conv1d_ref(x, w, b, res, relu)
    want[~valid] = 0
    err = np.abs(got - want)
    tol = 2.0 ** -7 * np.abs(want) + 1e-3  # one bf16 rounding of the output plus fp32 accumulation
    assert (err <= tol).all(), float(err.max())
    assert (got[~valid] == 0).all()

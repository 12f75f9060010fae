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


@pytest.mark.parametrize("cin,cout,rows", [(16, 64, 300), (64, 64, 1000), (64, 16, 257), (64, 64, 3000)])
def test_conv_backward_matches_float64(ctx, cin, cout, rows):
    """Input gradient (with residual and ReLU mask) and weight/bias gradients of one layer against
    float64, on samples separated by zero rows (the invalid rows)."""
    import torch
    rng = np.random.default_rng(1000 + cin + cout + rows)
    valid = np.ones(rows, bool)
    valid[::41] = False
    valid[:2] = False
    x = tl.bf16_round(rng.standard_normal((rows, cin)).astype(np.float32))
    x[~valid] = 0
    dy = tl.bf16_round(rng.standard_normal((rows, cout)).astype(np.float32))
    dy[~valid] = 0
    w = tl.bf16_round((rng.standard_normal((cout, cin, 5)) / np.sqrt(5 * cin)).astype(np.float32))
    res = tl.bf16_round(rng.standard_normal((rows, cin)).astype(np.float32))
    res[~valid] = 0
    mask = tl.bf16_round(np.maximum(rng.standard_normal((rows, cin)), 0).astype(np.float32))

    # Reference: rows between invalid rows are independent samples; the zero rows make the
    # whole-buffer convolution equal to the per-sample ones.
    dx_ref, dw_ref, db_ref = tl.conv1d_backward_ref(x, w, dy)
    dx_ref = np.where(mask > 0, dx_ref + res, 0.0)
    dx_ref[~valid] = 0

    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_dy = dev(tl.to_chunked(dy).view(np.int16))
    d_wt = dev(tl.pack_weights_t(w).view(np.int16))
    d_res = dev(tl.to_chunked(res).view(np.int16))
    d_mask = dev(tl.to_chunked(mask).view(np.int16))
    d_dx = torch.zeros((cin // 8, rows, 8), dtype=torch.int16, device="cuda")
    d_v = dev(valid.astype(np.uint8))
    d_e = torch.zeros(1, dtype=torch.int32, device="cuda")
    d_x = dev(tl.to_chunked(x).view(np.int16))
    dw0 = rng.standard_normal((5, cin, cout)).astype(np.float32)
    db0 = rng.standard_normal(cout).astype(np.float32)
    d_dw = dev(dw0)
    d_db = dev(db0)
    s = torch.cuda.current_stream()
    ctx.check(ctx.lib.pg_conv1d_backward_data_device(ctx.handle, cin, cout, d_dy.data_ptr(), d_wt.data_ptr(),
                                                     d_res.data_ptr(), d_mask.data_ptr(), d_dx.data_ptr(),
                                                     d_v.data_ptr(), rows, d_e.data_ptr(), s.cuda_stream))
    ctx.check(ctx.lib.pg_conv1d_backward_weights_device(ctx.handle, cin, cout, d_x.data_ptr(), d_dy.data_ptr(), rows,
                                                        d_dw.data_ptr(), d_db.data_ptr(), d_e.data_ptr(),
                                                        s.cuda_stream))
    s.synchronize()
    assert int(d_e.item()) == 0
    dx = tl.from_chunked(d_dx.cpu().numpy().view(np.uint16))
    tol = 2.0 ** -7 * np.abs(dx_ref) + 1e-3
    assert (np.abs(dx - dx_ref) <= tol).all(), float(np.abs(dx - dx_ref).max())
    # FP32 accumulation over the rows: bound by the sum of |products|.
    mag = np.stack([np.abs(np.vstack([np.zeros((2, cin)), x, np.zeros((2, cin))])[t:t + rows]).T @ np.abs(dy)
                    for t in range(5)])
    dw = d_dw.cpu().numpy() - dw0
    assert (np.abs(dw - dw_ref) <= 1e-5 * mag + 1e-4).all(), float(np.abs(dw - dw_ref).max())
    db = d_db.cpu().numpy() - db0
    assert np.allclose(db, db_ref, rtol=1e-5, atol=1e-3)

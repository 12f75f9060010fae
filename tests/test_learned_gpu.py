"""Learned channel estimator on the GPU: forward pass and gradients of the tensor-core network
against the float64 restatement (oracle/learned_ref.py, bf16 rounding at the same points), the
refinement path (features -> network -> corrected estimates and time-basis coefficients) against
the restatement, and what training on the GPU gains over the plain estimator on the channel at
every data symbol of the slot."""
import ctypes

import numpy as np
import pytest

import learned_ref as lr
from pusch_b200 import learned
from pusch_b200 import tclayout as tl

pytestmark = pytest.mark.gpu


def chunked_dev(a):
    import torch
    return torch.from_numpy(tl.to_chunked(a).view(np.int16)).cuda()


def random_rows(rng, lens):
    rows = sum(n + 2 for n in lens) + 2
    valid = np.zeros(rows, bool)
    r = 0
    for n in lens:
        r += 2
        valid[r:r + n] = True
        r += n
    return rows, valid


def test_forward_and_gradients_match_oracle(ctx):
    import torch
    rng = np.random.default_rng(5)
    rows, valid = random_rows(rng, [300, 37, 12, 600, 250])
    params = learned.init_params(7)
    params[-16 - 5 * 64 * 16:] *= 50.0
    x = tl.bf16_round((rng.standard_normal((rows, 16)) * valid[:, None]).astype(np.float32))
    dy = tl.bf16_round((rng.standard_normal((rows, 16)) * valid[:, None]).astype(np.float32))
    net = learned.LearnedEstimator(ctx, max_rows=rows, params=params)
    # Every device buffer stays referenced until the work that reads it has run.
    x_dev, dy_dev = chunked_dev(x), chunked_dev(dy)
    v_dev = torch.from_numpy(valid.astype(np.uint8)).cuda()
    y_dev = torch.zeros((2, rows, 8), dtype=torch.int16, device="cuda")
    net.forward(x_dev.data_ptr(), v_dev.data_ptr(), rows, y_dev.data_ptr())
    net.backward(dy_dev.data_ptr(), rows)
    y = tl.from_chunked(y_dev.cpu().numpy().view(np.uint16))
    g = net.grads()
    net.status()
    y_ref, cache = lr.forward(params.astype(np.float64), x.astype(np.float64), valid, bf16_acts=True)
    g_ref = lr.backward(cache, dy.astype(np.float64))
    # Forward: bf16 storage of 14 layers; FP32 accumulation order is the only difference.
    assert np.linalg.norm(y - y_ref) <= 2e-2 * np.linalg.norm(y_ref), np.abs(y - y_ref).max()
    assert (y[~valid] == 0).all()
    # Gradients, layer by layer (weights and biases).
    offs, total = lr.layer_offsets()
    for i, (cin, cout) in enumerate(lr.LAYERS):
        a, b = offs[i], offs[i] + 5 * cin * cout + cout
        err = np.linalg.norm(g[a:b] - g_ref[a:b]) / np.linalg.norm(g_ref[a:b])
        assert err < 3e-2, (i, err)
    net.close()


def make_batch(ctx, seed, rows):
    import torch
    src = learned.DmrsTrainingSource(seed)
    descs, grid, h_true, est_size, ues = src.batch(rows)
    n = len(descs)
    est = torch.empty(2 * est_size, dtype=torch.float32, device="cuda")
    ls = torch.empty_like(est)
    pr = torch.empty((n * 4, 5), dtype=torch.float32, device="cuda")
    ctx.check(ctx.lib.pg_pusch_estimate_ls_device(ctx.handle, ctypes.addressof(descs), n, grid.data_ptr(),
                                                  est.data_ptr(), ls.data_ptr(), pr.data_ptr(), None))
    torch.cuda.synchronize()
    return descs, est, ls, pr, h_true


@pytest.mark.parametrize("nrows", [20_000, 70_000])
def test_refine_matches_oracle(ctx, nrows):
    """20,000 rows run as one-tile windows of the fused network kernel only; 70,000 rows as
    two-tile windows and one-tile windows after them."""
    import torch
    descs, est, ls, pr, h_true = make_batch(ctx, 3, nrows)
    n = len(descs)
    params = learned.init_params(11)
    params[-16 - 5 * 64 * 16:] *= 30.0
    rows = int(ctx.lib.pg_le_rows(ctypes.addressof(descs), n))
    net = learned.LearnedEstimator(ctx, max_rows=rows, params=params)
    use = [i % 3 != 1 for i in range(n)]
    est_h = est.cpu().numpy().view(np.complex64).astype(np.complex128)
    ls_h = ls.cpu().numpy().view(np.complex64).astype(np.complex128)
    prh = pr.cpu().numpy().reshape(n, 4, 5)
    basis = torch.full_like(est, 7.0)
    net.refine(descs, ls.data_ptr(), est.data_ptr(), pr.data_ptr(), use=use, basis_ptr=basis.data_ptr())
    got = est.cpu().numpy().view(np.complex64).astype(np.complex128)
    got_b = basis.cpu().numpy().view(np.complex64).astype(np.complex128)
    net.status()
    # Restatement over the used UEs only (the layout skips the others).
    sel = [i for i in range(n) if use[i]]
    ues = [dict(nof_rb=descs[i].nof_rb, nof_layers=descs[i].nof_layers, nof_rx_ports=4, nd=2) for i in sel]
    seqs, R = lr.sequences(ues, [descs[i].est_offset for i in sel])
    assert R + 0 == rows - sum(4 * descs[i].nof_layers * (12 * descs[i].nof_rb + 2) for i in range(n) if not use[i])
    x, valid, gains = lr.features(seqs, R, est_h, ls_h, prh[sel, :, 0], prh[sel, :, 3:5],
                                  [descs[i].dmrs_scaling for i in sel])
    y, _ = lr.forward(params.astype(np.float64), x, valid, bf16_acts=True)
    want, want_b = lr.refine(seqs, est_h, y, gains)
    corr = want - est_h
    err = np.linalg.norm(got - want) / max(np.linalg.norm(corr), 1e-12)
    assert err < 3e-2, err
    used = np.zeros(got.size, bool)
    for i in range(n):
        o = descs[i].est_offset
        m = 4 * 2 * descs[i].nof_layers * 12 * descs[i].nof_rb
        if not use[i]:
            assert np.array_equal(got[o:o + m], est_h[o:o + m])
            assert (got_b[o:o + m] == 7 + 7j).all()      # untouched
        else:
            used[o:o + m] = True
    err_b = np.linalg.norm(got_b[used] - want_b[used]) / max(np.linalg.norm(want_b[used]), 1e-12)
    assert err_b < 3e-2, err_b
    net.close()


def full_grid_nmse(ctx, net, descs, est, ls, pr, h_true):
    """(plain, learned) NMSE of the channel at the data symbols, as the demodulator uses it."""
    import torch
    truth = learned.split_truth(descs, h_true)
    before = learned.data_symbol_nmse(descs, learned.grid_estimates(ctx, descs, est), truth)
    basis = torch.zeros_like(est)
    net.refine(descs, ls.data_ptr(), est.data_ptr(), pr.data_ptr(), basis_ptr=basis.data_ptr())
    after = learned.data_symbol_nmse(descs, learned.grid_estimates(ctx, descs, est, basis), truth)
    net.status()
    return before, after


def test_training_on_gpu_beats_plain_estimator(ctx):
    """A short training run on the GPU (the library's own forward/backward kernels and Adam)
    lowers the error of the channel at the data symbols below the plain estimator's on held-out
    batches."""
    net, hist = learned.train(ctx, steps=400, rows_per_step=40_000, seed=1, lr=1e-3, log_every=100, verbose=False)
    assert hist[-1][1] < hist[0][1]
    descs, est, ls, pr, h_true = make_batch(ctx, 999, 60_000)
    before, after = full_grid_nmse(ctx, net, descs, est, ls, pr, h_true)
    assert after < 0.9 * before, (before, after)
    net.close()


def test_committed_weights_gain_over_plain(ctx):
    """The committed trained parameters: the estimate error on held-out batches is well below the
    plain estimator's."""
    params = learned.load_params()
    if params is None:
        pytest.skip("no trained parameters committed")
    descs, est, ls, pr, h_true = make_batch(ctx, 4242, 80_000)
    rows = int(ctx.lib.pg_le_rows(ctypes.addressof(descs), len(descs)))
    net = learned.LearnedEstimator(ctx, max_rows=rows, params=params)
    before, after = full_grid_nmse(ctx, net, descs, est, ls, pr, h_true)
    assert after < 0.7 * before, (before, after)
    net.close()

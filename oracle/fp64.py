"""Test infrastructure only: FP64 numpy restatements of the reference's floating-point stages,
used to state the error of the float32 GPU kernels (and of the reference itself) against exact
arithmetic.

equalize_fp64 follows lib/phy/upper/equalization/equalize_zf_1xn.h:25-153 (one layer: maximum
ratio combining with per-port noise) and equalize_mmse_mxn_simd.h:14-75 with
channel_equalizer_generic_impl.cpp:511-653 (several layers: MMSE with the largest port noise).
"""
import numpy as np


def cbf16_to_c128(u):
    u = np.asarray(u, np.uint32)
    re = (u << 16).view(np.float32).astype(np.float64)
    im = (u & 0xFFFF0000).view(np.float32).astype(np.float64)
    return re + 1j * im


def equalize_fp64(ch_symbols, ch_estimates, noise_var_per_port, tx_scaling=1.0):
    """ch_symbols uint32 cbf16 [port][re]; ch_estimates uint32 cbf16 [port][layer][re].
    Returns complex128 [re][layer], float64 [re][layer]."""
    y = cbf16_to_c128(ch_symbols)            # [P, R]
    h = cbf16_to_c128(ch_estimates)          # [P, L, R]
    nv = np.asarray(noise_var_per_port, np.float64)
    P, L, R = h.shape
    if L == 1:
        hn = np.abs(h[:, 0, :]) ** 2
        ok_p = np.isfinite(hn)
        hn0 = np.where(ok_p, hn, 0.0)
        den = tx_scaling * hn0.sum(0)
        num = np.where(ok_p, y * np.conj(h[:, 0, :]), 0).sum(0)
        nacc = (hn0 * nv[:, None]).sum(0)
        ok = (den > 0) & np.isfinite(den)
        with np.errstate(all="ignore"):
            eq = np.where(ok, num / den, 0)
            var = np.where(ok, nacc / den ** 2, np.inf)
        return eq[:, None], var[:, None]
    n = nv.max()
    H = np.transpose(h, (2, 0, 1)) * tx_scaling       # [R, P, L]
    G = np.conj(np.transpose(H, (0, 2, 1))) @ H        # [R, L, L]
    ok = np.all(np.real(np.diagonal(G, axis1=1, axis2=2)) > 0, axis=1)
    G = G + n * np.eye(L)[None]
    with np.errstate(all="ignore"):
        W = np.linalg.solve(G, np.conj(np.transpose(H, (0, 2, 1))))   # [R, L, P]
        s = np.einsum("rlp,pr->rl", W, y)
        corr = np.real(np.einsum("rlp,rpl->rl", W, H))
        eq = np.where(ok[:, None], s / corr, 0)
        var = np.where(ok[:, None], 1.0 / corr - 1.0, np.inf)
    return eq, var


def rel_err(got, want, floor_frac=1e-3):
    """Elementwise |got - want| / max(|want|, floor_frac * rms(want)), over finite entries."""
    got = np.asarray(got)
    want = np.asarray(want)
    fin = np.isfinite(want) & np.isfinite(got)
    if not fin.any():
        return np.zeros(0)
    w = want[fin]
    g = got[fin]
    rms = np.sqrt(np.mean(np.abs(w) ** 2)) if w.size else 1.0
    return np.abs(g - w) / np.maximum(np.abs(w), floor_frac * rms)

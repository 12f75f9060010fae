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


# ----------------------------------------------------------------------------------------------
# Gold sequence (TS 38.211 Section 5.2.1), the reference's pseudo_random_generator
# (lib/phy/upper/sequence_generators/pseudo_random_generator_impl.cpp:40-136).

def gold_sequence(c_init, length, nc=1600):
    n = nc + length + 31
    x1 = np.zeros(n, np.uint8)
    x2 = np.zeros(n, np.uint8)
    x1[0] = 1
    for i in range(31):
        x2[i] = (c_init >> i) & 1
    # x1(n+31) = x1(n+3) + x1(n); x2(n+31) = x2(n+3) + x2(n+2) + x2(n+1) + x2(n), 28 at a time.
    i = 0
    while i + 31 < n:
        k = min(28, n - 31 - i)
        x1[i + 31:i + 31 + k] = x1[i + 3:i + 3 + k] ^ x1[i:i + k]
        x2[i + 31:i + 31 + k] = x2[i + 3:i + 3 + k] ^ x2[i + 2:i + 2 + k] ^ x2[i + 1:i + 1 + k] ^ x2[i:i + k]
        i += k
    return (x1[nc:nc + length] ^ x2[nc:nc + length]).astype(np.uint8)


def dmrs_pilots_type1(slot, symbol, n_id, n_scid, rb_start, nof_rb, nof_layers, nsymb=14):
    """DM-RS type 1 pilots of one OFDM symbol for layers 0..nof_layers-1 (ports 0/1 in CDM
    group 0): dmrs_pusch_estimator_impl.cpp:69-169 and TS 38.211 Section 6.4.1.1."""
    c_init = ((nsymb * slot + symbol + 1) * (2 * n_id + 1) * (1 << 17) + (2 * n_id + n_scid)) % (1 << 31)
    m0 = 6 * rb_start
    c = gold_sequence(c_init, 2 * (m0 + 6 * nof_rb)).astype(np.float64)
    m = np.arange(m0, m0 + 6 * nof_rb)
    r = ((1 - 2 * c[2 * m]) + 1j * (1 - 2 * c[2 * m + 1])) / np.sqrt(2.0)
    out = np.zeros((nof_layers, 6 * nof_rb), np.complex128)
    out[0] = r
    if nof_layers > 1:
        w = np.ones(6 * nof_rb)
        w[1::2] = -1
        out[1] = r * w
    return out


# Raised-cosine frequency-domain smoothing (port_channel_estimator_helpers.cpp:29-233): a 31-tap
# raised-cosine impulse (roll-off 0.2, 10 samples per symbol period) resampled by the pilot stride
# and normalised, applied to the pilots extended at both ends by virtual pilots extrapolated from
# a linear fit of the magnitude and of the unwrapped phase of the outermost pilots.
def _rc_taps():
    t = (np.arange(31) - 15) / 10.0
    beta = 0.2
    with np.errstate(divide="ignore", invalid="ignore"):
        h = np.sinc(t) * np.cos(np.pi * beta * t) / (1 - (2 * beta * t) ** 2)
    return h


def fd_filter_taps(nof_rb, stride):
    nrb = min(nof_rb, 3)
    ncoef = nrb * 10 + 1
    nout = ncoef // 2 // stride
    first = 15 - nout * stride
    taps = _rc_taps()[first:first + (2 * nout + 1) * stride:stride]
    return taps / taps.sum()


def _virtual_pilots(base, nv, is_start):
    idx = np.arange(nv, dtype=np.float64)
    ab = np.abs(base)
    ar = np.unwrap(np.angle(base))
    A = np.vstack([idx, np.ones(nv)]).T
    sa, ia = np.linalg.lstsq(A, ab, rcond=None)[0]
    sg, ig = np.linalg.lstsq(A, ar, rcond=None)[0]
    vi = np.arange(nv) + (-nv if is_start else nv)
    rho = sa * vi + ia
    return np.abs(rho) * np.exp(1j * (sg * vi + ig + np.where(rho > 0, 0, np.pi)))


def fd_smooth(pilots, nof_rb, stride=2):
    taps = fd_filter_taps(nof_rb, stride)
    nv = min(12, taps.size // 2)
    if nof_rb == 1:
        nv = pilots.size
    ext = np.concatenate([_virtual_pilots(pilots[:nv], nv, True), pilots, _virtual_pilots(pilots[-nv:], nv, False)])
    full = np.convolve(ext, taps, mode="same")
    return full[nv:nv + pilots.size]


def interpolate_linear(pilots, nof_sc, offset=0, stride=2):
    out = np.empty(nof_sc, np.complex128)
    pos = offset + stride * np.arange(pilots.size)
    out[:offset + 1] = pilots[0]
    for k in range(pilots.size - 1):
        for s in range(1, stride):
            out[pos[k] + s] = pilots[k] + (pilots[k + 1] - pilots[k]) * s / stride
        out[pos[k + 1]] = pilots[k + 1]
    out[pos[-1]:] = pilots[-1]
    return out


def estimate_port_fp64(grid, port, cfg):
    """One receive port of the DM-RS PUSCH estimator with FD 'filter', TD 'interpolate', no CFO
    compensation, type-1 DM-RS without hopping (port_channel_estimator_average_impl.cpp:322-557).
    grid: uint32 cbf16 [port][symbol][subcarrier]. Returns a dict with the frequency response
    per DM-RS symbol [dmrs][layer][12*nof_rb], noise_var, rsrp[layer], epre, snr."""
    nl = cfg["nof_layers"]
    beta = cfg.get("scaling", 1.0)
    rb0, nrb = cfg["rb_start"], cfg["nof_rb"]
    dsyms = cfg["dmrs_symbols"]
    nd = len(dsyms)
    g = cbf16_to_c128(np.asarray(grid)[port])
    npil = 6 * nrb
    rx = np.array([g[s, 12 * rb0:12 * (rb0 + nrb):2] for s in dsyms])            # [nd, npil]
    pil = np.array([dmrs_pilots_type1(cfg["slot"], s, cfg["n_id"], cfg.get("n_scid", 0), rb0, nrb, nl)
                    for s in dsyms])                                             # [nd, nl, npil]
    lse = rx[:, None, :] * np.conj(pil)
    if nl > 1:
        avg = (lse[..., 0::2] + lse[..., 1::2]) / 2
        lse[..., 0::2] = avg
        lse[..., 1::2] = avg
    lse = lse / beta
    filt = np.array([[fd_smooth(lse[d, l], nrb) for l in range(nl)] for d in range(nd)])
    rsrp = (np.abs(filt) ** 2).sum(axis=(0, 2)) * beta ** 2
    freq = np.array([[interpolate_linear(filt[d, l], 12 * nrb) for l in range(nl)] for d in range(nd)])
    scaled = filt.sum(axis=0) * (beta / nd)                                     # [nl, npil]
    noise = 0.0
    for d in range(nd):
        pred = (scaled * pil[d]).sum(axis=0)
        noise += (np.abs(pred - rx[d]) ** 2).sum()
    nof_dmrs_pilots = npil * nd
    ncdm = (nl + 1) // 2
    rsrp = rsrp / nof_dmrs_pilots
    epre = (np.abs(rx) ** 2).sum() / nof_dmrs_pilots
    nvar = noise / (nof_dmrs_pilots * ncdm - 1)
    rsrp_avg = rsrp.mean()
    nvar = max(rsrp_avg / 1e10, nvar)
    snr = (rsrp_avg * nl / beta / beta) / nvar if nvar > 0 else 0.0
    return dict(freq=freq, noise_var=nvar, rsrp=rsrp, epre=epre, snr=snr)


def td_weights(symbol, dmrs_symbols, first, last):
    """(DM-RS index i, weight w): the estimate of `symbol` is f[i] + (f[i+1] - f[i]) w
    (port_channel_estimator_average_impl.cpp:705-767); (i, 0) copies f[i]."""
    ds = sorted(s for s in dmrs_symbols if first <= s < last)
    before = [s for s in ds if s < symbol]
    after = [s for s in ds if s >= symbol]
    b = before[-1] if before else -1
    a = after[0] if after else -1
    if b == -1:
        second = [s for s in ds if s > a]
        if not second:
            return 0, 0.0
        b, a = a, second[0]
    if a == -1:
        second_last = [s for s in ds if s < b]
        if not second_last:
            return len(ds) - 1, 0.0
        a, b = b, second_last[-1]
    return ds.index(b), (symbol - b) / (a - b)

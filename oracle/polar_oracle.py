"""Test infrastructure only (the checker; never shipped, never on a product path): a CPU
restatement of the reference's decoding of polar-coded UCI (messages of 12 to 1706 bits).

Each step follows the reference:
- segmentation and CRC size: include/ocudu/ran/uci/uci_info.h:22-47;
- per codeblock: uci_decoder_impl::decode_codeblock_polar
  (lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:60-99);
- rate dematching: polar_rate_dematcher_impl.cpp:12-100 (channel de-interleaver, bit selection
  with promotion sums on repetition, zeros on puncturing, +127 on shortening, sub-block
  de-interleaving);
- decoding: polar_decoder_impl.cpp:74-332 (simplified successive cancellation over rate-0,
  rate-1 and rate-R nodes; f = soft_xor, g = saturated sum, rate-1 nodes re-encoded);
- deallocation: polar_deallocator_impl.cpp:10-24; the CRC: crc_calculator::calculate_bit.

The polar code itself (N, K_set, PC_set, sub-block interleaver) is taken from the caller as a dict
(the reference's polar_code_impl::set through oracle._ref, see Ref.polar_code), so this module
restates the decoding only. LLR arithmetic: log_likelihood_ratio (lib/phy/upper/log_likelihood_ratio.cpp).
"""
import numpy as np

LLR_MAX, LLR_INF = 120, 127


def sat_sum(a, b):
    """log_likelihood_ratio::operator+ (log_likelihood_ratio.cpp:21-55)."""
    if a == -b:
        return 0
    if abs(a) > LLR_MAX:
        return a
    if abs(b) > LLR_MAX:
        return b
    return max(-LLR_MAX, min(LLR_MAX, a + b))


def promotion_sum(a, b):
    """log_likelihood_ratio::promotion_sum (log_likelihood_ratio.cpp:57-70)."""
    if a == -b:
        return 0
    if abs(a) > LLR_MAX:
        return a
    if abs(b) > LLR_MAX:
        return b
    t = a + b
    return LLR_INF if t > LLR_MAX else (-LLR_INF if t < -LLR_MAX else t)


def soft_xor(x, y):
    m = min(abs(x), abs(y))
    return -m if x * y < 0 else m


def nof_codeblocks(A, E):
    return 2 if (A >= 360 and E >= 1088) or A >= 1013 else 1


def crc_size(A):
    return 0 if A < 12 else (6 if A < 20 else 11)


def rate_dematch(f, code, K):
    """polar_rate_dematcher_impl::rate_dematch with the channel interleaver present."""
    E, N = len(f), code["N"]
    # Channel de-interleaver (:53-79).
    T = 1
    while T * (T + 1) // 2 < E:
        T += 1
    e = [0] * E
    i_out = 0
    for r in range(T):
        i_in = r
        for c in range(T - r):
            if i_in >= E:
                break
            e[i_in] = int(f[i_out])
            i_out += 1
            i_in += T - c
    # Bit selection (:21-50).
    if E >= N:
        y = e[:N]
        for k in range(N, E):
            y[k % N] = promotion_sum(y[k % N], e[k])
    elif 16 * K <= 7 * E:
        y = [0] * (N - E) + e
    else:
        y = e + [LLR_INF] * (N - E)
    # Sub-block de-interleaver (:12-19).
    out = [0] * N
    for j in range(N):
        out[int(code["subblock"][j])] = y[j]
    return out


def polar_encode(x):
    """polar_encoder_impl::encode: the butterfly transform of F^{(x) n}."""
    u = list(x)
    h = 1
    while h < len(u):
        for i in range(len(u)):
            if i & h == 0:
                u[i] ^= u[i + h]
        h <<= 1
    return u


def ssc_decode(llr, info):
    """polar_decoder_impl::decode: returns the sub-channel bits u (N)."""
    N = len(llr)
    u = [0] * N

    def node(s, j, l):
        lo, hi = j << s, (j + 1) << s
        nk = int(info[lo:hi].sum())
        if nk == 0:  # rate 0 (:163-178)
            return [0] * (hi - lo)
        if nk == hi - lo:  # rate 1 (:180-205)
            x = [1 if v <= 0 else 0 for v in l]
            u[lo:hi] = polar_encode(x)
            return x
        h = (hi - lo) // 2  # rate R (:207-254)
        xl = node(s - 1, 2 * j, [soft_xor(l[i], l[i + h]) for i in range(h)])
        xr = node(s - 1, 2 * j + 1, [sat_sum(l[i + h], -l[i] if xl[i] else l[i]) for i in range(h)])
        return [a ^ b for a, b in zip(xl, xr)] + xr

    node(int(np.log2(N)), 0, list(llr))
    return u


def crc_remainder(bits, L):
    poly = 0x621 if L == 11 else 0x21
    mask, reg = (1 << L) - 1, 0
    for b in bits:
        top = ((reg >> (L - 1)) ^ int(b)) & 1
        reg = (reg << 1) & mask
        if top:
            reg ^= poly
    return reg


def decode_codeblock(f, code, K, nof_filler, nbits, L):
    """uci_decoder_impl::decode_codeblock_polar: (payload bits, valid)."""
    u = ssc_decode(rate_dematch(f, code, K), code["k_set"])
    pcs = sorted(code["pc_set"][:code["nPC"]]) + [1024]
    msg, ipc = [], 0
    for i in np.flatnonzero(code["k_set"]):  # polar_deallocator_impl.cpp:10-24
        if i == pcs[ipc]:
            ipc += 1
        elif len(msg) < K:
            msg.append(u[i])
    valid = crc_remainder(msg, L) == 0
    return np.array(msg[nof_filler:nof_filler + nbits], np.uint8), valid


def uci_polar_decode(A, llrs, polar_code):
    """uci_decoder_impl::decode_codeword_polar (:25-58); polar_code(K, E) gives the code dict."""
    E = len(llrs)
    C, L = nof_codeblocks(A, E), crc_size(A)
    A0, E0, F = A // C, E // C, A % C
    bits0, ok = decode_codeblock(llrs[:E0], polar_code(A0 + L + F, E0), A0 + L + F, F, A0, L)
    if C == 1:
        return bits0, ok
    A1 = -(-A // C)
    bits1, ok1 = decode_codeblock(llrs[E0:], polar_code(A1 + L, E - E0), A1 + L, 0, A1, L)
    return np.concatenate([bits0, bits1]), ok and ok1

"""Pseudo-random sequences of TS 38.211 Section 5.2.1 (Gold sequence of length 31) and the
sequences built on it: PUSCH DM-RS type 1 pilots (Section 6.4.1.1) and data scrambling (Section
6.3.1.1). Numpy, used by the seeded simulator and by host-side set-up."""
import functools

import numpy as np

NC = 1600


def gold(c_init, length, offset=0):
    """c(offset), ..., c(offset + length - 1) as uint8."""
    n = NC + offset + length + 31
    x1 = np.zeros(n, np.uint8)
    x2 = np.zeros(n, np.uint8)
    x1[0] = 1
    x2[:31] = (int(c_init) >> np.arange(31)) & 1
    i = 0
    while i + 31 < n:
        k = min(28, n - 31 - i)  # the recurrences reach back 28 positions at most
        x1[i + 31:i + 31 + k] = x1[i + 3:i + 3 + k] ^ x1[i:i + k]
        x2[i + 31:i + 31 + k] = x2[i + 3:i + 3 + k] ^ x2[i + 2:i + 2 + k] ^ x2[i + 1:i + 1 + k] ^ x2[i:i + k]
        i += k
    s = NC + offset
    return x1[s:s + length] ^ x2[s:s + length]


def dmrs_c_init(slot, symbol, n_id, n_scid=0, nsymb=14):
    return ((nsymb * slot + symbol + 1) * (2 * n_id + 1) * (1 << 17) + (2 * n_id + n_scid)) % (1 << 31)


def dmrs_type1(slot, symbol, n_id, rb_start, nof_rb, nof_layers, n_scid=0):
    """Pilots [layer][6*nof_rb] on the even subcarriers of the allocation (CDM group 0; layer 1
    carries the frequency OCC [+1, -1]), amplitude 1/sqrt(2), before the DM-RS scaling."""
    m0 = 6 * rb_start
    c = gold(dmrs_c_init(slot, symbol, n_id, n_scid), 2 * 6 * nof_rb, offset=2 * m0).astype(np.float32)
    r = ((1 - 2 * c[0::2]) + 1j * (1 - 2 * c[1::2])) / np.sqrt(2.0)
    out = np.repeat(r[None, :], nof_layers, axis=0).astype(np.complex64)
    if nof_layers > 1:
        out[1, 1::2] *= -1
    return out


def scrambling_c_init(rnti, n_id):
    """PUSCH data scrambling initialisation (TS 38.211 Section 6.3.1.1)."""
    return (rnti << 15) + n_id


def scrambling(rnti, n_id, length):
    return gold(scrambling_c_init(rnti, n_id), length)

"""The two-lanes-per-thread LDPC decoder's f16 arithmetic (csrc/ldpc_decoder.cu): every f16x2
constant is the exact f16 encoding of the integer it names, and the identities it uses are exact
over their whole input ranges (no GPU needed)."""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "ocudu-dapp-platform_b200", "csrc", "ldpc_decoder.cu")


def f16_bits(v):
    return int(np.array([np.float16(v)]).view(np.uint16)[0])


def test_f16x2_constants_are_exact():
    text = open(SRC).read()
    found = re.findall(r"constexpr uint32_t (kHm?\w+)\s*=\s*0x([0-9a-f]+)u; // (-?\d+(?:\.\d+)?)(?=\s|$)", text, re.M)
    assert len(found) >= 12
    for name, hexv, val in found:
        assert float(np.float16(float(val))) == float(val), name
        w = f16_bits(float(val))
        assert int(hexv, 16) == (w | (w << 16)), (name, hexv, val)
    # f16(0.8), the one constant that is not exact.
    m = re.search(r"constexpr uint32_t kH0p8\s*=\s*0x([0-9a-f]+)u;", text)
    w = f16_bits(0.8)
    assert int(m.group(1), 16) == (w | (w << 16))


def test_scale_as_f16_fma():
    """The Z = 384 decoder's 0.8 scaling max(fma(m, f16(0.8), 1023.5) - 1024, 0), rounded to f16 at
    each step, equals the reference's (m * 52428) >> 16 for every magnitude 0 <= m <= 120."""
    m = np.arange(0, 121)
    r = fma16(m, np.float16(0.8), 1023.5)
    s = np.maximum((r.astype(np.float64) - 1024).astype(np.float16), 0)
    assert (s.astype(np.int64) == (m * 52428) >> 16).all()


def fma16(a, b, c):
    return np.float16(np.float64(a) * np.float64(b) + np.float64(c))


def kernel_v(x, c, first):
    """The decoder's v (arrays): clamp(x - c) (not in the first iteration) bounded by
    104x -+ 12984, each step rounded to f16 as the f16x2 instructions do."""
    x16 = x.astype(np.float16)
    d = x16 if first else np.clip(x16 - c.astype(np.float16), -120, 120).astype(np.float16)
    lo = (x.astype(np.float64) * 104 - 12984).astype(np.float16)
    hi = (x.astype(np.float64) * 104 + 12984).astype(np.float16)
    return np.minimum(np.maximum(d, lo), hi)


def kernel_soft(v, cnew):
    t = (cnew.astype(np.float16) + v.astype(np.float16)).astype(np.float16)
    cl = np.clip(t, -120, 120).astype(np.float16)
    t8 = (t * np.float16(8)).astype(np.float16)
    return np.clip((cl.astype(np.float64) * -7 + t8.astype(np.float64)).astype(np.float16), -127, 127)


def test_identities_exact():
    """Over the reference's LLR domain ([-120, 120] and +-127; raw first-iteration tails up to
    +-126 too) and every stored message c and new message cnew (|.| <= 96): the decoder's v equals
    the reference's v2c except +-224 for +-127, which acts the same in the minimum search (start
    120) and in the message magnitude test, and the soft update gives the reference's value."""
    dom = np.array(list(range(-120, 121)) + [127, -127])
    cnew = np.arange(-96, 97)
    for first in (True, False):
        xs = np.array(list(range(-126, 127)) + [127, -127]) if first else dom
        cs = np.array([0]) if first else np.arange(-96, 97)
        x, c = np.meshgrid(xs, cs, indexing="ij")
        x, c = x.ravel(), c.ravel()
        ref = x if first else np.where(np.abs(x) == 127, x, np.clip(x - c, -120, 120))
        v = kernel_v(x, c, first).astype(np.float64)
        sat = np.abs(ref) == 127
        assert np.array_equal(v[sat], 224.0 * np.sign(ref[sat]))
        assert np.array_equal(v[~sat], ref[~sat].astype(np.float64))
        # Soft update for every new message.
        vv, rr = np.repeat(v, cnew.size), np.repeat(ref, cnew.size)
        cc = np.tile(cnew, v.size)
        t = cc + rr
        want = np.where(np.abs(rr) == 127, rr, np.where(t > 120, 127, np.where(t < -120, -127, t)))
        got = kernel_soft(vv, cc).astype(np.float64)
        assert np.array_equal(got, want.astype(np.float64))
    # promote(t) = clamp(8t - 7 clamp(t, +-120), +-127) for every t the update can see.
    for t in range(-320, 321):
        cl = np.clip(np.float16(t), -120, 120)
        u = np.clip(fma16(cl, -7, np.float16(t) * np.float16(8)), -127, 127)
        assert u == (127 if t > 120 else (-127 if t < -120 else t)), t
    # The message magnitude: s2 + (s1 - s2) * (|v| != min1) picks s2 exactly when |v| == min1.
    for m1 in range(0, 121):
        for a in list(range(0, 121)) + [224]:
            ne = np.float16(1.0 if np.float16(a) != np.float16(m1) else 0.0)
            for s1, s2 in ((0, 0), (3, 7), (96, 96), (40, 95)):
                mag = fma16(np.float16(s1) - np.float16(s2), ne, s2)
                assert mag == (s2 if a == m1 else s1)
    for b in range(1, 256):  # offset-binary byte <-> f16 through 1024 + byte
        v = np.float16(np.array([0x6400 | b], np.uint16).view(np.float16)[0]) - np.float16(1152)
        assert v == b - 128
        back = int(np.array([np.float16(v) + np.float16(1152)]).view(np.uint16)[0]) & 0xff
        assert back == b
    keys = [f16_bits(m) >> 4 for m in range(128)]
    assert len(set(keys)) == 128 and max(keys) < 1408


LIFTING_ABOVE_192 = [208, 224, 240, 256, 288, 320, 352, 384]


def pair_pos(ed, j, H):
    """The decoder's pair_pos: shared-memory pair index | swapped << 16 (32-bit unsigned)."""
    t = j + (ed & 0xFF)
    u = (t - H) & 0xFFFFFFFF
    w = min(t, u)
    sw = ((ed >> 8) ^ (1 if u < t else 0)) & 1
    return ((ed >> 9) + w) | (sw << 16)


def test_pair_store_addressing_covers_both_lanes():
    """Pair mode: for every lifting size above 192, every shift and every thread j < Z/2, the
    pair read for an edge holds variable lanes (j + s) mod Z (low half after the swap) and
    (j + Z/2 + s) mod Z (high half), and the threads of a row touch disjoint pairs."""
    for Z in LIFTING_ABOVE_192:
        H = Z // 2
        assert H % 8 == 0 and Z % 16 == 0
        col = 5
        for s in range(Z):
            f = 1 if s >= H else 0
            ed = ((col * 192) << 9) | (f << 8) | (s - f * H)
            seen = set()
            for j in range(H):
                p = pair_pos(ed, j, H)
                idx, sw = p & 0xFFFF, p >> 16
                wp = idx - col * 192
                assert 0 <= wp < H
                lanes = (wp, wp + H)  # D[col][w'] = (soft[w'], soft[w' + H])
                lo, hi = (lanes[1], lanes[0]) if sw else lanes
                assert lo == (j + s) % Z and hi == (j + H + s) % Z, (Z, s, j)
                assert idx not in seen
                seen.add(idx)


def test_pair_soft_byte_column_division_exact():
    """(i * ceil(2^24 / Z)) >> 24 is i // Z for every message bit i of both base graphs."""
    for Z in LIFTING_ABOVE_192:
        inv = ((1 << 24) + Z - 1) // Z
        i = np.arange(22 * Z, dtype=np.int64)
        assert ((i * inv) < 2 ** 32).all()
        assert np.array_equal((i * inv) >> 24, i // Z)


def test_pair_fill_layout():
    """The soft-bit fill: chunk q of eight pairs (column q // (H/8)) reads LLR indices k .. k+7 and
    k+H .. k+H+7 with k = (col - 2) Z + w0, and writes pairs D[col*192 + w0 + i] = (k + i, k + H + i);
    over all chunks this is every soft bit of the nfull columns exactly once."""
    for Z in LIFTING_ABOVE_192:
        H = Z // 2
        per_col = H // 8
        for nfull in (68, 52):
            got = {}
            for q in range(nfull * per_col):
                col = q // per_col
                w0 = (q - col * per_col) * 8
                k = (col - 2) * Z + w0
                for i in range(8):
                    got[col * 192 + w0 + i] = (k + i, k + H + i)
            soft = set()
            for idx, (a, b) in got.items():
                col, wp = divmod(idx, 192)
                assert a == col * Z + wp - 2 * Z and b == a + H
                soft.update((a, b))
            assert soft == set(range(-2 * Z, (nfull - 2) * Z))


def z_kernel_v(x, c, first):
    """The Z = 384 decoder's v: as kernel_v, on soft bits that may also be saturated as any
    magnitude of at least 128 or f16 infinity."""
    x16 = x.astype(np.float16)
    with np.errstate(over="ignore", invalid="ignore"):
        d = x16 if first else np.clip((x16.astype(np.float64) - c).astype(np.float16), -120, 120).astype(np.float16)
        lo = (x16.astype(np.float64) * 104 - 12984).astype(np.float16)
        hi = (x16.astype(np.float64) * 104 + 12984).astype(np.float16)
    return np.minimum(np.maximum(d, lo), hi)


def z_kernel_soft(v, cnew):
    """The Z = 384 decoder's soft update: 8t - 7 clamp(t, +-120) without the final clamp."""
    with np.errstate(over="ignore", invalid="ignore"):
        t = (cnew.astype(np.float64) + v.astype(np.float64)).astype(np.float16)
        cl = np.clip(t, -120, 120).astype(np.float16)
        t8 = (t.astype(np.float64) * 8).astype(np.float16)
        return (cl.astype(np.float64) * -7 + t8.astype(np.float64)).astype(np.float16)


def test_z384_unclamped_saturation_acts_as_127():
    """Soft bits the reference saturates to +-127 are, in the Z = 384 decoder, any magnitude of at
    least 128 or infinity (no clamp after the soft update). Over every finite soft bit, saturated
    ones of many magnitudes, every stored message c and new message cnew (|.| <= 96): the v2c has
    the reference's sign, acts alike in the minimum search (start 120) and the message-magnitude
    test, and the soft update gives the reference's value, saturated ones as magnitudes >= 128,
    never a NaN and never a magnitude in (120, 128)."""
    big = [128, 129, 200, 1000, 2047, 5000, 60000, np.inf]
    for first in (True, False):
        fin = list(range(-126, 127)) if first else list(range(-120, 121))
        xs = np.array(fin + [127, -127] + big + [-b for b in big], np.float64)
        cs = np.array([0]) if first else np.arange(-96, 97)
        cnew = np.arange(-96, 97)
        x, c, cn = np.meshgrid(xs, cs, cnew, indexing="ij")
        x, c, cn = x.ravel(), c.ravel(), cn.ravel()
        sat = np.abs(x) >= 127
        xr = np.where(sat, np.sign(x) * 127, x)                      # the reference's soft bit
        ref_v = xr if first else np.where(sat, xr, np.clip(xr - c, -120, 120))
        v = z_kernel_v(x, c, first).astype(np.float64)
        assert not np.isnan(v).any()
        assert (np.sign(v) == np.sign(ref_v)).all()
        assert (np.minimum(np.abs(v), 120) == np.minimum(np.abs(ref_v), 120)).all()
        fin_v = np.abs(ref_v) < 127
        assert (v[fin_v] == ref_v[fin_v]).all()
        assert (np.abs(v[~fin_v]) >= 217).all()
        ref_t = cn + ref_v
        ref_soft = np.where(np.abs(ref_v) == 127, ref_v, np.where(np.abs(ref_t) > 120, np.sign(ref_t) * 127, ref_t))
        u = z_kernel_soft(v, cn).astype(np.float64)
        assert not np.isnan(u).any()
        assert not ((np.abs(u) > 120) & (np.abs(u) < 128)).any()
        got = np.where(np.abs(u) >= 128, np.sign(u) * 127, u)
        assert (got == ref_soft).all()

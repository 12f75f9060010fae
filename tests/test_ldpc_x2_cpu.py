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
    found = re.findall(r"constexpr uint32_t (kHm?\w+)\s*=\s*0x([0-9a-f]+)u; // (-?\d+)", text)
    assert len(found) >= 10
    for name, hexv, val in found:
        assert float(np.float16(int(val))) == int(val), name
        w = f16_bits(int(val))
        assert int(hexv, 16) == (w | (w << 16)), (name, hexv, val)


def fma16(a, b, c):
    return np.float16(np.float64(a) * np.float64(b) + np.float64(c))


def test_identities_exact():
    for x in list(range(-120, 121)) + [127, -127]:
        lo, hi = fma16(x, 37, -4572), fma16(x, 37, 4572)
        for c in range(-96, 97):
            d = np.clip(np.float16(x) - np.float16(c), -120, 120)
            v = min(max(d, lo), hi)
            assert v == (x if abs(x) == 127 else max(-120, min(120, x - c))), (x, c)
    for t in range(-223, 224):
        cl = np.clip(np.float16(t), -120, 120)
        u = np.clip(fma16(cl, -7, np.float16(t) * np.float16(8)), -127, 127)
        assert u == (127 if t > 120 else (-127 if t < -120 else t)), t
    for b in range(1, 256):  # offset-binary byte <-> f16 through 1024 + byte
        v = np.float16(np.array([0x6400 | b], np.uint16).view(np.float16)[0]) - np.float16(1152)
        assert v == b - 128
        back = int(np.array([np.float16(v) + np.float16(1152)]).view(np.uint16)[0]) & 0xff
        assert back == b
    keys = [f16_bits(m) >> 4 for m in range(128)]
    assert len(set(keys)) == 128 and max(keys) < 1408

"""Open Fronthaul BFP decompression without a GPU: a numpy restatement of the reference's two
roundings (the x86 vector decompressor for 9, 14 and 16 bits, the generic one otherwise),
checked against the reference's compiled decompressor on data its compressor produced and on
random payloads; the library's compressed PRB size against the reference's."""
import numpy as np

from pusch_b200 import _native


def bf16_rne(f32):
    u = np.asarray(f32, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) & 0xFFFF


def restated_decompress(width, data, nprb):
    """Per PRB: exponent byte, 24 big-endian fields of `width` bits, sign-extended, scaled."""
    pb = 1 + 3 * width
    out = np.zeros(12 * nprb, np.uint32)
    mul = width in (9, 14, 16)
    for p in range(nprb):
        b = data[p * pb:(p + 1) * pb]
        e = int(b[0])
        bits = np.unpackbits(b[1:])
        vals = []
        for k in range(24):
            f = bits[k * width:(k + 1) * width]
            v = int("".join(map(str, f)), 2) if width else 0
            if v >= 1 << (width - 1):
                v -= 1 << width
            vals.append(v)
        vals = np.array(vals, np.int64)
        if mul:
            scale = np.float32(np.float32(1 << e) / np.float32(32767.0))
            f = (vals.astype(np.float32) * scale).astype(np.float32)
        else:
            scaler = np.int64(np.int16(np.int64(1 << e).astype(np.int16)))
            f = ((vals * scaler).astype(np.float32) / np.float32(32767.0)).astype(np.float32)
        h = bf16_rne(f)
        out[12 * p:12 * p + 12] = h[0::2] | (h[1::2] << 16)
    return out


def random_grid_words(rng, nprb, scale):
    x = (rng.standard_normal(24 * nprb) * scale).astype(np.float32)
    h = bf16_rne(x)
    return (h[0::2] | (h[1::2] << 16)).astype(np.uint32)


def test_prb_size_matches_reference(ref):
    lib = _native.load()
    rng = np.random.default_rng(0)
    for w in range(1, 17):
        data = ref.bfp_compress(w, random_grid_words(rng, 2, 0.1))
        assert lib.pg_bfp_prb_bytes(w) == data.size // 2 == 1 + 3 * w
    assert lib.pg_bfp_prb_bytes(0) < 0 and lib.pg_bfp_prb_bytes(17) < 0


def test_restatement_matches_reference(ref):
    rng = np.random.default_rng(3)
    for w in (2, 4, 7, 8, 9, 12, 14, 15, 16):
        nprb = 24
        data = ref.bfp_compress(w, random_grid_words(rng, nprb, 0.2))
        want, _ = ref.bfp_decompress(w, data, nprb)
        assert np.array_equal(restated_decompress(w, data, nprb), want), w
        raw = rng.integers(0, 256, nprb * (1 + 3 * w), dtype=np.uint8)
        raw[::1 + 3 * w] = rng.integers(0, 16 - w + 1, nprb)  # exponents of the format's range
        want, _ = ref.bfp_decompress(w, raw, nprb)
        assert np.array_equal(restated_decompress(w, raw, nprb), want), w


def test_simulator_compressor_matches_reference(ref):
    """The simulator's BFP compressor (the radio unit's side, used to feed the benchmark) writes the
    same bytes as the reference's compressor for widths 8 to 16, saturation included. (Below 8 bits
    the reference's generic packer writes the sign-extension bits of a negative sample into the
    preceding field, so its bytes are not the format's; decompression is compared on the reference's
    own bytes for every width.)"""
    from pusch_b200 import sim
    rng = np.random.default_rng(2)
    for w in range(8, 17):
        for scale in (0.01, 0.2, 3.0):
            g = random_grid_words(rng, 300, scale)
            assert np.array_equal(sim.bfp_compress(g, w), ref.bfp_compress(w, g)), (w, scale)

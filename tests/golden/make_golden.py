"""Generates the golden fixtures in tests/golden/ from the reference's own compiled CPU code
(oracle/_ref/libocudu_ref.so, built by `make -C oracle ref` from the reference sources).

Inputs come from this project's seeded simulator; outputs (decoded bits, iteration counts, CRCs,
dematched buffers, encoded codewords) come from the reference. Run in a container that holds the
reference:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ocudu-dapp-platform_b200"))

from oracle import Ref  # noqa: E402
from pusch_b200 import codec  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def kb(bg):
    return 22 if bg == 1 else 10


def nshort(bg):
    return 66 if bg == 1 else 50


def make_cb(rng, bg, z, filler, crc_poly, e_len, ebn0, scale=4.0):
    """A rate-dematched-style LLR buffer of length N: noisy LLRs for the first e_len positions of
    the shortened codeword, +127 at filler positions, zeros after e_len."""
    k = kb(bg) * z
    order = 16 if crc_poly == 0 else 24
    info = rng.integers(0, 2, k - filler - order, dtype=np.uint8)
    msg = np.concatenate([codec.attach_crc(crc_poly, info), np.zeros(filler, np.uint8)])
    cw = codec.ldpc_encode(bg, z, msg)
    n = nshort(bg) * z
    sigma = np.sqrt(1.0 / (2.0 * (k / max(e_len, 1)) * 10.0 ** (ebn0 / 10.0)))
    y = (1.0 - 2.0 * cw) + sigma * rng.standard_normal(n)
    llr = np.clip(np.rint(2.0 * y / sigma ** 2 * scale), -120, 120).astype(np.int8)
    llr[e_len:] = 0
    if filler:
        llr[k - 2 * z - filler:k - 2 * z] = 127
    return llr


def ldpc_cases(ref, rng):
    cases = []
    # Config-2 shaped codeblocks: BG1/BG2 Z=384, full buffer, CRC24B, 10 iterations.
    for i in range(8):
        bg = 1 + (i % 2)
        cases.append((bg, 384, 0, 2, 10, nshort(bg) * 384, 1.0 + 0.25 * i))
    # Assorted lifting sizes, fillers, shortened inputs, CRC polynomials and iteration caps.
    for bg, z, f, poly, it, frac, eb in [
        (1, 2, 8, 0, 6, 1.0, 3.0), (2, 3, 5, 0, 6, 0.8, 2.0), (1, 7, 20, 0, 8, 0.6, 3.0),
        (2, 15, 30, 1, 6, 0.7, 2.5), (1, 64, 100, 1, 6, 0.5, 4.0), (2, 208, 0, 2, 10, 0.9, 1.5),
        (1, 288, 424, 1, 6, 0.45, 5.0), (2, 384, 72, 2, 4, 0.6, 3.0), (1, 384, 64, 2, 6, 0.5, 6.0),
        (1, 160, 0, 2, 1, 1.0, 3.0), (2, 52, 12, 0, 20, 1.0, 0.5), (1, 384, 0, 2, 10, 1.0, -1.0),
        (1, 120, 0, 255, 6, 0.8, 4.0), (2, 96, 8, 255, 6, 1.0, 0.0),
    ]:
        n = nshort(bg) * z
        k = kb(bg) * z
        e_len = max(int(frac * n), k + 2 * z)
        cases.append((bg, z, f, poly, it, e_len, eb))
    meta, llrs, bits, iters = [], [], [], []
    for (bg, z, f, poly, it, e_len, eb) in cases:
        cpoly = 2 if poly == 255 else poly
        llr = make_cb(rng, bg, z, f, cpoly, e_len, eb)
        nof_crc = 16 if cpoly == 0 else 24
        got, out = ref.ldpc_decode(bg, z, llr, filler=f, crc_poly=(-1 if poly == 255 else poly), max_iter=it,
                                   nof_crc_bits=nof_crc)
        meta.append([bg, z, f, poly, it, llr.size])
        llrs.append(llr)
        bits.append(out)
        iters.append(got)
    # Special inputs: all zeros, and fewer than K*Z significant soft bits (both fail, all ones).
    for bg, z in [(1, 384), (2, 64)]:
        n = nshort(bg) * z
        k = kb(bg) * z
        for kind in ("zeros", "short"):
            llr = np.zeros(n, np.int8)
            if kind == "short":
                llr[: k - 3] = rng.integers(-120, 121, k - 3)
            got, out = ref.ldpc_decode(bg, z, llr, filler=0, crc_poly=2, max_iter=6, prefill=0xFF)
            meta.append([bg, z, 0, 2, 6, n])
            llrs.append(llr)
            bits.append(out)
            iters.append(got)
    off = np.cumsum([0] + [x.size for x in llrs])
    boff = np.cumsum([0] + [x.size for x in bits])
    return dict(meta=np.array(meta, np.int32), llr_offsets=off.astype(np.int64), llrs=np.concatenate(llrs),
                bit_offsets=boff.astype(np.int64), bits=np.concatenate(bits), iterations=np.array(iters, np.int32))


def rm_cases(ref, rng):
    meta, ins, prevs, outs = [], [], [], []
    for t in range(30):
        bg = 1 + t % 2
        z = [384, 64, 16, 7, 2, 104, 36, 13, 22, 8][t % 10]
        qm = [1, 2, 4, 6, 8][t % 5]
        rv = (t // 5) % 4
        k = kb(bg) * z
        n = nshort(bg) * z
        f = int(rng.integers(0, (k - 2 * z) // 3))
        nref = 0 if t % 3 else int(rng.integers(k, n + 1))
        e = qm * int(rng.integers(1, (13 * n) // (10 * qm)))
        llr = rng.integers(-120, 121, e).astype(np.int8)
        prev = rng.integers(-120, 121, n).astype(np.int8)
        new_data = int(t % 4 != 3)
        out = ref.rate_dematch(bg, z, llr, rv=rv, qm=qm, Nref=nref, filler=f, new_data=new_data, out=prev.copy())
        meta.append([bg, z, rv, qm, nref, f, new_data, e])
        ins.append(llr)
        prevs.append(prev)
        outs.append(out)
    return dict(meta=np.array(meta, np.int32), in_offsets=np.cumsum([0] + [x.size for x in ins]).astype(np.int64),
                ins=np.concatenate(ins), buf_offsets=np.cumsum([0] + [x.size for x in prevs]).astype(np.int64),
                prevs=np.concatenate(prevs), outs=np.concatenate(outs))


def crc_cases(ref, rng):
    meta, bits, crcs = [], [], []
    for poly in (0, 1, 2):
        for length in (1, 7, 8, 9, 31, 33, 100, 1000, 3816, 8424, 8448):
            b = rng.integers(0, 2, length, dtype=np.uint8)
            meta.append([poly, length])
            bits.append(b)
            crcs.append(ref.crc(poly, b))
    return dict(meta=np.array(meta, np.int32), offsets=np.cumsum([0] + [x.size for x in bits]).astype(np.int64),
                bits=np.concatenate(bits), crcs=np.array(crcs, np.uint32))


def enc_cases(ref, rng):
    meta, msgs, cws = [], [], []
    for bg, z in [(1, 384), (2, 384), (1, 2), (2, 7), (1, 288), (2, 208), (1, 15), (2, 52)]:
        k = kb(bg) * z
        m = rng.integers(0, 2, k, dtype=np.uint8)
        meta.append([bg, z])
        msgs.append(m)
        cws.append(ref.ldpc_encode(bg, z, m))
    return dict(meta=np.array(meta, np.int32), msg_offsets=np.cumsum([0] + [x.size for x in msgs]).astype(np.int64),
                msgs=np.concatenate(msgs), cw_offsets=np.cumsum([0] + [x.size for x in cws]).astype(np.int64),
                cws=np.concatenate(cws))


def to_cbf16(x):
    x = np.ascontiguousarray(x, np.complex64)
    u = x.view(np.float32).reshape(x.shape + (2,)).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF
    return (r[..., 0] | (r[..., 1] << 16)).astype(np.uint32)


def demap_cases(ref, rng):
    meta, syms, nvs, llrs = [], [], [], []
    for qm in (2, 4, 6, 8):
        n = 3000
        s = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) * rng.uniform(0.2, 1.2)).astype(np.complex64)
        s[:8] = 0
        s[8:16] = 1e-10
        nv = rng.uniform(1e-3, 1.0, n).astype(np.float32)
        nv[16:20] = 0
        nv[20] = np.inf
        meta.append([qm, n])
        syms.append(s)
        nvs.append(nv)
        llrs.append(ref.demodulate_soft(qm, s, nv))
    return dict(meta=np.array(meta, np.int32), symbols=np.concatenate(syms), noise=np.concatenate(nvs),
                llrs=np.concatenate(llrs))


def eq_cases(ref, rng):
    out = {}
    for idx, (alg, p, l, nre) in enumerate([(1, 2, 1, 612), (1, 4, 1, 600), (1, 4, 2, 3276), (1, 2, 2, 500),
                                           (0, 2, 1, 300), (1, 8, 2, 256), (1, 4, 4, 256)]):
        y = to_cbf16((rng.standard_normal((p, nre)) + 1j * rng.standard_normal((p, nre))) / np.sqrt(2))
        h = to_cbf16((rng.standard_normal((p, l, nre)) + 1j * rng.standard_normal((p, l, nre))) / np.sqrt(2))
        h[:, :, :3] = 0  # zero channel: (0, inf) outputs
        nv = rng.uniform(0.01, 0.3, p).astype(np.float32)
        tx = float(rng.choice([1.0, 0.7071]))
        eq, var = ref.equalize(alg, y, h, nv, tx)
        out[f"c{idx}_meta"] = np.array([alg, p, l, nre], np.int32)
        out[f"c{idx}_y"] = y
        out[f"c{idx}_h"] = h
        out[f"c{idx}_nv"] = nv
        out[f"c{idx}_tx"] = np.array([tx], np.float32)
        out[f"c{idx}_eq"] = eq
        out[f"c{idx}_var"] = var
    return out


def est_cases(ref):
    from pusch_b200 import sim
    out = {}
    cases = [dict(rb_start=3, nof_rb=51, nof_layers=1, ports=2, dmrs=(2,), channel="flat", snr=10.0),
             dict(rb_start=10, nof_rb=20, nof_layers=2, ports=4, dmrs=(2, 11), channel="pdp", snr=20.0),
             dict(rb_start=0, nof_rb=1, nof_layers=1, ports=1, dmrs=(3,), channel="flat", snr=5.0),
             dict(rb_start=57, nof_rb=2, nof_layers=2, ports=2, dmrs=(2, 11), channel="pdp", snr=15.0)]
    beta = float(np.float32(10 ** (3 / 20)))
    for i, c in enumerate(cases):
        ue = sim.PuschUe(rb_start=c["rb_start"], nof_rb=c["nof_rb"], nof_layers=c["nof_layers"], modulation_order=2,
                         tbs_bits=24 if c["nof_rb"] < 3 else 1000, base_graph=2, dmrs_symbols=c["dmrs"],
                         snr_db=c["snr"], channel=c["channel"], n_id=17 * i, rnti=0x4601 + i)
        slot = sim.make_pusch_slot([ue], c["ports"], nof_prb_grid=60, slot=i + 1, seed=100 + i)
        out[f"c{i}_meta"] = np.array([c["rb_start"], c["nof_rb"], c["nof_layers"], c["ports"], i + 1, 17 * i,
                                      0x4601 + i, sum(1 << s for s in c["dmrs"])], np.int32)
        out[f"c{i}_grid"] = slot.grid
        for p in range(c["ports"]):
            freq, sym, sc = ref.port_estimate(slot.grid, p, i + 1, 17 * i, c["rb_start"], c["nof_rb"], c["nof_layers"],
                                              list(c["dmrs"]), beta)
            out[f"c{i}_p{p}_freq"] = freq
            out[f"c{i}_p{p}_sym"] = sym
            out[f"c{i}_p{p}_scalars"] = np.array([sc["noise_var"], sc["epre"], sc["snr"], *sc["rsrp"]], np.float64)
    return out


def est_full_cell_case(ref):
    """One full-cell allocation at the headline shape: 273 PRB, 4 receive ports, 2 layers, DM-RS at
    symbols 2 and 11, exponential-PDP channel at 25 dB (estimate_273prb.npz, same keys as
    estimate.npz)."""
    from pusch_b200 import sim
    out = {}
    beta = float(np.float32(10 ** (3 / 20)))
    ue = sim.PuschUe(rb_start=0, nof_rb=273, nof_layers=2, modulation_order=8, tbs_bits=417976, base_graph=1,
                     dmrs_symbols=(2, 11), snr_db=25.0, channel="pdp", n_id=301, rnti=0x4711)
    slot = sim.make_pusch_slot([ue], 4, nof_prb_grid=273, slot=7, seed=273)
    out["c0_meta"] = np.array([0, 273, 2, 4, 7, 301, 0x4711, (1 << 2) | (1 << 11)], np.int32)
    out["c0_grid"] = slot.grid
    for p in range(4):
        freq, sym, sc = ref.port_estimate(slot.grid, p, 7, 301, 0, 273, 2, [2, 11], beta)
        out[f"c0_p{p}_freq"] = freq
        out[f"c0_p{p}_sym"] = sym
        out[f"c0_p{p}_scalars"] = np.array([sc["noise_var"], sc["epre"], sc["snr"], *sc["rsrp"]], np.float64)
    return out


def main():
    ref = Ref()
    rng = np.random.default_rng(20261203)
    np.savez_compressed(os.path.join(OUT, "ldpc_decode.npz"), variant=ref.variant, **ldpc_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "rate_dematch.npz"), **rm_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "crc.npz"), **crc_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "ldpc_encode.npz"), **enc_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "demap.npz"), **demap_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "equalize.npz"), **eq_cases(ref, rng))
    np.savez_compressed(os.path.join(OUT, "estimate.npz"), **est_cases(ref))
    np.savez_compressed(os.path.join(OUT, "estimate_273prb.npz"), **est_full_cell_case(ref))
    print("golden fixtures written; reference LDPC variant:", ref.variant)


if __name__ == "__main__":
    main()

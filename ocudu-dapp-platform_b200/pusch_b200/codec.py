"""Transmit-side coding used by the project's seeded PUSCH simulator: CRC attachment and LDPC
encoding (TS 38.212 Sections 5.1 and 5.3.2). Numpy, vectorised over codeblocks; this is input
generation, not the measured receive path.

The encoder is this project's own: the 4Z x 4Z core-parity block of the lifted parity-check
matrix is inverted over GF(2) once per (base graph, Z); the extension parity bits then follow
row by row from the lower-triangular identity structure of rows 4.. of both base graphs.
"""
import functools
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "..", "csrc", "ldpc_base_graphs.inc")

CRC_POLYS = {0: (0x11021, 16), 1: (0x1864CFB, 24), 2: (0x1800063, 24)}  # CRC16, CRC24A, CRC24B


@functools.lru_cache(maxsize=None)
def base_graph(bg):
    """Returns (row degrees, edge columns, edge V[8]) of base graph bg from the shared table."""
    text = open(TABLE).read()

    def arr(name):
        m = re.search(r"PG_BG%d_%s\[[^\]]*\](?:\[8\])? = \{(.*?)\};" % (bg, name), text, re.S)
        return [int(x) for x in re.findall(r"\d+", m.group(1))]

    deg = np.array(arr("ROW_DEG"), np.int32)
    col = np.array(arr("EDGE_COL"), np.int32)
    v = np.array(arr("EDGE_V"), np.int32).reshape(-1, 8)
    return deg, col, v


def set_index(z):
    for i, a in enumerate((2, 3, 5, 7, 9, 11, 13, 15)):
        t = z
        while t % 2 == 0 and t > a:
            t //= 2
        if t == a:
            return i
    raise ValueError(f"{z} is not a lifting size")


@functools.lru_cache(maxsize=None)
def lifted_edges(bg, z):
    """Per row: list of (column, shift) with shift = V mod Z."""
    deg, col, v = base_graph(bg)
    s = set_index(z)
    rows, e = [], 0
    for d in deg:
        rows.append([(int(col[e + k]), int(v[e + k, s] % z)) for k in range(d)])
        e += d
    return rows


def _gf2_inverse(a):
    """Inverse of a square GF(2) matrix given as a bool array (Gauss-Jordan on packed rows)."""
    n = a.shape[0]
    aug = np.concatenate([a.astype(np.uint8), np.eye(n, dtype=np.uint8)], axis=1)
    packed = np.packbits(aug, axis=1).view(np.uint8)
    words = packed.shape[1]
    for c in range(n):
        byte, bit = c // 8, 7 - (c % 8)
        colbits = (packed[:, byte] >> bit) & 1
        cand = np.nonzero(colbits[c:])[0]
        if cand.size == 0:
            raise ValueError("singular core parity block")
        p = c + cand[0]
        if p != c:
            packed[[c, p]] = packed[[p, c]]
            colbits = (packed[:, byte] >> bit) & 1
        rows = np.nonzero(colbits)[0]
        rows = rows[rows != c]
        packed[rows] ^= packed[c]
    del words
    full = np.unpackbits(packed, axis=1)[:, : 2 * n]
    return full[:, n:].astype(np.uint8)


def _roll_rows(x, s):
    """y[..., j] = x[..., (j + s) mod Z]: the lifted circulant applied to a node."""
    return np.roll(x, -s, axis=-1)


@functools.lru_cache(maxsize=None)
def _core_inverse(bg, z):
    kb = 22 if bg == 1 else 10
    rows = lifted_edges(bg, z)
    a = np.zeros((4 * z, 4 * z), np.uint8)
    j = np.arange(z)
    for r in range(4):
        for c, s in rows[r]:
            if kb <= c < kb + 4:
                a[r * z + j, (c - kb) * z + (j + s) % z] = 1
    return _gf2_inverse(a)


def ldpc_encode(bg, z, msg):
    """Encodes message bits msg[..., K_b*Z] (fillers as 0) into the shortened codeword
    [..., N_short*Z] (the first 2Z systematic bits are not transmitted)."""
    kb = 22 if bg == 1 else 10
    m_rows = 46 if bg == 1 else 42
    msg = np.asarray(msg, np.uint8)
    lead = msg.shape[:-1]
    nodes = np.zeros(lead + (kb + m_rows, z), np.uint8)
    nodes[..., :kb, :] = msg.reshape(lead + (kb, z))
    rows = lifted_edges(bg, z)
    lam = np.zeros(lead + (4, z), np.uint8)
    for r in range(4):
        for c, s in rows[r]:
            if c < kb:
                lam[..., r, :] ^= _roll_rows(nodes[..., c, :], s)
    inv = _core_inverse(bg, z)
    rhs = lam.reshape(lead + (4 * z,)).astype(np.float32)
    core = (rhs @ inv.T.astype(np.float32)).astype(np.int64) & 1
    nodes[..., kb:kb + 4, :] = core.reshape(lead + (4, z)).astype(np.uint8)
    for r in range(4, m_rows):
        acc = np.zeros(lead + (z,), np.uint8)
        ext = kb + r
        for c, s in rows[r]:
            if c == ext:
                assert s == 0
                continue
            acc ^= _roll_rows(nodes[..., c, :], s)
        nodes[..., ext, :] = acc
    return nodes[..., 2:, :].reshape(lead + ((kb + m_rows - 2) * z,))


@functools.lru_cache(maxsize=None)
def _crc_table(poly):
    g, order = CRC_POLYS[poly]
    mask = (1 << order) - 1
    tab = np.zeros(256, np.uint32)
    for b in range(256):
        r = b << (order - 8)
        for _ in range(8):
            r = ((r << 1) ^ g) & mask if r & (1 << (order - 1)) else (r << 1) & mask
        tab[b] = r
    return tab, order, mask


def crc(poly, bits):
    """CRC (init 0, MSB first) of bits[..., L]; vectorised over leading dimensions."""
    bits = np.asarray(bits, np.uint8)
    tab, order, mask = _crc_table(poly)
    L = bits.shape[-1]
    lead = bits.shape[:-1]
    pad = (-L) % 8
    # Leading zeros do not change a zero-initialised CRC.
    b = np.concatenate([np.zeros(lead + (pad,), np.uint8), bits], axis=-1)
    by = np.packbits(b, axis=-1).astype(np.uint32)
    r = np.zeros(lead, np.uint32)
    for k in range(by.shape[-1]):
        idx = ((r >> (order - 8)) ^ by[..., k]) & 0xFF
        r = ((r << 8) & mask) ^ tab[idx]
    return r


def attach_crc(poly, bits):
    """bits[..., L] -> bits[..., L + order] with the CRC appended MSB first."""
    _, order = CRC_POLYS[poly]
    r = crc(poly, bits)
    sh = np.arange(order - 1, -1, -1, dtype=np.uint32)
    tail = ((r[..., None] >> sh) & 1).astype(np.uint8)
    return np.concatenate([np.asarray(bits, np.uint8), tail], axis=-1)


def rate_match(bg, z, cw, e, rv=0, qm=2, nref=0, nof_filler_bits=0):
    """TS 38.212 Section 5.4.2: bit selection from the circular buffer (filler bits skipped) and
    bit interleaving. cw[..., N_short*Z] -> [..., E]."""
    cw = np.asarray(cw, np.uint8)
    kb = 22 if bg == 1 else 10
    n = cw.shape[-1]
    ncb = min(nref, n) if nref > 0 else n
    sys_bits = (kb - 2) * z
    info = sys_bits - nof_filler_bits
    shift = (0, 17, 33, 56)[rv] if bg == 1 else (0, 13, 25, 43)[rv]
    k0 = (shift * ncb // n) * z
    valid = np.concatenate([np.arange(0, info), np.arange(sys_bits, ncb)])
    # Rotate the valid positions to start at k0 (or at the first valid position after it).
    start = np.searchsorted(valid, k0)
    order = np.roll(valid, -start)
    idx = order[np.arange(e) % order.size]
    sel = cw[..., idx]
    if qm > 1:
        kq = e // qm
        sel = sel.reshape(sel.shape[:-1] + (qm, kq)).swapaxes(-1, -2).reshape(sel.shape)
    return sel


# TS 38.212 Table 5.3.2-1: the 51 lifting sizes, ascending.
LIFTING_SIZES = tuple(sorted({a * (1 << j) for a in (2, 3, 5, 7, 9, 11, 13, 15) for j in range(8)
                              if a * (1 << j) <= 384}))


def segment_tx(tbs_bits, bg, qm, nof_layers, nof_ch_symbols):
    """Transmit-side segmentation of one UL-SCH transport block: codeblock count and size
    (TS 38.212 Section 5.2.2, with the K_b of Section 5.2.2 for base graph 2) and the
    rate-matching lengths E of Section 5.4.2.1 (the first C - mod(G', C) codeblocks get the floor).
    Returns the fields of pg_sch_segmentation as a dict. The simulator uses it to build its
    codewords, so input generation does not depend on the receive library."""
    if bg not in (1, 2) or tbs_bits <= 0 or not 1 <= nof_layers <= 4 or qm not in (1, 2, 4, 6, 8):
        raise ValueError("invalid segmentation request")
    if nof_ch_symbols % nof_layers:
        raise ValueError("channel symbols not a multiple of the layers")
    tb_crc = 16 if tbs_bits <= 3824 else 24
    b = tbs_bits + tb_crc
    kcb = 8448 if bg == 1 else 3840
    c = 1 if b <= kcb else -(-b // (kcb - 24))
    l = 24 if c > 1 else 0
    b_out = b + c * l
    if bg == 1:
        kb = 22
    else:
        kb = 10 if b > 640 else (9 if b > 560 else (8 if b > 192 else 6))
    z = next((ls for ls in LIFTING_SIZES if ls * c * kb >= b_out), 0)
    if z == 0:
        raise ValueError("transport block too large")
    k = (22 if bg == 1 else 10) * z
    k_prime = -(-b_out // c)
    per_layer = nof_ch_symbols // nof_layers
    return {"nof_cbs": c, "lifting_size": z, "cb_length": k, "nof_filler_bits": k - k_prime,
            "cb_crc_bits": l, "tb_crc_bits": tb_crc, "nof_short_cbs": c - per_layer % c,
            "e_short": (per_layer // c) * nof_layers * qm, "e_long": -(-per_layer // c) * nof_layers * qm}


def ulsch_encode(tb_bits, bg, qm, nof_layers, nof_ch_symbols, seg, rv=0, nref=0):
    """Transport block bits -> codeword bits (G = nof_ch_symbols * Qm): TB CRC, code block
    segmentation with CB CRC24B, filler bits, LDPC encoding and rate matching (TS 38.212
    Sections 5.1-5.4, 6.2). seg is the segmentation dictionary (pusch_b200.sch.segment)."""
    tb_bits = np.asarray(tb_bits, np.uint8)
    tbs = tb_bits.size
    b = attach_crc(0 if tbs <= 3824 else 1, tb_bits)
    c = seg["nof_cbs"]
    z = seg["lifting_size"]
    k = seg["cb_length"]
    f = seg["nof_filler_bits"]
    if c > 1:
        parts = b.reshape(c, -1)
        cbs = attach_crc(2, parts)
    else:
        cbs = b.reshape(1, -1)
    msgs = np.concatenate([cbs, np.zeros((c, f), np.uint8)], axis=1)
    assert msgs.shape[1] == k
    cws = ldpc_encode(bg, z, msgs)
    out = []
    for i in range(c):
        e = seg["e_short"] if i < seg["nof_short_cbs"] else seg["e_long"]
        out.append(rate_match(bg, z, cws[i], e, rv=rv, qm=qm, nref=nref, nof_filler_bits=f))
    g = np.concatenate(out)
    assert g.size == nof_ch_symbols * qm
    return g


def _level(bits, m):
    """Per-dimension Gray level of TS 38.211 Section 5.1 from bits[..., m] (MSB first)."""
    t = np.ones(bits.shape[:-1], np.int32)
    for k in range(m - 1, 0, -1):
        t = (1 << (m - k)) - (1 - 2 * bits[..., k].astype(np.int32)) * t
    return (1 - 2 * bits[..., 0].astype(np.int32)) * t


def modulate(bits, qm):
    """Bits [N*qm] -> complex64 symbols [N] (TS 38.211 Section 5.1, unit average energy)."""
    b = np.asarray(bits, np.uint8).reshape(-1, qm)
    if qm == 1:
        return ((1 - 2.0 * b[:, 0]) * (1 + 1j) / np.sqrt(2)).astype(np.complex64)
    m = qm // 2
    energy = {1: 2.0, 2: 10.0, 3: 42.0, 4: 170.0}[m]
    i = _level(b[:, 0::2], m)
    q = _level(b[:, 1::2], m)
    return ((i + 1j * q) / np.sqrt(energy)).astype(np.complex64)

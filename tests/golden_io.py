"""Readers for the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def ldpc_cases():
    d = load("ldpc_decode.npz")
    out = []
    for i, m in enumerate(d["meta"]):
        bg, z, f, poly, it, n = (int(x) for x in m)
        llr = d["llrs"][d["llr_offsets"][i]:d["llr_offsets"][i + 1]]
        bits = d["bits"][d["bit_offsets"][i]:d["bit_offsets"][i + 1]]
        out.append(dict(bg=bg, z=z, filler=f, poly=poly, max_iter=it, llrs=llr, bits=bits,
                        iterations=int(d["iterations"][i])))
    return out


def rm_cases():
    d = load("rate_dematch.npz")
    out = []
    for i, m in enumerate(d["meta"]):
        bg, z, rv, qm, nref, f, nd, e = (int(x) for x in m)
        out.append(dict(bg=bg, z=z, rv=rv, qm=qm, nref=nref, filler=f, new_data=nd,
                        llrs=d["ins"][d["in_offsets"][i]:d["in_offsets"][i + 1]],
                        prev=d["prevs"][d["buf_offsets"][i]:d["buf_offsets"][i + 1]],
                        out=d["outs"][d["buf_offsets"][i]:d["buf_offsets"][i + 1]]))
    return out


def crc_cases():
    d = load("crc.npz")
    return [dict(poly=int(m[0]), bits=d["bits"][d["offsets"][i]:d["offsets"][i + 1]], crc=int(d["crcs"][i]))
            for i, m in enumerate(d["meta"])]


def enc_cases():
    d = load("ldpc_encode.npz")
    return [dict(bg=int(m[0]), z=int(m[1]), msg=d["msgs"][d["msg_offsets"][i]:d["msg_offsets"][i + 1]],
                 cw=d["cws"][d["cw_offsets"][i]:d["cw_offsets"][i + 1]]) for i, m in enumerate(d["meta"])]


def kbits(bg, z):
    return (22 if bg == 1 else 10) * z


def demap_cases():
    d = load("demap.npz")
    out, off = [], 0
    for qm, n in d["meta"]:
        qm, n = int(qm), int(n)
        out.append(dict(qm=qm, symbols=d["symbols"][off:off + n], noise=d["noise"][off:off + n],
                        llrs=d["llrs"][off * 0:0]))
        off += n
    loff = 0
    for c in out:
        n = c["symbols"].size
        c["llrs"] = d["llrs"][loff:loff + n * c["qm"]]
        loff += n * c["qm"]
    return out


def eq_cases():
    d = load("equalize.npz")
    out, i = [], 0
    while f"c{i}_meta" in d:
        alg, p, l, nre = (int(x) for x in d[f"c{i}_meta"])
        out.append(dict(alg=alg, ports=p, layers=l, nre=nre, y=d[f"c{i}_y"], h=d[f"c{i}_h"], nv=d[f"c{i}_nv"],
                        tx=float(d[f"c{i}_tx"][0]), eq=d[f"c{i}_eq"], var=d[f"c{i}_var"]))
        i += 1
    return out


def est_cases(names=("estimate.npz", "estimate_273prb.npz")):
    out = []
    for name in names:
        out += _est_file(load(name))
    return out


def _est_file(d):
    out, i = [], 0
    while f"c{i}_meta" in d:
        rb0, nrb, nl, ports, slot, n_id, rnti, mask = (int(x) for x in d[f"c{i}_meta"])
        dm = [s for s in range(14) if (mask >> s) & 1]
        out.append(dict(rb_start=rb0, nof_rb=nrb, nof_layers=nl, ports=ports, slot=slot, n_id=n_id, rnti=rnti,
                        dmrs=dm, grid=d[f"c{i}_grid"],
                        freq=[d[f"c{i}_p{p}_freq"] for p in range(ports)],
                        sym=[d[f"c{i}_p{p}_sym"] for p in range(ports)],
                        scalars=[d[f"c{i}_p{p}_scalars"] for p in range(ports)]))
        i += 1
    return out

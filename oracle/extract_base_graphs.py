"""Writes the LDPC base-graph table (TS 38.212 Tables 5.3.2-2 and 5.3.2-3) in this project's
compact layout, reading the values out of the reference's compiled graph objects
(lib/phy/upper/channel_coding/ldpc/ldpc_graph_impl.h:84, get_lifted_node) through
oracle/_ref/libocudu_ref.so.

The table is standard data: every 5G NR LDPC implementation must hold exactly these shift
coefficients. The layout written here is this project's own: per base graph, the check-row
degrees, the variable-node column of each edge in the reference decoder's edge order
(lib/phy/upper/channel_coding/ldpc/ldpc_luts_impl.cpp BG*_adjacency_matrix, rows listed in
increasing column order) and the shift coefficient V of each edge for each of the eight
lifting-size sets (the lifted shift is V mod Z).

Usage (run once in a container that holds the reference; the output is committed):
    python oracle/extract_base_graphs.py > ocudu-dapp-platform_b200/csrc/ldpc_base_graphs.inc
"""
import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# Largest lifting size of each set a in {2, 3, 5, 7, 9, 11, 13, 15} (TS 38.212 Table 5.3.2-1).
SET_ZMAX = [256, 384, 320, 224, 288, 352, 208, 240]
SET_A = [2, 3, 5, 7, 9, 11, 13, 15]
ALL_Z = sorted({a * (1 << j) for a in SET_A for j in range(8) if a * (1 << j) <= 384})


def set_index(z):
    for i, a in enumerate(SET_A):
        t = z
        while t % 2 == 0 and t > a:
            t //= 2
        if t == a:
            return i
    raise ValueError(z)


def main():
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libocudu_ref.so"))
    out = sys.stdout
    out.write("// Generated by oracle/extract_base_graphs.py - do not edit.\n")
    out.write("// TS 38.212 Table 5.3.2-2 (BG1) and 5.3.2-3 (BG2) shift coefficients in this\n")
    out.write("// project's layout: per check row, its edges in increasing column order; per edge the\n")
    out.write("// column and the coefficient V for lifting-size sets 0..7 (shift = V mod Z).\n")
    assert len(ALL_Z) == 51
    for bg, nrows in ((1, 46), (2, 42)):
        degs, cols, vals = [], [], []
        buf = (ctypes.c_int * 32)()
        for r in range(nrows):
            n = lib.ref_ldpc_graph_row(bg, r, buf)
            degs.append(n)
            for e in range(n):
                c = buf[e]
                v = [lib.ref_ldpc_graph_shift(bg, SET_ZMAX[s], r, c) for s in range(8)]
                assert min(v) >= 0
                cols.append(c)
                vals.append(v)
                # Every lifting size must reproduce the reference's lifted shift.
                for z in ALL_Z:
                    assert lib.ref_ldpc_graph_shift(bg, z, r, c) == v[set_index(z)] % z, (bg, z, r, c)
            # No other column of the row has an edge.
            ncols = 68 if bg == 1 else 52
            for c in range(ncols):
                if c not in [buf[e] for e in range(n)]:
                    assert lib.ref_ldpc_graph_shift(bg, 384, r, c) == -1
        out.write(f"#define PG_BG{bg}_ROWS {nrows}\n#define PG_BG{bg}_EDGES {len(cols)}\n")
        out.write(f"static const unsigned char PG_BG{bg}_ROW_DEG[{nrows}] = {{{', '.join(map(str, degs))}}};\n")
        out.write(f"static const unsigned char PG_BG{bg}_EDGE_COL[{len(cols)}] = {{\n")
        for i in range(0, len(cols), 20):
            out.write("    " + ", ".join(map(str, cols[i:i + 20])) + ",\n")
        out.write("};\n")
        out.write(f"static const unsigned short PG_BG{bg}_EDGE_V[{len(cols)}][8] = {{\n")
        for v in vals:
            out.write("    {" + ", ".join(map(str, v)) + "},\n")
        out.write("};\n")


if __name__ == "__main__":
    main()

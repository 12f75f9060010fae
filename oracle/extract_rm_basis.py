"""Writes the Reed-Muller (32, 11) basis of the UCI short block code (TS 38.212 Table 5.3.3.3-1)
in this project's layout, reading it out of the reference's compiled encoder
(lib/phy/upper/channel_coding/short/short_block_encoder_impl.cpp) through oracle/_ref/libocudu_ref.so:
encoding the 11-bit unit message e_n into 32 bits gives basis sequence n.

The table is standard data: every 5G NR UCI implementation must hold exactly these sequences.
The layout written here is this project's own: one 16-bit word per codeword position i, bit n =
M(i, n).

Usage (run once in a container that holds the reference; the output is committed):
    python oracle/extract_rm_basis.py > ocudu-dapp-platform_b200/csrc/uci_rm_basis.inc
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libocudu_ref.so"))
    words = [0] * 32
    for n in range(11):
        msg = np.zeros(11, np.uint8)
        msg[n] = 1
        out = np.zeros(32, np.uint8)
        lib.ref_short_block_encode(11, msg.ctypes.data_as(ctypes.c_void_p), 32, 2, out.ctypes.data_as(ctypes.c_void_p))
        for i in range(32):
            words[i] |= int(out[i] & 1) << n
    print("// Reed-Muller (32, 11) basis of the UCI short block code (TS 38.212 Table 5.3.3.3-1): word i holds")
    print("// bit n = M(i, n). Generated by oracle/extract_rm_basis.py from the reference's encoder.")
    print("static const unsigned short PG_UCI_RM_BASIS[32] = {")
    for k in range(0, 32, 8):
        print("    " + ", ".join("0x%03x" % w for w in words[k:k + 8]) + ",")
    print("};")


if __name__ == "__main__":
    main()

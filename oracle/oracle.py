"""Test infrastructure only: ctypes bindings to the two CPU checkers.

* ``Ref``  - the reference's own CPU code compiled by oracle/Makefile into
  oracle/_ref/libocudu_ref.so (the AVX-512 variant when the host has it, else AVX2; they
  decode bit-identically).
* ``Port`` - the plain-C restatement oracle/pusch_oracle.c (oracle/_build/libpusch_oracle.so).

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libocudu_ref.so")
PORT_SO = os.path.join(HERE, "_build", "libpusch_oracle.so")

CRC16, CRC24A, CRC24B, CRC24C, CRC11, CRC6 = range(6)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def kb(bg):
    return 22 if bg == 1 else 10


def n_short(bg):
    return 66 if bg == 1 else 50


class Ref:
    """The reference's compiled CPU implementation."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle ref`)")
        lib = ctypes.CDLL(path)
        lib.ref_ldpc_decode.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_int,
                                                                                  ctypes.c_void_p]
        lib.ref_ldpc_decode.restype = ctypes.c_int
        lib.ref_ldpc_auto_variant.restype = ctypes.c_char_p
        lib.ref_crc_calculate.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.ref_crc_calculate.restype = ctypes.c_uint
        lib.ref_crc_calculate_byte.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.ref_crc_calculate_byte.restype = ctypes.c_uint
        lib.ref_ldpc_encode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_ldpc_encode_rm.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_rate_dematch.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.ref_demodulate_soft.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p]
        lib.ref_sch_segmentation.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        lib.ref_ldpc_decode_batch_mt.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ref_ldpc_decode_batch_mt.restype = ctypes.c_double
        lib.ref_port_estimate.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 9 + [ctypes.c_uint32, ctypes.c_float,
                                                                                 ctypes.c_void_p, ctypes.c_void_p,
                                                                                 ctypes.c_void_p]
        lib.ref_equalize.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p] * 3 + [ctypes.c_float, ctypes.c_void_p,
                                                                                   ctypes.c_void_p]
        self.lib = lib
        self.variant = lib.ref_ldpc_auto_variant().decode()

    def ldpc_decode(self, bg, Z, llrs, filler=0, crc_poly=CRC24B, max_iter=10, nof_crc_bits=24, variant=None,
                    prefill=0xFF):
        """Returns (iterations or 0, packed K*Z bits)."""
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        K = kb(bg) * Z
        out = np.full((K + 7) // 8, prefill, np.uint8)
        v = (variant or self.variant).encode()
        it = self.lib.ref_ldpc_decode(v, bg, Z, filler, nof_crc_bits, crc_poly, max_iter, _ptr(llrs), llrs.size,
                                      _ptr(out))
        if it < 0:
            raise RuntimeError(f"decoder variant {v!r} unavailable on this CPU")
        return it, out

    def crc(self, poly, bits):
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        packed = np.packbits(bits) if bits.size else np.zeros(1, np.uint8)
        return self.lib.ref_crc_calculate(poly, _ptr(packed), bits.size)

    def ldpc_decode_batch_mt(self, meta, llr_offsets, llrs, threads, variant=None):
        """Multi-threaded batch decode in C++ (no interpreter in the loop). meta: int32 [n, 6]
        {bg, Z, filler, crc_poly, max_iterations, nof_llrs}. Returns (iterations, wall seconds)."""
        meta = np.ascontiguousarray(meta, dtype=np.int32)
        offs = np.ascontiguousarray(llr_offsets, dtype=np.int64)
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        it = np.zeros(meta.shape[0], np.int32)
        v = (variant or self.variant).encode()
        dt = self.lib.ref_ldpc_decode_batch_mt(v, meta.shape[0], _ptr(meta), _ptr(offs), _ptr(llrs), _ptr(it),
                                               threads)
        return it, dt

    def ldpc_encode(self, bg, Z, msg_bits):
        msg = np.packbits(np.ascontiguousarray(msg_bits, dtype=np.uint8))
        cw = np.zeros(n_short(bg) * Z, np.uint8)
        self.lib.ref_ldpc_encode(bg, Z, _ptr(msg), _ptr(cw))
        return cw

    def ldpc_encode_rm(self, bg, Z, msg_bits, E, rv=0, qm=1, Nref=0, filler=0):
        msg = np.packbits(np.ascontiguousarray(msg_bits, dtype=np.uint8))
        out = np.zeros(E, np.uint8)
        self.lib.ref_ldpc_encode_rm(bg, Z, rv, qm, Nref, filler, E, _ptr(msg), _ptr(out))
        return out

    def rate_dematch(self, bg, Z, llrs, rv=0, qm=1, Nref=0, filler=0, new_data=True, out=None):
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        if out is None:
            out = np.zeros(n_short(bg) * Z, np.int8)
        self.lib.ref_rate_dematch(bg, Z, rv, qm, Nref, filler, int(bool(new_data)), _ptr(llrs), llrs.size, _ptr(out))
        return out

    def demodulate_soft(self, qm, symbols, noise_vars):
        sym = np.ascontiguousarray(symbols, dtype=np.complex64)
        nv = np.ascontiguousarray(noise_vars, dtype=np.float32)
        out = np.zeros(sym.size * qm, np.int8)
        self.lib.ref_demodulate_soft(qm, _ptr(sym), _ptr(nv), sym.size, _ptr(out))
        return out

    def equalize(self, algorithm, ch_symbols, ch_estimates, noise_var_per_port, tx_scaling=1.0):
        """ch_symbols uint32 cbf16 [port][re], ch_estimates uint32 cbf16 [port][layer][re]."""
        y = np.ascontiguousarray(ch_symbols, np.uint32)
        h = np.ascontiguousarray(ch_estimates, np.uint32)
        nports, nre = y.shape
        nl = h.shape[1]
        nv = np.ascontiguousarray(noise_var_per_port, np.float32)
        eq = np.zeros((nre, nl), np.complex64)
        var = np.zeros((nre, nl), np.float32)
        self.lib.ref_equalize(algorithm, nre, nports, nl, _ptr(y), _ptr(h), _ptr(nv), ctypes.c_float(tx_scaling),
                              _ptr(eq), _ptr(var))
        return eq, var

    def port_estimate(self, grid, port, slot, n_id, rb_start, nof_rb, nof_layers, dmrs_symbols, scaling, n_scid=0):
        """The reference's port estimator (FD filter, TD interpolate). grid: uint32 cbf16
        [nports][14][nsubc]. Returns (freq complex64 [nd][nl][12 nof_rb] (FP32 internal),
        symbol estimates uint32 cbf16 [14][nl][12 nof_rb], dict of scalars)."""
        g = np.ascontiguousarray(grid, np.uint32)
        nports, _, nsubc = g.shape
        nd = len(dmrs_symbols)
        freq = np.zeros((nd, nof_layers, 12 * nof_rb), np.complex64)
        sym = np.zeros((14, nof_layers, 12 * nof_rb), np.uint32)
        sc = np.zeros(3 + nof_layers, np.float32)
        mask = sum(1 << s for s in dmrs_symbols)
        self.lib.ref_port_estimate(_ptr(g), nports, nsubc, port, slot, n_id, n_scid, rb_start, nof_rb, nof_layers, mask,
                                   ctypes.c_float(scaling), _ptr(freq), _ptr(sym), _ptr(sc))
        return freq, sym, dict(noise_var=float(sc[0]), epre=float(sc[1]), snr=float(sc[2]),
                               rsrp=sc[3:].astype(np.float64))

    def port_estimate_full(self, grid, port, slot, n_id, rb_start, nof_rb, nof_layers, dmrs_symbols, scaling,
                           n_scid=0):
        """port_estimate plus the pilots the reference used (complex64 [nd][nl][6 nof_rb]) and its
        CFO (Hz, NaN when none) and time alignment (s) in the scalars dict."""
        g = np.ascontiguousarray(grid, np.uint32)
        nports, _, nsubc = g.shape
        nd = len(dmrs_symbols)
        freq = np.zeros((nd, nof_layers, 12 * nof_rb), np.complex64)
        sym = np.zeros((14, nof_layers, 12 * nof_rb), np.uint32)
        sc = np.zeros(3 + nof_layers, np.float32)
        pil = np.zeros((nd, nof_layers, 6 * nof_rb), np.complex64)
        ct = np.zeros(2, np.float64)
        mask = sum(1 << s for s in dmrs_symbols)
        f = self.lib.ref_port_estimate_full
        f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 9 + [ctypes.c_uint32, ctypes.c_float] + [ctypes.c_void_p] * 5
        f(_ptr(g), nports, nsubc, port, slot, n_id, n_scid, rb_start, nof_rb, nof_layers, mask, ctypes.c_float(scaling),
          _ptr(freq), _ptr(sym), _ptr(sc), _ptr(pil), _ptr(ct))
        return freq, sym, dict(noise_var=float(sc[0]), epre=float(sc[1]), snr=float(sc[2]),
                               rsrp=sc[3:].astype(np.float64), cfo_hz=float(ct[0]), ta_s=float(ct[1]), pilots=pil)

    def pusch_decode_mt(self, descs, grid, tb_bytes, threads):
        """The reference's CPU receive path over a pg_pusch_ue array (ctypes) and its grids.
        Returns (ok flags, mean iterations, TB bytes, wall seconds)."""
        n = len(descs)
        g = np.ascontiguousarray(grid, np.uint32)
        tb = np.zeros(max(tb_bytes, 1), np.uint8)
        ok = np.zeros(n, np.int32)
        it = np.zeros(n, np.float32)
        self.lib.ref_pusch_decode_mt.restype = ctypes.c_double
        self.lib.ref_pusch_decode_mt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        dt = self.lib.ref_pusch_decode_mt(ctypes.addressof(descs), n, _ptr(g), _ptr(tb), _ptr(ok), _ptr(it), threads)
        return ok.astype(bool), it, tb, float(dt)

    def pusch_decode_detail(self, descs, grid, tb_bytes, nof_llrs, threads):
        """pusch_decode_mt plus the stage taps (ref_pusch_decode_detail): returns a dict with ok
        (bool per UE), mean_iters, tb (bytes), nof_cbs (per UE), cb_iters (one list per UE: the
        ldpc_decoder result of every codeblock, 0 = not decoded) and llrs (the descrambled codeword
        LLRs of every UE at its llr_offset)."""
        n = len(descs)
        g = np.ascontiguousarray(grid, np.uint32)
        tb = np.zeros(max(tb_bytes, 1), np.uint8)
        ok = np.zeros(n, np.int32)
        it = np.zeros(n, np.float32)
        cb_first = (np.arange(n, dtype=np.int32) * 160).astype(np.int32)  # at most 152 codeblocks per TB
        cb_it = np.full(160 * n, -1, np.int32)
        ncb = np.zeros(n, np.int32)
        llrs = np.zeros(max(nof_llrs, 1), np.int8)
        f = self.lib.ref_pusch_decode_detail
        f.restype = ctypes.c_double
        f.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 8 + [ctypes.c_int]
        dt = f(ctypes.addressof(descs), n, _ptr(g), _ptr(tb), _ptr(ok), _ptr(it), _ptr(cb_first), _ptr(cb_it), _ptr(ncb),
               _ptr(llrs), threads)
        cbs = [cb_it[cb_first[i]:cb_first[i] + ncb[i]].copy() for i in range(n)]
        return dict(ok=ok.astype(bool), mean_iters=it, tb=tb, nof_cbs=ncb, cb_iters=cbs, llrs=llrs, seconds=float(dt))

    def pusch_mcs(self, table, index):
        r = ctypes.c_float()
        qm = self.lib.ref_pusch_mcs(0 if table == 1 else 1, index, ctypes.byref(r))
        return qm, float(r.value)

    def tbs(self, nof_symb_sh, nof_dmrs_prb, nof_oh_prb, qm, rate_x1024, nof_layers, n_prb):
        return int(self.lib.ref_tbs(nof_symb_sh, nof_dmrs_prb, nof_oh_prb, qm, ctypes.c_float(rate_x1024), nof_layers,
                                    n_prb))

    def base_graph(self, rate_x1024, tbs_bits):
        return int(self.lib.ref_base_graph(ctypes.c_float(rate_x1024 / 1024.0), tbs_bits))

    def sch_segmentation(self, tbs_bits, bg):
        o = np.zeros(4, np.int32)
        self.lib.ref_sch_segmentation(tbs_bits, bg, _ptr(o))
        return dict(C=int(o[0]), Z=int(o[1]), K=int(o[2]), tb_crc=int(o[3]))

    def ulsch_demultiplex(self, cfg, llrs, block_size=4096):
        """The reference's ulsch_demultiplex on descrambled soft bits (ref_shim_uci.cpp). cfg: a dict
        with the fields of pg_ulsch_demux_config. Returns (sch, harq_ack, csi_part1, complete)."""
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        G = llrs.size
        sch, ack, csi = np.zeros(G, np.int8), np.zeros(G, np.int8), np.zeros(G, np.int8)
        lens = np.zeros(4, np.int32)
        f = self.lib.ref_ulsch_demultiplex
        f.argtypes = [ctypes.c_int] * 13 + [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        f(cfg["modulation_order"], cfg["nof_layers"], cfg["nof_prb"], cfg["start_symbol_index"], cfg["nof_symbols"],
          cfg["dmrs_symbol_mask"], cfg["dmrs_type"], cfg["nof_cdm_groups_without_data"], cfg["nof_harq_ack_rvd"],
          cfg["nof_harq_ack_bits"], cfg["nof_enc_harq_ack_bits"], cfg["nof_csi_part1_bits"],
          cfg["nof_enc_csi_part1_bits"], cfg["c_init"], _ptr(llrs), G, block_size, _ptr(sch), G, _ptr(ack), G,
          _ptr(csi), G, _ptr(lens))
        return sch[:lens[0]].copy(), ack[:lens[1]].copy(), csi[:lens[2]].copy(), bool(lens[3])

    def ulsch_information(self, tbs_bits, rate_x1024, qm, nof_layers, harq_ack, csi1, csi2, alpha, beta_ack,
                          beta_csi1, beta_csi2, nof_rb, start, nof_symbols, dmrs_mask, nof_cdm, contains_dc=False):
        """The reference's get_ulsch_information (lib/ran/pusch/ulsch_info.cpp) for DM-RS type 1:
        (UL-SCH, HARQ-ACK, reserved HARQ-ACK, CSI-1, CSI-2 soft bits, HARQ-ACK, CSI-1, CSI-2 REs, DC
        overlap bits)."""
        out = np.zeros(9, np.uint32)
        f = self.lib.ref_ulsch_information
        f.argtypes = [ctypes.c_uint, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint,
                      ctypes.c_uint, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint,
                      ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, ctypes.c_void_p]
        f(tbs_bits, rate_x1024, qm, nof_layers, harq_ack, csi1, csi2, alpha, beta_ack, beta_csi1, beta_csi2, nof_rb,
          start, nof_symbols, dmrs_mask, nof_cdm, int(contains_dc), _ptr(out))
        return tuple(int(x) for x in out)

    def short_block_encode(self, msg, E, qm):
        msg = np.ascontiguousarray(msg, dtype=np.uint8)
        out = np.zeros(E, np.uint8)
        self.lib.ref_short_block_encode.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_void_p]
        self.lib.ref_short_block_encode(msg.size, _ptr(msg), E, qm, _ptr(out))
        return out

    def short_block_detect(self, K, llrs, qm):
        """The reference's short_block_detector::detect: (bits, valid)."""
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        out = np.zeros(K, np.uint8)
        self.lib.ref_short_block_detect.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_void_p]
        ok = self.lib.ref_short_block_detect(K, _ptr(llrs), llrs.size, qm, _ptr(out))
        return out, bool(ok)

    def polar_code(self, K, E):
        """The reference's polar_code_impl::set (uplink): dict as pusch_b200.uci.polar_code, or None."""
        N = 1024
        info = np.zeros(4, np.int32)
        kset = np.zeros(N, np.uint8)
        pc = np.zeros(4, np.uint16)
        sub = np.zeros(N, np.uint16)
        f = self.lib.ref_polar_code
        f.argtypes = [ctypes.c_uint, ctypes.c_uint] + [ctypes.c_void_p] * 4
        if not f(K, E, _ptr(info), _ptr(kset), _ptr(pc), _ptr(sub)):
            return None
        n_ = int(info[1])
        return dict(n=int(info[0]), N=n_, nPC=int(info[2]), k_set=kset[:n_].copy(), pc_set=[int(x) for x in pc],
                    subblock=sub[:n_].copy())

    def uci_polar_encode(self, msg, E):
        """Polar-coded UCI test vector: A message bits -> E bits (segmentation, CRC, polar encoding,
        rate matching with the channel interleaver, all by the reference's pieces)."""
        msg = np.ascontiguousarray(msg, dtype=np.uint8)
        out = np.zeros(E, np.uint8)
        f = self.lib.ref_uci_polar_encode
        f.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
        f(msg.size, _ptr(msg), E, _ptr(out))
        return out

    def uci_polar_decode(self, A, llrs):
        """The reference's uci_decoder::decode of an A-bit polar-coded message: (bits, valid)."""
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        out = np.zeros(A, np.uint8)
        f = self.lib.ref_uci_polar_decode
        f.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
        ok = f(A, _ptr(llrs), llrs.size, _ptr(out))
        return out, bool(ok)

    def bfp_compress(self, width, iq_words, generic=False):
        """The reference's BFP compressor on complex bf16 words (12 per PRB): compressed bytes."""
        iq_words = np.ascontiguousarray(iq_words, dtype=np.uint32)
        nprb = iq_words.size // 12
        out = np.zeros(nprb * (1 + 3 * width), np.uint8)
        self.lib.ref_bfp_compress.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int]
        self.lib.ref_bfp_compress(width, _ptr(iq_words), nprb, _ptr(out), int(generic))
        return out

    def bfp_decompress(self, width, data, nprb, generic=False):
        """The reference's BFP decompressor: complex bf16 words (12 per PRB)."""
        data = np.ascontiguousarray(data, dtype=np.uint8)
        out = np.zeros(12 * nprb, np.uint32)
        self.lib.ref_bfp_decompress.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_int]
        rc = self.lib.ref_bfp_decompress(width, _ptr(data), nprb, _ptr(out), int(generic))
        return out, int(rc)

    def uci_min_encoded_bits(self, K):
        return int(self.lib.ref_uci_min_encoded_bits(K))


class Port:
    """The plain-C restatement (oracle/pusch_oracle.c)."""

    def __init__(self, path=PORT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle oracle`)")
        lib = ctypes.CDLL(path)
        lib.pgo_crc.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.pgo_crc.restype = ctypes.c_uint32
        lib.pgo_ldpc_decode.argtypes = [ctypes.c_int] * 5 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.pgo_ldpc_decode.restype = ctypes.c_int
        lib.pgo_rate_dematch.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.pgo_ldpc_edge_shift.argtypes = [ctypes.c_int] * 3
        lib.pgo_demodulate_soft.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p]
        self.lib = lib

    def demodulate_soft(self, qm, symbols, noise_vars):
        sym = np.ascontiguousarray(symbols, dtype=np.complex64)
        nv = np.ascontiguousarray(noise_vars, dtype=np.float32)
        out = np.zeros(sym.size * qm, np.int8)
        self.lib.pgo_demodulate_soft(qm, _ptr(sym), _ptr(nv), sym.size, _ptr(out))
        return out

    def crc(self, poly, bits):
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        packed = np.packbits(bits) if bits.size else np.zeros(1, np.uint8)
        return self.lib.pgo_crc(poly, _ptr(packed), bits.size)

    def ldpc_decode(self, bg, Z, llrs, filler=0, crc_poly=CRC24B, max_iter=10):
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        K = kb(bg) * Z
        out = np.zeros((K + 7) // 8, np.uint8)
        it = self.lib.pgo_ldpc_decode(bg, Z, filler, crc_poly, max_iter, _ptr(llrs), llrs.size, _ptr(out))
        return it, out

    def rate_dematch(self, bg, Z, llrs, rv=0, qm=1, Nref=0, filler=0, new_data=True, out=None):
        llrs = np.ascontiguousarray(llrs, dtype=np.int8)
        if out is None:
            out = np.zeros(n_short(bg) * Z, np.int8)
        self.lib.pgo_rate_dematch(bg, Z, rv, qm, Nref, filler, int(bool(new_data)), _ptr(llrs), llrs.size, _ptr(out))
        return out

"""ctypes binding of the pusch_b200 C ABI (include/pusch_b200.h).

The library is built in-tree (ocudu-dapp-platform_b200/csrc/Makefile) into
pusch_b200/_lib/libpusch_b200.so. There is no CPU fallback: if the library is missing or no
sm_100 device is present, creating a context raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpusch_b200.so")

PG_OK, PG_ERR_INVALID, PG_ERR_CUDA, PG_ERR_CAPACITY, PG_ERR_TIMEOUT, PG_ERR_NO_DEVICE = range(6)
PG_CRC16, PG_CRC24A, PG_CRC24B = 0, 1, 2
PG_CRC_NONE = 255
# pg_ldpc_kernel: one lifted lane per thread, two lanes per thread (f16x2), two lanes per thread pair.
(PG_LDPC_KERNEL_ONE_LANE, PG_LDPC_KERNEL_TWO_LANES, PG_LDPC_KERNEL_SPLIT, PG_LDPC_KERNEL_Z384,
 PG_LDPC_KERNEL_Z384_SPLIT) = 0, 1, 2, 3, 4
PG_LDPC_ORDER_GIVEN, PG_LDPC_ORDER_LONGEST_FIRST = 0, 1

STATUS_NAMES = {0: "PG_OK", 1: "PG_ERR_INVALID", 2: "PG_ERR_CUDA", 3: "PG_ERR_CAPACITY", 4: "PG_ERR_TIMEOUT",
                5: "PG_ERR_NO_DEVICE"}


class PgConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_codeblocks", ctypes.c_int), ("max_llrs", ctypes.c_int)]


class PgLdpcCb(ctypes.Structure):
    _fields_ = [
        ("llr_offset", ctypes.c_uint32),
        ("nof_llrs", ctypes.c_uint32),
        ("out_offset", ctypes.c_uint32),
        ("lifting_size", ctypes.c_uint16),
        ("nof_filler_bits", ctypes.c_uint16),
        ("base_graph", ctypes.c_uint8),
        ("crc_poly", ctypes.c_uint8),
        ("max_iterations", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8),
    ]


assert ctypes.sizeof(PgLdpcCb) == 20


class PgRmCb(ctypes.Structure):
    _fields_ = [("in_offset", ctypes.c_uint32), ("rm_length", ctypes.c_uint32), ("out_offset", ctypes.c_uint32),
                ("nref", ctypes.c_uint32), ("lifting_size", ctypes.c_uint16), ("nof_filler_bits", ctypes.c_uint16),
                ("base_graph", ctypes.c_uint8), ("rv", ctypes.c_uint8), ("modulation_order", ctypes.c_uint8),
                ("new_data", ctypes.c_uint8)]


class PgCrcItem(ctypes.Structure):
    _fields_ = [("bit_offset", ctypes.c_uint32), ("nof_bits", ctypes.c_uint32), ("poly", ctypes.c_uint32)]


class PgTbDesc(ctypes.Structure):
    _fields_ = [("cb_first", ctypes.c_uint32), ("nof_cbs", ctypes.c_uint32), ("cb_payload_bits", ctypes.c_uint32),
                ("tbs_bits", ctypes.c_uint32), ("tb_out_offset", ctypes.c_uint32), ("crc_poly", ctypes.c_uint32)]


class PgSchSegmentation(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("nof_cbs", "lifting_size", "cb_length", "nof_filler_bits",
                                                "cb_crc_bits", "tb_crc_bits", "nof_short_cbs", "e_short", "e_long")]


class PgSchTb(ctypes.Structure):
    _fields_ = [("llr_offset", ctypes.c_uint32), ("nof_ch_symbols", ctypes.c_uint32), ("tbs_bits", ctypes.c_uint32),
                ("tb_out_offset", ctypes.c_uint32), ("nref", ctypes.c_uint32), ("base_graph", ctypes.c_uint8),
                ("modulation_order", ctypes.c_uint8), ("nof_layers", ctypes.c_uint8), ("rv", ctypes.c_uint8),
                ("max_iterations", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 3)]


class PgSchResult(ctypes.Structure):
    _fields_ = [("tb_crc_ok", ctypes.c_uint32), ("nof_cbs", ctypes.c_uint32), ("nof_cbs_crc_ok", ctypes.c_uint32),
                ("mean_iterations", ctypes.c_float), ("max_iterations_run", ctypes.c_uint32)]


class PgLeAdam(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("weight_decay", ctypes.c_float)]


class PgPuschPlanTuning(ctypes.Structure):
    _fields_ = [("rm_ctas_per_cb", ctypes.c_int), ("demod_res_per_thread", ctypes.c_int),
                ("demod_block", ctypes.c_int), ("ldpc_ctas_per_sm", ctypes.c_int), ("ldpc_kernel", ctypes.c_int),
                ("ldpc_order", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PgUlschInfoConfig(ctypes.Structure):
    _fields_ = [("tbs_bits", ctypes.c_uint32), ("target_code_rate", ctypes.c_float), ("alpha_scaling", ctypes.c_float),
                ("beta_offset_harq_ack", ctypes.c_float), ("beta_offset_csi_part1", ctypes.c_float),
                ("beta_offset_csi_part2", ctypes.c_float), ("nof_harq_ack_bits", ctypes.c_uint16),
                ("nof_csi_part1_bits", ctypes.c_uint16), ("nof_csi_part2_bits", ctypes.c_uint16),
                ("nof_rb", ctypes.c_uint16), ("dmrs_symbol_mask", ctypes.c_uint16), ("base_graph", ctypes.c_uint8),
                ("modulation_order", ctypes.c_uint8), ("nof_layers", ctypes.c_uint8), ("start_symbol", ctypes.c_uint8),
                ("nof_symbols", ctypes.c_uint8), ("nof_cdm_groups_without_data", ctypes.c_uint8),
                ("contains_dc", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 3)]


class PgUlschInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("nof_ul_sch_bits", "nof_harq_ack_bits", "nof_harq_ack_rvd",
                                               "nof_csi_part1_bits", "nof_csi_part2_bits", "nof_harq_ack_re",
                                               "nof_csi_part1_re", "nof_csi_part2_re", "nof_dc_overlap_bits")]


class PgUlschDemuxConfig(ctypes.Structure):
    _fields_ = [("llr_offset", ctypes.c_uint32), ("nof_llrs", ctypes.c_uint32), ("sch_offset", ctypes.c_uint32),
                ("harq_ack_offset", ctypes.c_uint32), ("csi_part1_offset", ctypes.c_uint32),
                ("c_init", ctypes.c_uint32), ("nof_harq_ack_rvd", ctypes.c_uint32),
                ("nof_enc_harq_ack_bits", ctypes.c_uint32), ("nof_enc_csi_part1_bits", ctypes.c_uint32),
                ("nof_prb", ctypes.c_uint16), ("dmrs_symbol_mask", ctypes.c_uint16),
                ("modulation_order", ctypes.c_uint8), ("nof_layers", ctypes.c_uint8),
                ("start_symbol_index", ctypes.c_uint8), ("nof_symbols", ctypes.c_uint8), ("dmrs_type", ctypes.c_uint8),
                ("nof_cdm_groups_without_data", ctypes.c_uint8), ("nof_harq_ack_bits", ctypes.c_uint16),
                ("nof_csi_part1_bits", ctypes.c_uint16)]


class PgPuschUci(ctypes.Structure):
    _fields_ = [("nof_harq_ack_rvd", ctypes.c_uint32), ("nof_enc_harq_ack_bits", ctypes.c_uint32),
                ("nof_enc_csi_part1_bits", ctypes.c_uint32), ("nof_harq_ack_bits", ctypes.c_uint16),
                ("nof_csi_part1_bits", ctypes.c_uint16), ("nof_cdm_groups_without_data", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8 * 3)]


class PgPuschUciResult(ctypes.Structure):
    _fields_ = [("harq_ack", ctypes.c_uint8 * 11), ("csi_part1", ctypes.c_uint8 * 11), ("harq_ack_valid", ctypes.c_uint8),
                ("csi_part1_valid", ctypes.c_uint8)]


class PgUciShortBlock(ctypes.Structure):
    _fields_ = [("llr_offset", ctypes.c_uint32), ("nof_llrs", ctypes.c_uint32), ("out_offset", ctypes.c_uint32),
                ("nof_bits", ctypes.c_uint8), ("modulation_order", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 2)]


class PgUciPolar(ctypes.Structure):
    _fields_ = [("llr_offset", ctypes.c_uint32), ("nof_llrs", ctypes.c_uint32), ("out_offset", ctypes.c_uint32),
                ("nof_bits", ctypes.c_uint16), ("reserved", ctypes.c_uint16)]


class PgPolarCodeInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint16), ("N", ctypes.c_uint16), ("K", ctypes.c_uint16), ("E", ctypes.c_uint16),
                ("nPC", ctypes.c_uint8), ("nWmPC", ctypes.c_uint8), ("pc_set", ctypes.c_uint16 * 4),
                ("k_set", ctypes.c_uint32 * 32), ("subblock", ctypes.c_uint16 * 1024)]


class PgPortEstimateCfg(ctypes.Structure):
    _fields_ = [("grid_nof_subc", ctypes.c_uint32), ("scaling", ctypes.c_float), ("rb_start", ctypes.c_uint16),
                ("nof_rb", ctypes.c_uint16), ("dmrs_symbol_mask", ctypes.c_uint16), ("first_symbol", ctypes.c_uint8),
                ("nof_symbols", ctypes.c_uint8), ("nof_layers", ctypes.c_uint8), ("scs_khz", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8 * 2)]


class PgPortEstimateResult(ctypes.Structure):
    _fields_ = [("noise_var", ctypes.c_float), ("epre", ctypes.c_float), ("snr", ctypes.c_float),
                ("rsrp", ctypes.c_float * 2), ("cfo_hz", ctypes.c_float), ("time_alignment_s", ctypes.c_double)]


assert ctypes.sizeof(PgPortEstimateCfg) == 20 and ctypes.sizeof(PgPortEstimateResult) == 32


class PgPuschPlanInfo(ctypes.Structure):
    _fields_ = [("nof_ues", ctypes.c_uint32), ("nof_codeblocks", ctypes.c_uint32), ("tb_bytes", ctypes.c_uint64),
                ("nof_llrs", ctypes.c_uint64), ("grid_words", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
                ("nof_kernels", ctypes.c_uint32), ("h2d_grid_bytes", ctypes.c_uint32)]


assert ctypes.sizeof(PgRmCb) == 24 and ctypes.sizeof(PgSchTb) == 28 and ctypes.sizeof(PgTbDesc) == 24

# Every symbol the public header declares, with (restype, argtypes).
_VP = ctypes.c_void_p
SIGNATURES = {
    "pg_abi_version": (ctypes.c_int, []),
    "pg_create": (ctypes.c_int, [ctypes.POINTER(PgConfig), ctypes.POINTER(_VP)]),
    "pg_destroy": (None, [_VP]),
    "pg_last_error": (ctypes.c_char_p, [_VP]),
    "pg_ldpc_decode_batch_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_ldpc_decode_batch_resident": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_ldpc_decode_batch_static_scratch": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_ldpc_decode_batch_host": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP,
                                                 ctypes.c_size_t, _VP]),
    "pg_ldpc_output_bytes": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "pg_set_kernel_timing": (ctypes.c_int, [_VP, ctypes.c_int]),
    "pg_rate_dematch_batch_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP]),
    "pg_rate_dematch_batch_host": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP, ctypes.c_size_t]),
    "pg_crc_calculate_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP]),
    "pg_crc_calculate_host": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP]),
    "pg_tb_assemble_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP]),
    "pg_sch_segment": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                                      ctypes.POINTER(PgSchSegmentation)]),
    "pg_sch_decode_batch_host": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP, ctypes.c_size_t,
                                                _VP]),
    "pg_last_kernel_ms": (ctypes.c_float, [_VP]),
    "pg_equalize_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP,
                                          ctypes.c_float, _VP, _VP, _VP]),
    "pg_equalize_host": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP,
                                        ctypes.c_float, _VP, _VP]),
    "pg_demodulate_soft_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_demodulate_soft_host": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    "pg_ulsch_information": (ctypes.c_int, [_VP, _VP]),
    "pg_descramble_device": (ctypes.c_int, [_VP, ctypes.c_uint32, _VP, _VP, ctypes.c_size_t, _VP]),
    "pg_descramble_host": (ctypes.c_int, [_VP, ctypes.c_uint32, _VP, _VP, ctypes.c_size_t]),
    "pg_pusch_est_size": (ctypes.c_size_t, [_VP]),
    "pg_pusch_estimate_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_pusch_symbol_estimates_device": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "pg_pusch_demodulate_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP]),
    "pg_pusch_process_host": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP, ctypes.c_size_t, _VP,
                                             _VP]),
    "pg_pusch_plan_create": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_size_t, _VP]),
    "pg_pusch_plan_create_uci": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_size_t, _VP]),
    "pg_pusch_plan_uci_results": (ctypes.c_int, [_VP, _VP]),
    "pg_pusch_plan_uci_message": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_size_t, _VP]),
    "pg_pusch_plan_destroy": (None, [_VP]),
    "pg_pusch_plan_info": (ctypes.c_int, [_VP, _VP]),
    "pg_pusch_plan_set_graph": (ctypes.c_int, [_VP, ctypes.c_int]),
    "pg_pusch_plan_execute_device": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "pg_pusch_plan_execute_host": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_size_t, _VP, _VP]),
    "pg_conv1d_forward_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP,
                                                ctypes.c_int, ctypes.c_int, _VP, _VP]),
    "pg_conv1d_backward_data_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP,
                                                      ctypes.c_int, _VP, _VP]),
    "pg_conv1d_backward_weights_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.c_int,
                                                         _VP, _VP, _VP, _VP]),
    "pg_last_learned_ms": (ctypes.c_float, [_VP]),
    "pg_le_nof_params": (ctypes.c_size_t, []),
    "pg_le_rows": (ctypes.c_size_t, [_VP, ctypes.c_int]),
    "pg_le_create": (ctypes.c_int, [_VP, ctypes.c_int, _VP]),
    "pg_le_destroy": (None, [_VP]),
    "pg_le_set_params": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t]),
    "pg_le_get_params": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t]),
    "pg_le_get_grads": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t]),
    "pg_le_status": (ctypes.c_int, [_VP]),
    "pg_le_forward_device": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, _VP, _VP]),
    "pg_le_backward_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP]),
    "pg_le_refine_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP]),
    "pg_le_train_step_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "pg_pusch_estimate_ls_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP]),
    "pg_pusch_plan_set_learned": (ctypes.c_int, [_VP, _VP, _VP]),
    "pg_pusch_plan_set_harq": (ctypes.c_int, [_VP, _VP, _VP]),
    "pg_ulsch_demultiplex_sizes": (ctypes.c_int, [_VP, _VP]),
    "pg_bfp_prb_bytes": (ctypes.c_int, [ctypes.c_int]),
    "pg_pusch_plan_submit_host": (ctypes.c_int, [_VP, _VP]),
    "pg_pusch_plan_collect_host": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t, _VP, _VP]),
    "pg_bfp_decompress_device": (ctypes.c_int, [_VP, _VP, ctypes.c_uint32, ctypes.c_int, _VP, _VP]),
    "pg_pusch_plan_execute_host_bfp": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t, ctypes.c_int, _VP, ctypes.c_size_t,
                                                      _VP, _VP]),
    "pg_ulsch_demultiplex_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP]),
    "pg_uci_short_block_detect_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_uci_polar_decode_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP, _VP, _VP]),
    "pg_polar_code": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, _VP]),
    "pg_pusch_plan_get_tuning": (ctypes.c_int, [_VP, _VP]),
    "pg_pusch_plan_set_tuning": (ctypes.c_int, [_VP, _VP]),
    "pg_pusch_plan_autotune": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP]),
    "pg_set_ldpc_ctas_per_sm": (ctypes.c_int, [_VP, ctypes.c_int]),
    "pg_get_ldpc_kernel": (ctypes.c_int, [_VP]),
    "pg_set_ldpc_order": (ctypes.c_int, [_VP, ctypes.c_int]),
    "pg_set_ldpc_kernel": (ctypes.c_int, [_VP, ctypes.c_int]),
    "pg_port_channel_estimate_host": (ctypes.c_int, [_VP] * 7),
    "pg_sch_decode_batch_resident": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, ctypes.c_size_t, _VP, _VP, _VP,
                                                    ctypes.c_size_t, _VP]),
}

_lib = None


def load():
    """Loads the library (once) and declares every exported signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"pusch_b200 native library not built: {LIB_PATH} (run __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class PgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Context:
    """Owns one pg_context (one CUDA device)."""

    def __init__(self, device=0, max_codeblocks=1024, max_llrs=0):
        self.lib = load()
        cfg = PgConfig(device, max_codeblocks, max_llrs)
        h = ctypes.c_void_p()
        rc = self.lib.pg_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != PG_OK:
            raise PgError(rc, "pg_create failed (is an sm_100 GPU visible?)")
        self.handle = h
        self.max_codeblocks = max_codeblocks

    def check(self, rc):
        if rc != PG_OK:
            raise PgError(rc, self.lib.pg_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

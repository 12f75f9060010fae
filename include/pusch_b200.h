/* pusch_b200 - C ABI of the B200 (sm_100a) PUSCH receive path.
 *
 * A flat C interface (plain pointers, sizes and POD structs; int status codes) that the
 * reference's PHY factory interfaces bind through thin C++17 adapters (see
 * ocudu-dapp-platform_b200/adapters). Each entry point names the reference interface it
 * replaces. Paths are relative to the reference project root.
 *
 * Conventions
 *  - Every entry returns PG_OK (0) on success or a PG_ERR_* code; pg_last_error() gives text.
 *  - "_device" entry points take device pointers and enqueue on the given CUDA stream
 *    (cudaStream_t passed as void*, NULL = legacy default stream); they do not synchronise.
 *  - "_host" entry points take host pointers, copy in, run and copy out, and return when the
 *    results are in host memory.
 *  - LLRs are int8 in the reference's log_likelihood_ratio domain
 *    (include/ocudu/phy/upper/log_likelihood_ratio.h:235): finite values in [-120, 120],
 *    +/-127 = +/-infinity.
 *  - Bit buffers are packed MSB first (ocudu::bit_buffer layout).
 *  - A context is bound to one CUDA device and is not thread safe (like the reference objects;
 *    use one context per worker thread).
 */
#ifndef PUSCH_B200_H
#define PUSCH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_ABI_VERSION 1

enum pg_status {
  PG_OK            = 0,
  PG_ERR_INVALID   = 1, /* an argument or descriptor is out of range */
  PG_ERR_CUDA      = 2, /* a CUDA runtime call failed */
  PG_ERR_CAPACITY  = 3, /* the request exceeds the capacity the context was created with */
  PG_ERR_TIMEOUT   = 4, /* a bounded wait expired */
  PG_ERR_NO_DEVICE = 5  /* no usable sm_100 device */
};

/* CRC generator polynomials (include/ocudu/phy/upper/channel_coding/crc_calculator.h:17-24). */
enum pg_crc_poly {
  PG_CRC16   = 0,
  PG_CRC24A  = 1,
  PG_CRC24B  = 2,
  PG_CRC_NONE = 255 /* no CRC early stop: syndrome check after the last iteration */
};

typedef struct pg_context pg_context;

typedef struct pg_config {
  int device;         /* CUDA device ordinal */
  int max_codeblocks; /* largest LDPC batch one call may carry (sizes the message scratch) */
  int max_llrs;       /* largest total LLR count one _host call may carry */
} pg_config;

/* Creates a context on cfg->device. Replaces the reference's factory-time set-up
 * (lib/phy/upper/upper_phy_factories.cpp:665 create_ul_processor_factory). */
int pg_create(const pg_config* cfg, pg_context** out);
void pg_destroy(pg_context* ctx);
const char* pg_last_error(const pg_context* ctx);
int pg_abi_version(void);

/* ---------------------------------------------------------------------------------------- */
/* LDPC decoding                                                                             */

/* One codeblock of a decode batch.
 * Replaces the per-call configuration of ldpc_decoder::decode
 * (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h:26-58): base graph, lifting size,
 * filler bits, CRC (its length selects CRC16 or CRC24 as the reference's nof_crc_bits does) and
 * maximum iterations. */
typedef struct pg_ldpc_cb {
  uint32_t llr_offset;      /* first LLR of this codeblock in the batch LLR buffer */
  uint32_t nof_llrs;        /* LLRs given: (K_b+2)*Z <= nof_llrs <= N_short*Z (rate-dematched) */
  uint32_t out_offset;      /* byte offset of this codeblock's K_b*Z decoded bits */
  uint16_t lifting_size;    /* Z, one of the 51 TS 38.212 lifting sizes */
  uint16_t nof_filler_bits; /* F: the last F of the K_b*Z message bits are fillers */
  uint8_t  base_graph;      /* 1 or 2 */
  uint8_t  crc_poly;        /* pg_crc_poly */
  uint8_t  max_iterations;  /* 1..255 */
  uint8_t  reserved;
} pg_ldpc_cb;

/* Batched layered normalised min-sum decoding, bit-exact with the reference's
 * ldpc_decoder_avx512 / ldpc_decoder_avx2
 * (lib/phy/upper/channel_coding/ldpc/ldpc_decoder_impl.cpp:41-145). For codeblock i:
 * iterations[i] = number of iterations when the CRC (or, with PG_CRC_NONE, the syndrome)
 * passes, else 0 - the reference's std::optional<unsigned>. bits receive ceil(K_b*Z/8) bytes at
 * out_offset; when fewer than K_b*Z soft bits are non-zero they are all ones.
 * Device pointers; the descriptors are read from host memory and staged by the library. */
int pg_ldpc_decode_batch_device(pg_context* ctx, const pg_ldpc_cb* cbs, int nof_cbs, const int8_t* llrs,
                                uint8_t* bits, int32_t* iterations, void* stream);

/* Same, with the descriptors already in device memory (nothing is staged: suitable for CUDA
 * graph capture and device-built work lists). */
int pg_ldpc_decode_batch_resident(pg_context* ctx, const pg_ldpc_cb* cbs_dev, int nof_cbs, const int8_t* llrs,
                                  uint8_t* bits, int32_t* iterations, void* stream);

/* Largest batch pg_ldpc_decode_batch_static_scratch accepts: its check-to-variable scratch is a
 * fixed device array of this many codeblocks of BG1 at Z = 384 (121,344 bytes each, 7.4 MiB). */
#define PG_STATIC_SCRATCH_MAX_CODEBLOCKS 64

/* No counterpart in the reference: an addition of this library. Same decode as
 * pg_ldpc_decode_batch_resident (descriptors already in device memory, same results), but the
 * call allocates no device memory and does not use the context's scratch: the check-to-variable
 * messages live in a device array of the library module, reserved when the module loads, so the
 * batch is bounded by PG_STATIC_SCRATCH_MAX_CODEBLOCKS instead of the context's max_codeblocks;
 * larger batches fail with PG_ERR_CAPACITY. For callers that must not allocate while decoding:
 * a real-time PHY worker under a slot deadline, where an allocation's driver locks and device
 * synchronisation have no latency bound, and a process whose device memory was reserved at
 * start-up, which must not meet out-of-memory during traffic.
 * The array's device address is looked up when the context is created (pg_create), so the call
 * itself makes no CUDA runtime call besides its launch (and, with kernel timing enabled, the two
 * event records read by pg_last_kernel_ms). All calls on a device share the one array: calls whose kernels may
 * overlap in time (different streams without ordering, several host threads) race on it, so
 * order them on one stream or synchronise between them. */
int pg_ldpc_decode_batch_static_scratch(pg_context* ctx, const pg_ldpc_cb* cbs_dev, int nof_cbs, const int8_t* llrs,
                                        uint8_t* bits, int32_t* iterations, void* stream);

/* Same, from and to host memory (H2D of the LLRs and D2H of bits and iterations inside the
 * call). This is what the ldpc_decoder / pusch_resident_codeblock_decoder::decode_batch
 * adapters call (include/ocudu/phy/upper/channel_processors/pusch/
 * pusch_resident_codeblock_decoder.h). */
int pg_ldpc_decode_batch_host(pg_context* ctx, const pg_ldpc_cb* cbs, int nof_cbs, const int8_t* llrs,
                              size_t nof_llrs_total, uint8_t* bits, size_t bits_bytes, int32_t* iterations);

/* Size in bytes of the decoded-bit output of one codeblock: ceil(K_b*Z/8). */
int pg_ldpc_output_bytes(int base_graph, int lifting_size);

/* Enables (1) or disables (0) CUDA-event timing of the decode kernel launches (LDPC decoding,
 * UL-SCH demultiplexing, short-block UCI detection). */
int pg_set_kernel_timing(pg_context* ctx, int enabled);

/* Device time of the most recent of those kernels in milliseconds (CUDA events on its stream),
 * or a negative value when none was recorded. */
float pg_last_kernel_ms(pg_context* ctx);

/* LDPC decoding kernels; every one gives the same bits and iteration counts. No counterpart in the
 * reference, whose decoder runs one codeblock per CPU task. */
enum pg_ldpc_kernel {
  PG_LDPC_KERNEL_ONE_LANE  = 0, /* 384 threads per codeblock, one lifted lane per thread, two CTAs per SM */
  PG_LDPC_KERNEL_TWO_LANES = 1, /* 192 threads per codeblock; even Z > 192: two lanes per thread as f16x2
                                   halves; four CTAs per SM */
  PG_LDPC_KERNEL_SPLIT     = 2, /* 384 threads per codeblock; even Z > 192: two lanes per thread pair, each
                                   row's edges split between the two threads; two CTAs per SM */
  PG_LDPC_KERNEL_Z384      = 3, /* 192 threads per codeblock; Z = 384 with the lifted edge tables in shared
                                   memory and f16 soft-bit pairs stored once, other Z as TWO_LANES; up to
                                   three CTAs per SM */
  PG_LDPC_KERNEL_Z384_SPLIT = 4 /* 384 threads per codeblock; Z = 384 as Z384 with each row's edges split
                                   over the two threads of a lane pair, other Z as SPLIT; two CTAs per SM */
};

/* Selects the kernel of the context's batch decodes (pg_ldpc_decode_batch_{host,device,resident}
 * and pg_sch_decode_batch_host); slot plans choose theirs through their tuning. */
int pg_set_ldpc_kernel(pg_context* ctx, int kernel);
/* Work order of the context's batch decodes: the codeblocks as given, or longest first (the
 * default): an estimate of each codeblock's decoding time from its input (the edges its rows cover
 * times Z, over the LLR magnitude per message bit) orders the persistent decoders' work list, so that
 * the long decodes start first. Results do not depend on the order. */
enum pg_ldpc_order { PG_LDPC_ORDER_GIVEN = 0, PG_LDPC_ORDER_LONGEST_FIRST = 1 };
int pg_set_ldpc_order(pg_context* ctx, int mode);
/* The kernel of the context's batch decodes (pg_ldpc_kernel), or a negative error code. */
int pg_get_ldpc_kernel(const pg_context* ctx);
/* Resident CTAs per SM of the context's batch decodes (1-4, capped by the kernel's own limit; 0:
 * the kernel's limit, the default). Fewer CTAs than codeblocks make the persistent CTAs share the
 * codeblocks dynamically; more make every codeblock start at once. */
int pg_set_ldpc_ctas_per_sm(pg_context* ctx, int ctas_per_sm);


/* ---------------------------------------------------------------------------------------- */
/* Rate dematching                                                                           */

/* One codeblock of a rate-dematching batch: the fields of codeblock_metadata that
 * ldpc_rate_dematcher::rate_dematch reads (include/ocudu/phy/upper/codeblock_metadata.h). */
typedef struct pg_rm_cb {
  uint32_t in_offset;       /* first of this codeblock's E rate-matched LLRs in the input */
  uint32_t rm_length;       /* E (a multiple of the modulation order) */
  uint32_t out_offset;      /* first of this codeblock's N = N_short*Z buffer LLRs in the output */
  uint32_t nref;            /* N_ref (limited-buffer rate matching), 0 = unlimited */
  uint16_t lifting_size;    /* Z */
  uint16_t nof_filler_bits; /* F */
  uint8_t  base_graph;      /* 1 or 2 */
  uint8_t  rv;              /* redundancy version 0..3 */
  uint8_t  modulation_order;/* Qm: 1, 2, 4, 6 or 8 */
  uint8_t  new_data;        /* 1: overwrite the buffer; 0: soft-combine into it (HARQ) */
} pg_rm_cb;

/* Batched rate dematching, replacing ldpc_rate_dematcher::rate_dematch
 * (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h:36-39;
 * lib/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher_impl.cpp:29-250). Device pointers; the
 * output buffers are read when new_data == 0. */
int pg_rate_dematch_batch_device(pg_context* ctx, const pg_rm_cb* cbs, int nof_cbs, const int8_t* in, int8_t* out,
                                 void* stream);
/* Same from and to host memory (out is read for soft combining and written back). */
int pg_rate_dematch_batch_host(pg_context* ctx, const pg_rm_cb* cbs, int nof_cbs, const int8_t* in, size_t in_len,
                               int8_t* out, size_t out_len);

/* ---------------------------------------------------------------------------------------- */
/* CRC and transport-block assembly                                                          */

/* One CRC computation over nof_bits bits starting at bit_offset of a packed MSB-first buffer. */
typedef struct pg_crc_item {
  uint32_t bit_offset;
  uint32_t nof_bits;
  uint32_t poly; /* PG_CRC16, PG_CRC24A or PG_CRC24B */
} pg_crc_item;

/* Batched crc_calculator::calculate(const bit_buffer&)
 * (include/ocudu/phy/upper/channel_coding/crc_calculator.h:67-77): remainder of each bit string
 * (zero initial value, MSB first, no output XOR; 0 means the string ends in a valid CRC). */
int pg_crc_calculate_device(pg_context* ctx, const pg_crc_item* items, int nof_items, const uint8_t* data,
                            uint32_t* crcs, void* stream);
int pg_crc_calculate_host(pg_context* ctx, const pg_crc_item* items, int nof_items, const uint8_t* data,
                          size_t data_len, uint32_t* crcs);

/* One transport block to assemble from decoded codeblocks (all codeblocks of a TB have the same
 * payload size per TS 38.212 Section 5.2.2). */
typedef struct pg_tb_desc {
  uint32_t cb_first;        /* index of the TB's first codeblock in cb_bit_offsets */
  uint32_t nof_cbs;         /* C */
  uint32_t cb_payload_bits; /* K' - L per codeblock (L = 24 when C > 1, else 0) */
  uint32_t tbs_bits;        /* transport block size, a multiple of 8 */
  uint32_t tb_out_offset;   /* byte offset of the TB payload in tb_out */
  uint32_t crc_poly;        /* PG_CRC16 or PG_CRC24A */
} pg_tb_desc;

/* Concatenates the codeblock payloads of each TB into tb_out (TBS/8 bytes) and computes the TB CRC
 * remainder over TBS + CRC bits (0 = TB CRC passes), as the reference's TB join
 * (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:612-710). cb_bit_offsets[i] is
 * the bit offset of codeblock i's decoded bits in cb_bits (device memory, like all buffers). */
int pg_tb_assemble_device(pg_context* ctx, const pg_tb_desc* tbs, int nof_tbs, const uint8_t* cb_bits,
                          const uint32_t* cb_bit_offsets, uint8_t* tb_out, uint32_t* tb_crc, void* stream);

/* ---------------------------------------------------------------------------------------- */
/* Segmentation and transport-block decoding (pusch_decoder)                                 */

/* Segmentation of one UL-SCH transport block (TS 38.212 Sections 5.2.2 and 5.4.2.1), the
 * quantities the reference's ldpc_segmenter_rx computes
 * (lib/phy/upper/channel_coding/ldpc/ldpc_segmenter_rx_impl.cpp:33-85,
 * include/ocudu/ran/sch/sch_segmentation.h:40-118). */
typedef struct pg_sch_segmentation {
  uint32_t nof_cbs;         /* C */
  uint32_t lifting_size;    /* Z_c */
  uint32_t cb_length;       /* K = K_b * Z_c (22 or 10 info columns) */
  uint32_t nof_filler_bits; /* F */
  uint32_t cb_crc_bits;     /* 24 when C > 1, else 0 */
  uint32_t tb_crc_bits;     /* 16 or 24 */
  uint32_t nof_short_cbs;   /* codeblocks with E = floor(...); the rest have E = ceil(...) */
  uint32_t e_short;         /* E of the short codeblocks */
  uint32_t e_long;          /* E of the long codeblocks */
} pg_sch_segmentation;

int pg_sch_segment(uint32_t tbs_bits, int base_graph, int modulation_order, int nof_layers,
                   uint32_t nof_ch_symbols, pg_sch_segmentation* out);

/* One UL-SCH transport block to decode from its (descrambled) codeword LLRs: the configuration
 * of pusch_decoder::new_data / set_nof_softbits (include/ocudu/phy/upper/channel_processors/
 * pusch/pusch_decoder.h:38-145). */
typedef struct pg_sch_tb {
  uint32_t llr_offset;      /* first codeword LLR (G = nof_ch_symbols * Qm * layers LLRs) */
  uint32_t nof_ch_symbols;  /* channel symbols of the codeword (all layers) */
  uint32_t tbs_bits;        /* transport block size */
  uint32_t tb_out_offset;   /* byte offset of the decoded TB */
  uint32_t nref;            /* N_ref, 0 = unlimited */
  uint8_t  base_graph;
  uint8_t  modulation_order;
  uint8_t  nof_layers;
  uint8_t  rv;
  uint8_t  max_iterations;
  uint8_t  reserved[3];
} pg_sch_tb;

/* Per-TB result: the reference's pusch_decoder_result (tb_crc_ok, codeblock counts and the
 * LDPC iteration statistics). */
typedef struct pg_sch_result {
  uint32_t tb_crc_ok;
  uint32_t nof_cbs;
  uint32_t nof_cbs_crc_ok;
  float    mean_iterations;  /* over the TB's codeblocks (failed codeblocks count max_iterations) */
  uint32_t max_iterations_run;
} pg_sch_result;

/* Decodes a batch of transport blocks end to end on the GPU: segmentation (host), rate
 * dematching, LDPC decoding with CRC early stop, TB assembly and TB CRC - the work of
 * pusch_decoder_impl (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:22-921) for
 * new transmissions. Host buffers in and out. */
int pg_sch_decode_batch_host(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* llrs,
                             size_t nof_llrs_total, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results);

/* pg_sch_decode_batch_host with the codeword soft bits already in device memory (llrs, a device
 * buffer of nof_llrs_total soft bits; the TBs, results and tb_out are host memory): the
 * transport-block decode of pusch_resident_codeblock_decoder::decode_resident_softbits
 * (include/ocudu/phy/upper/channel_processors/pusch/pusch_resident_codeblock_decoder.h:126-137).
 * c_init (host, one per TB, may be NULL): the soft bits are still scrambled and are descrambled on the
 * device with the Gold sequence of that initialisation from position bit_offset[t] (NULL: 0) -
 * TS 38.211 Section 6.3.1.1; the caller's buffer is left unchanged. */
int pg_sch_decode_batch_resident(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* llrs,
                                 size_t nof_llrs_total, const uint32_t* c_init, const uint32_t* bit_offset,
                                 uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results);

/* ---------------------------------------------------------------------------------------- */
/* Equalisation and soft demapping                                                           */

enum pg_eq_algorithm { PG_EQ_ZF = 0, PG_EQ_MMSE = 1 };

/* Channel equalisation, replacing channel_equalizer::equalize
 * (include/ocudu/phy/upper/equalization/channel_equalizer.h:71-76;
 * lib/phy/upper/equalization/channel_equalizer_generic_impl.cpp:511-653).
 * ch_symbols: complex bf16 (cbf16_t, real in the low 16 bits) [port][re];
 * ch_estimates: complex bf16 [port][layer][re]; noise_var_per_port: host array of nof_ports;
 * outputs layer-interleaved: eq_symbols complex float [re][layer], eq_noise_vars [re][layer].
 * One layer uses the per-port reduction (ZF and MMSE alike, as the reference); two and four
 * layers use MMSE with the largest port noise variance. */
int pg_equalize_device(pg_context* ctx, int algorithm, int nof_re, int nof_ports, int nof_layers,
                       const uint32_t* ch_symbols, const uint32_t* ch_estimates, const float* noise_var_per_port,
                       float tx_scaling, float* eq_symbols, float* eq_noise_vars, void* stream);
int pg_equalize_host(pg_context* ctx, int algorithm, int nof_re, int nof_ports, int nof_layers,
                     const uint32_t* ch_symbols, const uint32_t* ch_estimates, const float* noise_var_per_port,
                     float tx_scaling, float* eq_symbols, float* eq_noise_vars);

/* Soft demapping to int8 LLRs, replacing demodulation_mapper::demodulate_soft
 * (include/ocudu/phy/upper/channel_modulation/demodulation_mapper.h:48-51). symbols: complex
 * float; noise_vars: one per symbol; llrs: modulation_order per symbol (2, 4, 6 or 8). */
int pg_demodulate_soft_device(pg_context* ctx, int modulation_order, int nof_symbols, const float* symbols,
                              const float* noise_vars, int8_t* llrs, void* stream);
int pg_demodulate_soft_host(pg_context* ctx, int modulation_order, int nof_symbols, const float* symbols,
                            const float* noise_vars, int8_t* llrs);

/* Descrambling of soft bits (TS 38.211 Section 6.3.1.1, c_init = RNTI * 2^15 + n_ID): llrs_out[i]
 * = -llrs_in[i] where the Gold sequence bit c(i) is 1, else llrs_in[i]; in place allowed. The step
 * the reference's PUSCH demodulator applies after soft demapping (revert_scrambling,
 * pusch_demodulator_impl.cpp:23-33,409-414) and its offline replay tool repeats
 * (apps/tools/pusch_replay/ocudu_pusch_replay.cpp:266-296). At most 14 * 3276 * 2 * 8 soft bits. */
int pg_descramble_device(pg_context* ctx, uint32_t c_init, const int8_t* llrs_in, int8_t* llrs_out, size_t n,
                         void* stream);
int pg_descramble_host(pg_context* ctx, uint32_t c_init, const int8_t* llrs_in, int8_t* llrs_out, size_t n);

/* ---------------------------------------------------------------------------------------- */
/* PUSCH slot processing: DM-RS channel estimation, demodulation, decoding                   */

/* One UE's PUSCH PDU, the device work-list entry of the slot kernels (the fields of
 * pusch_processor::pdu_t the receive path reads: include/ocudu/phy/upper/channel_processors/
 * pusch/pusch_processor.h). DM-RS type 1, one CDM group (layers 0 and 1), two CDM groups without
 * data (no data on DM-RS symbols), no frequency hopping, no transform precoding, no UCI. */
typedef struct pg_pusch_ue {
  uint32_t grid_offset;      /* element offset of the UE's cell grid: cbf16 [port][14][grid_nof_subc] */
  uint32_t grid_nof_subc;    /* subcarriers of that grid (12 x carrier PRBs) */
  uint32_t llr_offset;       /* first codeword LLR of this UE in the LLR buffer */
  uint32_t est_offset;       /* first complex float of this UE's frequency response buffer */
  uint32_t tbs_bits;         /* transport block size */
  uint32_t tb_out_offset;    /* byte offset of the decoded TB */
  uint32_t nref;             /* N_ref for limited-buffer rate matching, 0 = unlimited */
  float    dmrs_scaling;     /* DM-RS amplitude relative to data (sqrt(2) for two CDM groups) */
  uint16_t rb_start;
  uint16_t nof_rb;
  uint16_t dmrs_symbol_mask; /* bit s set: OFDM symbol s carries DM-RS */
  uint16_t n_id;             /* DM-RS scrambling identity */
  uint16_t rnti;
  uint16_t n_id_data;        /* data scrambling identity */
  int16_t  dc_subcarrier;    /* grid subcarrier of DC (its channel estimate is zeroed), -1 = none */
  uint8_t  slot;             /* slot index within the frame */
  uint8_t  n_scid;
  uint8_t  first_symbol;
  uint8_t  nof_symbols;
  uint8_t  nof_rx_ports;     /* 1, 2 or 4 */
  uint8_t  nof_layers;       /* 1 or 2 */
  uint8_t  modulation_order; /* 2, 4, 6 or 8 */
  uint8_t  base_graph;
  uint8_t  rv;
  uint8_t  max_iterations;
} pg_pusch_ue;

/* Per (UE, receive port) estimator outputs (port_channel_estimator_results,
 * include/ocudu/phy/upper/signal_processors/channel_estimator/port_channel_estimator.h:107-139). */
typedef struct pg_port_result {
  float noise_var;
  float epre;
  float snr;
  float rsrp[2];
} pg_port_result;

/* Complex floats of one UE's frequency-response buffer: ports x DM-RS symbols x layers x 12 nof_rb. */
size_t pg_pusch_est_size(const pg_pusch_ue* ue);

/* DM-RS channel estimation for every (UE, receive port), replacing
 * port_channel_estimator::compute with FD "filter", TD "interpolate", no CFO compensation
 * (lib/phy/upper/signal_processors/channel_estimator/port_channel_estimator_average_impl.cpp:322-557)
 * and the pilot generation of dmrs_pusch_estimator_impl (dmrs_pusch_estimator_impl.cpp:69-169).
 * Writes the FP32 frequency response at every DM-RS symbol (est, layout
 * [port][dmrs symbol][layer][subcarrier]) and one pg_port_result per (UE, port), port-major per UE
 * (results[u * 4 + port]). Device pointers. */
int pg_pusch_estimate_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids, float* est,
                             pg_port_result* results, void* stream);

/* Per-symbol channel estimates of one UE as the reference's
 * port_channel_estimator_results::get_symbol_ch_estimate returns them: cbf16 [port][symbol][layer]
 * [12 nof_rb] for symbols 0..13 (time interpolation between DM-RS symbols, rounded to bf16).
 * basis (may be NULL): the learned estimator's time-basis coefficients of the UE (same layout as
 * est, see pg_le_refine_device), added to the interpolation with two DM-RS symbols. Device
 * pointers. */
int pg_pusch_symbol_estimates_device(pg_context* ctx, const pg_pusch_ue* ue, const float* est, const float* basis,
                                     uint32_t* out,
                                     void* stream);

/* One receive port of one allocation for port_channel_estimator::compute
 * (include/ocudu/phy/upper/signal_processors/channel_estimator/port_channel_estimator.h:86-89): the
 * fields of its configuration the estimator reads. DM-RS type 1, CDM group 0 (one or two layers), one
 * or two DM-RS symbols, contiguous resource blocks, no frequency hopping, normal cyclic prefix. */
typedef struct pg_port_estimate_cfg {
  uint32_t grid_nof_subc;    /* subcarriers of each grid row */
  float    scaling;          /* DM-RS amplitude relative to data (configuration::scaling) */
  uint16_t rb_start;
  uint16_t nof_rb;
  uint16_t dmrs_symbol_mask; /* bit s: OFDM symbol s carries DM-RS */
  uint8_t  first_symbol;
  uint8_t  nof_symbols;
  uint8_t  nof_layers;       /* 1 or 2 */
  uint8_t  scs_khz;          /* 15, 30, 60 or 120 */
  uint8_t  reserved[2];
} pg_port_estimate_cfg;

/* The scalars of port_channel_estimator_results (port_channel_estimator.h:107-139). */
typedef struct pg_port_estimate_result {
  float  noise_var;
  float  epre;
  float  snr;
  float  rsrp[2];
  float  cfo_hz;           /* NaN with one DM-RS symbol (the reference's empty optional) */
  double time_alignment_s; /* DFT-based time alignment estimate */
} pg_port_estimate_result;

/* port_channel_estimator::compute with FD "filter", TD "interpolate", no CFO compensation, for one
 * port, from and to host memory: grid cbf16 [14][grid_nof_subc] (that port's slot), pilots complex
 * float [dmrs symbol][layer][6 nof_rb] (the caller's DM-RS sequences, as dmrs_pusch_estimator
 * builds them). Writes the FP32 frequency response freq_response [dmrs symbol][layer][12 nof_rb],
 * optionally the per-symbol estimates symbol_estimates cbf16 [14][layer][12 nof_rb] (what
 * get_symbol_ch_estimate returns), and the scalars, including the CFO
 * (port_channel_estimator_average_impl.cpp:593-615) and the time alignment of
 * time_alignment_estimator_dft (lib/phy/support/time_alignment_estimator/
 * time_alignment_estimator_dft_impl.cpp:97-233). */
int pg_port_channel_estimate_host(pg_context* ctx, const pg_port_estimate_cfg* cfg, const uint32_t* grid,
                                  const float* pilots, float* freq_response, uint32_t* symbol_estimates,
                                  pg_port_estimate_result* result);

/* Demodulation of every UE: per data RE the channel estimate of its OFDM symbol (time interpolation
 * between DM-RS symbols, rounded to bf16, DC subcarrier zeroed), equalisation (one layer: MRC with
 * per-port noise; two layers: MMSE with the largest port noise), soft demapping and descrambling
 * (c_init = RNTI * 2^15 + n_ID_data), writing ue.llr_offset.. of llrs in codeword order. Replaces
 * pusch_demodulator::demodulate (lib/phy/upper/channel_processors/pusch/pusch_demodulator_impl.cpp:254-461).
 * Device pointers; est and port_results as written by pg_pusch_estimate_device. */
int pg_pusch_demodulate_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                               const float* est, const pg_port_result* port_results, int8_t* llrs, void* stream);

/* Whole PUSCH receive path for a batch of UEs (any number of cells): H2D of the grids, channel
 * estimation, demodulation, rate dematching, LDPC decoding, TB assembly and CRC, D2H of the TBs and
 * results - pusch_processor::process for new transmissions without UCI
 * (lib/phy/upper/channel_processors/pusch/pusch_processor_impl.cpp:349-900). The library assigns
 * the est_offset and llr_offset fields; tb_out_offset, grid_offset/grid_nof_subc are the caller's.
 * grids: host cbf16 words; port_results: nof_ues * 4 entries (may be NULL). */
int pg_pusch_process_host(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                          size_t grid_words, uint8_t* tb_out, size_t tb_out_len, pg_port_result* port_results,
                          pg_sch_result* results);

/* ---------------------------------------------------------------------------------------- */
/* Slot plans: one batch of PDUs (any number of UEs and cells) prepared once, executed per slot */

/* A plan holds everything of pusch_processor::process that depends only on the PDUs
 * (lib/phy/upper/channel_processors/pusch/pusch_processor_impl.cpp:349-900): segmentation, the
 * work lists of every stage (uploaded to the device once), the device workspace and the
 * descrambling sequences. Executing it enqueues DM-RS estimation, demodulation, rate dematching,
 * LDPC decoding, TB assembly and CRC and the per-UE results on one stream with no host
 * synchronisation. The plan keeps a pointer to its context, which must outlive it; a plan is used
 * by one thread at a time. */
typedef struct pg_pusch_plan pg_pusch_plan;

typedef struct pg_pusch_plan_info_t {
  uint32_t nof_ues;
  uint32_t nof_codeblocks;
  uint64_t tb_bytes;     /* transport-block output bytes (max tb_out_offset + TBS/8) */
  uint64_t nof_llrs;     /* codeword LLRs of all UEs */
  uint64_t grid_words;   /* cbf16 words of the grids buffer */
  uint64_t device_bytes; /* device memory the plan holds */
  uint32_t nof_kernels;  /* kernels one execution launches with the current tuning and estimator */
  uint32_t h2d_grid_bytes; /* grid bytes a host execution copies: per cell grid, the subcarriers its
                              UEs occupy on every port and symbol (no kernel reads the rest) */
} pg_pusch_plan_info_t;

/* ues: host array of nof_ues PDUs whose grids lie in a buffer of grid_words cbf16 words; the
 * library assigns est_offset and llr_offset, the caller tb_out_offset, grid_offset and
 * grid_nof_subc. */
int  pg_pusch_plan_create(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, size_t grid_words,
                          pg_pusch_plan** out);

/* UCI multiplexed on one UE's PUSCH (HARQ-ACK and CSI Part 1 of 1 to 1706 bits each): the fields of
 * the reference's ulsch_demultiplex::configuration (include/ocudu/phy/upper/channel_processors/
 * pusch/ulsch_demultiplex.h:31-90) that pg_pusch_ue does not carry. All zero: no UCI. */
typedef struct pg_pusch_uci {
  uint32_t nof_harq_ack_rvd;            /* G^HARQ-ACK_rvd, reserved HARQ-ACK soft bits */
  uint32_t nof_enc_harq_ack_bits;       /* G^HARQ-ACK */
  uint32_t nof_enc_csi_part1_bits;      /* G^CSI-1 */
  uint16_t nof_harq_ack_bits;           /* O^HARQ-ACK, 0..1706 (above 11: polar-coded) */
  uint16_t nof_csi_part1_bits;          /* O^CSI-1, 0..1706 */
  uint8_t  nof_cdm_groups_without_data; /* DM-RS type 1: 1 or 2 */
  uint8_t  reserved[3];
} pg_pusch_uci;

/* Decoded UCI of one UE after an execution: the bits of each message of up to 11 bits (one per
 * byte, message bit i at index i; zeros for a longer message, whose bits pg_pusch_plan_uci_message
 * gives) and each message's validity (1: the reference's short-block detection test passes, or
 * every polar codeblock passes its CRC; 0 also when the UE carries no such message). */
typedef struct pg_pusch_uci_result {
  uint8_t harq_ack[11];
  uint8_t csi_part1[11];
  uint8_t harq_ack_valid;
  uint8_t csi_part1_valid;
} pg_pusch_uci_result;

/* pg_pusch_plan_create with UCI on PUSCH: uci holds one entry per UE (NULL: none). Each execution
 * demultiplexes the UCI UEs' codewords on the GPU (as pusch_processor_impl.cpp:616-712 configures
 * it: ulsch_demultiplex, the UL-SCH stream to the decoder, the UCI streams to the UCI decoders),
 * decodes the UL-SCH stream as usual, detects the short-block messages (1 to 11 bits) and decodes
 * the polar-coded ones (12 to 1706 bits; their codes are built when the plan is created, and a
 * message without a polar code for its encoded size makes the creation PG_ERR_INVALID). */
int  pg_pusch_plan_create_uci(pg_context* ctx, const pg_pusch_ue* ues, const pg_pusch_uci* uci, int nof_ues,
                              size_t grid_words, pg_pusch_plan** out);
/* UCI results of the plan's last execution (nof_ues entries, host memory). Reads device memory
 * synchronously: call after that execution's stream has completed. */
int  pg_pusch_plan_uci_results(pg_pusch_plan* plan, pg_pusch_uci_result* out);
/* One UCI message of the plan's last execution, any size: UE ue, field 0 HARQ-ACK / 1 CSI Part 1;
 * bits receives the message's bits (one per byte; len at least its size) and *valid its validity.
 * PG_ERR_INVALID when the UE carries no such message. Synchronous, as pg_pusch_plan_uci_results. */
int  pg_pusch_plan_uci_message(pg_pusch_plan* plan, int ue, int field, uint8_t* bits, size_t len, uint8_t* valid);
void pg_pusch_plan_destroy(pg_pusch_plan* plan);
int  pg_pusch_plan_info(const pg_pusch_plan* plan, pg_pusch_plan_info_t* info);

/* enabled = 1: execute_device captures its launches into a CUDA graph on the first call (and
 * again whenever its buffers or stream change) and replays the graph afterwards. Streams other
 * than the legacy default stream only; on the default stream the launches are enqueued directly. */
int pg_pusch_plan_set_graph(pg_pusch_plan* plan, int enabled);

/* HARQ soft combining (the reference's rate-dematch soft buffer,
 * lib/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher_impl.cpp:98-194, and its rx_buffer per HARQ
 * process, lib/phy/upper/rx_buffer_pool_impl.cpp, pusch_decoder_impl.cpp:412-430). The plan keeps
 * each UE's dematched codeblocks on the device between executions: for the UEs with new_data[u] ==
 * 0 the next execution combines the received LLRs into them (saturating sums, as the reference)
 * instead of overwriting them, with redundancy version rv[u] (0..3). new_data or rv may be NULL
 * (unchanged). Call it between executions (no execution of the plan in flight); it synchronises
 * the context's stream. A plan holds one soft buffer per UE, valid until its next new-data
 * execution. */
int pg_pusch_plan_set_harq(pg_pusch_plan* plan, const uint8_t* new_data, const uint8_t* rv);

/* Launch shapes of a plan's stages (the autotuner's search space). No counterpart in the
 * reference, whose stages are sized per UE and per codeblock by its thread pools. */
typedef struct pg_pusch_plan_tuning {
  int rm_ctas_per_cb;       /* rate dematching: CTAs per codeblock, 1..32 (default 8) */
  int demod_res_per_thread; /* demodulation: resource elements per thread, 1..8 (default 1) */
  int demod_block;          /* demodulation: threads per CTA, 64, 128 or 256 (default 256) */
  int ldpc_ctas_per_sm;     /* persistent LDPC decoders: CTAs per SM, 1..4 (default 2; the one-lane-per-
                               thread decoder holds at most 2) */
  int ldpc_kernel;          /* LDPC decoder (pg_ldpc_kernel), PG_LDPC_KERNEL_ONE_LANE .. _Z384_SPLIT
                               (default PG_LDPC_KERNEL_Z384) */
  int ldpc_order;           /* work order of the persistent decoders: 0 = largest codeblocks first, fixed
                               when the plan is created; 1 = longest predicted decode first, from every
                               execution's LLRs (pg_set_ldpc_order's estimate; default 1) */
} pg_pusch_plan_tuning;

int pg_pusch_plan_get_tuning(const pg_pusch_plan* plan, pg_pusch_plan_tuning* out);
/* Sets the shapes (validated); a captured graph is re-captured on the next execution. */
int pg_pusch_plan_set_tuning(pg_pusch_plan* plan, const pg_pusch_plan_tuning* tuning);

/* Autotuner: times whole-slot executions of the plan on `grids` (device) for candidate shapes of
 * each stage (coordinate descent, two passes; each candidate the minimum of `reps` executions
 * timed by CUDA events on the context's stream), keeps the fastest and returns it (best and
 * best_ms may be NULL). Results do not depend on the shapes. Synchronises. */
int pg_pusch_plan_autotune(pg_pusch_plan* plan, const uint32_t* grids, int reps, pg_pusch_plan_tuning* best,
                           float* best_ms);

/* Enqueues the slot on stream: grids (device, grid_words cbf16 words) -> tb_out (device,
 * tb_bytes; the assembled TB of every UE, valid where results[u].tb_crc_ok), results (device,
 * one pg_sch_result per UE) and port_results (device, nof_ues * 4 entries, or NULL). */
int pg_pusch_plan_execute_device(pg_pusch_plan* plan, const uint32_t* grids, uint8_t* tb_out, pg_sch_result* results,
                                 pg_port_result* port_results, void* stream);

/* The same from and to host memory: H2D of the grids, execution, D2H of results, port results
 * (may be NULL) and TBs; returns when the results are in host memory. As the reference, a TB's
 * payload is written to tb_out only when its CRC passes. */
int pg_pusch_plan_execute_host(pg_pusch_plan* plan, const uint32_t* grids, uint8_t* tb_out, size_t tb_out_len,
                               pg_sch_result* results, pg_port_result* port_results);

/* ---------------------------------------------------------------------------------------- */
/* Learned channel estimator: tensor-core building blocks                                    */

/* One 1-D convolution layer (kernel 5, zero 'same' padding) on the tensor cores: BF16 operands,
 * FP32 accumulation. Activations are [C/8][rows][8] bf16 (8-channel chunks, one 16-byte row per
 * position); samples are concatenated with at least two zero rows between them; rows with
 * row_valid[r] != 0 receive the layer output, the other rows are written as zeros. w: packed weights [5 taps][cin/8][cout][8] bf16
 * (w[t][ci/8][co][ci%8] = W[co][ci][t]); bias: cout floats; res: optional residual added before
 * the activation (same layout as y, may be NULL); relu != 0 applies max(0, .). (cin, cout) is
 * (16, 64), (64, 64) or (64, 16). err: device int set to 1 if a tensor-core completion wait
 * expired. No counterpart in the reference (the learned estimator is an addition). */
int pg_conv1d_forward_device(pg_context* ctx, int cin, int cout, const void* x, const void* w, const float* bias,
                             const void* res, void* y, const uint8_t* row_valid, int rows, int relu, int* err,
                             void* stream);

/* Input gradient of a (cin -> cout) layer: dx = conv(dy, W') with the packed transposed weights
 * w_t [5][cout/8][cin][8] (W'[ci][co][t] = W[co][ci][4 - t]), plus res (may be NULL), then zeroed
 * where the forward ReLU output `mask` ([cin/8][rows][8], may be NULL) is not positive. dy is
 * [cout/8][rows][8], dx [cin/8][rows][8]; rows that are not valid are written as zeros. No counterpart in the
 * reference. */
int pg_conv1d_backward_data_device(pg_context* ctx, int cin, int cout, const void* dy, const void* w_t,
                                   const void* res, const void* mask, void* dx, const uint8_t* row_valid, int rows,
                                   int* err, void* stream);

/* Weight and bias gradients of a (cin -> cout) layer, ADDED to dw (FP32 [5][cin][cout]:
 * dw[t][ci][co] += sum_r x[r + t - 2][ci] dy[r][co]) and db (FP32 [cout], may be NULL). x and dy in
 * the activation layout; rows outside samples must be zero in both. No counterpart in the
 * reference. */
int pg_conv1d_backward_weights_device(pg_context* ctx, int cin, int cout, const void* x, const void* dy, int rows,
                                      float* dw, float* db, int* err, void* stream);

/* Device time in milliseconds of the learned-estimator stage (features, network, corrected
 * estimates) of the most recent slot-plan execution of a timed context (pg_set_kernel_timing),
 * or a negative value when none was recorded. No counterpart in the reference. */
float pg_last_learned_ms(pg_context* ctx);

/* ---------------------------------------------------------------------------------------- */
/* Learned channel estimator                                                                 */

/* No counterpart in the reference: an addition of this library. A residual 1-D convolutional
 * network (input layer 16 -> 64 channels, 6 residual blocks of two 64 -> 64 layers, output layer
 * 64 -> 16; kernel 5; BF16 weights and activations, FP32 accumulation on the tensor cores) that
 * refines, per (UE, receive port, layer) allocation, the frequency responses of
 * pg_pusch_estimate_device at the DM-RS symbols from the plain estimate, the LS estimates and the
 * noise level. The plain estimator stays the per-allocation fallback (allocations can be left out;
 * non-finite corrections are dropped). Parameters: per layer, weights [5][cin][cout] then bias
 * [cout], FP32, layers in network order. A net is used by one thread and one plan at a time. */
typedef struct pg_le_net pg_le_net;

/* Optimiser of pg_le_train_step_device (Adam; weight decay on the weights only). */
typedef struct pg_le_adam {
  float lr;
  float beta1;
  float beta2;
  float eps;
  float weight_decay;
} pg_le_adam;

/* FP32 parameters of the network (256,848). */
size_t pg_le_nof_params(void);
/* Rows of the network's layout for a list of UEs (12 nof_rb per port and layer, plus gaps). */
size_t pg_le_rows(const pg_pusch_ue* ues, int nof_ues);
/* Creates a network with buffers for max_rows rows (about 2.1 KB of device memory per row). The
 * parameters start at zero: set them with pg_le_set_params. */
int  pg_le_create(pg_context* ctx, int max_rows, pg_le_net** out);
void pg_le_destroy(pg_le_net* net);
/* Host FP32 parameters in and out (count = pg_le_nof_params()); setting them resets Adam. */
int pg_le_set_params(pg_le_net* net, const float* params, size_t count);
int pg_le_get_params(pg_le_net* net, float* params, size_t count);
/* Gradients accumulated by the last pg_le_backward_device (same layout as the parameters). */
int pg_le_get_grads(pg_le_net* net, float* grads, size_t count);
/* Waits for the device and returns PG_ERR_TIMEOUT if a tensor-core completion wait of any of the
 * net's kernels expired since it was created. */
int pg_le_status(pg_le_net* net);

/* The network on given inputs: x [2][rows][8] bf16 features, row_valid per row, y [2][rows][8]
 * bf16 outputs (device pointers). The activations stay in the net for pg_le_backward_device. */
int pg_le_forward_device(pg_le_net* net, const void* x, const uint8_t* row_valid, int rows, void* y, void* stream);
/* Gradients of every parameter for the output gradient dy [2][rows][8] bf16 of the last forward
 * call (replaces the previous gradients). */
int pg_le_backward_device(pg_le_net* net, const void* dy, int rows, void* stream);

/* Refines est (as written by pg_pusch_estimate_ls_device, with its LS output ls and port results)
 * in place for the UEs with use[u] != 0 (use may be NULL: every UE), and, for UEs with two DM-RS
 * symbols, writes the network's time-basis coefficients to basis (may be NULL; same layout and
 * offsets as est, the slots of DM-RS symbols 0 and 1 holding a_1 and a_2). The channel at OFDM
 * symbol s is then h(s) = h_0 + (h_1 - h_0) w + a_1 w (1 - w) + a_2 w (1 - w) (2 w - 1) with
 * w = (s - d0) / (d1 - d0): the reference's linear time interpolation between the DM-RS symbols d0
 * and d1 (port_channel_estimator_average_impl.cpp:705-767) plus two terms the network learns, which
 * vanish at the DM-RS symbols. ues: host array with the est_offset of each UE. */
int pg_le_refine_device(pg_le_net* net, const pg_pusch_ue* ues, int nof_ues, const float* ls, float* est,
                        float* basis, const pg_port_result* port_results, const uint8_t* use, void* stream);
/* One training step on a batch of UEs: features -> forward -> mean squared error, over every data
 * symbol of the slot, of the channel the outputs give (refined DM-RS responses and time-basis terms,
 * as pg_le_refine_device applies them) against the true channel h_true ([port][14][layer]
 * [12 nof_rb] per UE, UEs back to back in the order given) -> backward -> Adam.
 * loss (device, 2 floats, may be NULL): the network's MSE and the plain estimator's MSE, both in
 * units of the allocations' mean channel power. */
int pg_le_train_step_device(pg_le_net* net, const pg_pusch_ue* ues, int nof_ues, const float* ls, const float* est,
                            const pg_port_result* port_results, const float* h_true, const pg_le_adam* opt,
                            float* loss, void* stream);

/* DM-RS estimation as pg_pusch_estimate_device that also writes the LS estimates (same layout as
 * est: the pilots' even subcarriers, zero on the odd ones) for the learned estimator; ls may be
 * NULL. */
int pg_pusch_estimate_ls_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                                float* est, float* ls, pg_port_result* results, void* stream);

/* Uses net (NULL: none) to refine the plan's channel estimates between estimation and
 * demodulation, for the UEs with use[u] != 0 (use: host array of nof_ues, or NULL for all).
 * The net must hold pg_le_rows of those UEs; a captured graph is re-captured on the next
 * execution. */
int pg_pusch_plan_set_learned(pg_pusch_plan* plan, pg_le_net* net, const uint8_t* use);


/* ---------------------------------------------------------------------------------------------
 * UCI on PUSCH: HARQ-ACK and CSI Part 1 of up to 1706 bits (the placeholder and reserved-RE rules
 * of messages of one or two bits; longer messages are demultiplexed alike). CSI Part 2 is not
 * supported (PG_ERR_INVALID). */

/* One codeword to demultiplex: the fields of ulsch_demultiplex::configuration
 * (include/ocudu/phy/upper/channel_processors/pusch/ulsch_demultiplex.h:31-58) plus the buffers.
 * The encoded sizes are multiples of modulation_order * nof_layers (as get_ulsch_information,
 * lib/ran/pusch/ulsch_info.cpp, produces them). */
typedef struct pg_ulsch_demux_config {
  uint32_t llr_offset;             /* descrambled codeword soft bits of this PDU in the input */
  uint32_t nof_llrs;               /* codeword soft bits of the allocation (checked) */
  uint32_t sch_offset;             /* output offsets, soft bits */
  uint32_t harq_ack_offset;
  uint32_t csi_part1_offset;
  uint32_t c_init;                 /* scrambling initial state, RNTI * 2^15 + n_ID (placeholders) */
  uint32_t nof_harq_ack_rvd;       /* reserved HARQ-ACK soft bits, G^HARQ-ACK_rvd */
  uint32_t nof_enc_harq_ack_bits;  /* G^HARQ-ACK */
  uint32_t nof_enc_csi_part1_bits; /* G^CSI-1 */
  uint16_t nof_prb;
  uint16_t dmrs_symbol_mask;       /* bit s: slot symbol s carries DM-RS */
  uint8_t  modulation_order;       /* 1, 2, 4, 6, 8 */
  uint8_t  nof_layers;             /* 1..4 */
  uint8_t  start_symbol_index;
  uint8_t  nof_symbols;
  uint8_t  dmrs_type;              /* 1 or 2 */
  uint8_t  nof_cdm_groups_without_data;
  uint16_t nof_harq_ack_bits;      /* O^HARQ-ACK, 0..1706 */
  uint16_t nof_csi_part1_bits;     /* O^CSI-1, 0..1706 */
} pg_ulsch_demux_config;

/* The rate-matching sizes of UCI multiplexed on PUSCH (TS 38.212 Sections 6.3.2.4.1.1-3 and
 * 6.3.2.4.2.1-3), replacing get_ulsch_information (include/ocudu/ran/pusch/ulsch_info.h:144,
 * lib/ran/pusch/ulsch_info.cpp:137-342) for DM-RS type 1: from the grant, the encoded soft-bit counts
 * of the UL-SCH, HARQ-ACK (and the reserved HARQ-ACK bits), CSI Part 1 and CSI Part 2 - the numbers
 * a pg_ulsch_demux_config or pg_pusch_uci takes. Host computation, no GPU. */
typedef struct pg_ulsch_info_config {
  uint32_t tbs_bits;                    /* 0: no UL-SCH on this PUSCH */
  float    target_code_rate;            /* R in (0, 1) (MCS rate / 1024); used without UL-SCH */
  float    alpha_scaling;               /* alpha (0.5, 0.65, 0.8 or 1) */
  float    beta_offset_harq_ack;        /* beta_offset values of TS 38.213 Table 9.3-1/2 */
  float    beta_offset_csi_part1;
  float    beta_offset_csi_part2;
  uint16_t nof_harq_ack_bits;           /* O^HARQ-ACK */
  uint16_t nof_csi_part1_bits;          /* O^CSI-1 */
  uint16_t nof_csi_part2_bits;          /* O^CSI-2 */
  uint16_t nof_rb;
  uint16_t dmrs_symbol_mask;            /* bit s: slot symbol s carries DM-RS */
  uint8_t  base_graph;                  /* LDPC base graph of the UL-SCH (1 or 2) */
  uint8_t  modulation_order;            /* 1, 2, 4, 6, 8 */
  uint8_t  nof_layers;                  /* 1..4 */
  uint8_t  start_symbol;
  uint8_t  nof_symbols;
  uint8_t  nof_cdm_groups_without_data; /* 1 or 2 */
  uint8_t  contains_dc;                 /* the allocation holds the DC subcarrier */
  uint8_t  reserved[3];
} pg_ulsch_info_config;

typedef struct pg_ulsch_info {
  uint32_t nof_ul_sch_bits;     /* G^UL-SCH */
  uint32_t nof_harq_ack_bits;   /* G^HARQ-ACK */
  uint32_t nof_harq_ack_rvd;    /* G^HARQ-ACK_rvd */
  uint32_t nof_csi_part1_bits;  /* G^CSI-1 */
  uint32_t nof_csi_part2_bits;  /* G^CSI-2 */
  uint32_t nof_harq_ack_re;     /* Q'_ACK */
  uint32_t nof_csi_part1_re;    /* Q'_CSI-1 */
  uint32_t nof_csi_part2_re;    /* Q'_CSI-2 */
  uint32_t nof_dc_overlap_bits; /* rate-matched bits on the DC subcarrier */
} pg_ulsch_info;

int pg_ulsch_information(const pg_ulsch_info_config* cfg, pg_ulsch_info* out);

/* Soft bits of the UL-SCH, HARQ-ACK and CSI Part 1 streams of one codeword (host computation, no
 * GPU): sizes[0..2]. PG_ERR_INVALID when the configuration is inconsistent or unsupported. */
int pg_ulsch_demultiplex_sizes(const pg_ulsch_demux_config* cfg, uint32_t* sizes);

/* Demultiplexes n codewords of descrambled soft bits (device llrs, as pg_pusch_demodulate_device
 * writes them) into UL-SCH, HARQ-ACK and CSI Part 1 streams (device buffers; the UCI ones may be
 * NULL when no PDU carries that field) - ulsch_demultiplex::demultiplex followed by the codeword's
 * blocks (lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.cpp:183-573): one- and
 * two-bit messages get their placeholder bits re-scrambled, and the REs of one- and two-bit
 * HARQ-ACK are zero in the UL-SCH stream. cfgs is a host array. */
int pg_ulsch_demultiplex_device(pg_context* ctx, const pg_ulsch_demux_config* cfgs, int n, const int8_t* llrs,
                                int8_t* sch, int8_t* harq_ack, int8_t* csi_part1, void* stream);

/* One short-block UCI message: short_block_detector::detect
 * (include/ocudu/phy/upper/channel_coding/short/short_block_detector.h), called by
 * uci_decoder_impl::decode for 1..11 bits (lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:101-111). */
typedef struct pg_uci_short_block {
  uint32_t llr_offset; /* demultiplexed soft bits */
  uint32_t nof_llrs;   /* E */
  uint32_t out_offset; /* nof_bits output bytes, one bit per byte */
  uint8_t  nof_bits;   /* 1..11 */
  uint8_t  modulation_order;
  uint8_t  reserved[2];
} pg_uci_short_block;

/* Detects n messages (items: host array; llrs, bits, valid: device buffers). valid[i] = 1 when the
 * reference's detection test passes; an invalid input span gives all-ones bits and valid 0. */
int pg_uci_short_block_detect_device(pg_context* ctx, const pg_uci_short_block* items, int n, const int8_t* llrs,
                                     uint8_t* bits, uint8_t* valid, void* stream);

/* One polar-coded UCI message of 12 to 1706 bits: uci_decoder_impl::decode_codeword_polar
 * (lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:25-99), called by
 * uci_decoder_impl::decode above 11 bits (:101-111): segmentation into one or two codeblocks
 * (include/ocudu/ran/uci/uci_info.h:22-47), per codeblock the polar code of polar_code_impl::set
 * (lib/phy/upper/channel_coding/polar/polar_code_impl.cpp:432-480, uplink nMax = 10, channel
 * interleaver present), rate dematching, simplified successive-cancellation decoding, deallocation
 * and the CRC6 / CRC11 check. */
typedef struct pg_uci_polar {
  uint32_t llr_offset; /* demultiplexed soft bits */
  uint32_t nof_llrs;   /* E of the message (both codeblocks) */
  uint32_t out_offset; /* nof_bits output bytes, one bit per byte */
  uint16_t nof_bits;   /* A, 12..1706 */
  uint16_t reserved;
} pg_uci_polar;

/* Decodes n messages (items: host array; llrs, bits, valid: device buffers). valid[i] = 1 when
 * every codeblock of message i passes its CRC (the reference's uci_status::valid). A message whose
 * code the reference's polar_code_impl rejects (E above 8192 per codeblock, K outside 18..25 and
 * 31..1023, E not above K + nPC) is PG_ERR_INVALID. */
int pg_uci_polar_decode_device(pg_context* ctx, const pg_uci_polar* items, int n, const int8_t* llrs, uint8_t* bits,
                               uint8_t* valid, void* stream);

/* The polar code of one codeblock as pg_uci_polar_decode_device builds it (host computation, no
 * GPU): polar_code_impl::set for K (payload + CRC + filler bits) and E. */
typedef struct pg_polar_code_info {
  uint16_t n, N, K, E;
  uint8_t  nPC, nWmPC;
  uint16_t pc_set[4];     /* sorted parity-check sub-channels, unused entries 1024 */
  uint32_t k_set[32];     /* bit i of word i / 32: sub-channel i carries message, CRC or parity */
  uint16_t subblock[1024]; /* sub-block interleaver J(0 .. N - 1) */
} pg_polar_code_info;
int pg_polar_code(uint32_t K, uint32_t E, pg_polar_code_info* out);


/* Pipelined host execution of consecutive slots: pg_pusch_plan_submit_host enqueues one slot and
 * returns without waiting - the host-to-device copy of its grids runs on a stream of its own into
 * one of two staging buffers, overlapping the processing of the slots before it; the grids then move into the plan's
 * grid buffer, the plan runs and its results come back to a pinned buffer of the slot.
 * pg_pusch_plan_collect_host waits for the oldest submitted slot and writes its results as
 * pg_pusch_plan_execute_host does. At most three slots are in flight (PG_ERR_INVALID beyond); the
 * grids of a slot are read asynchronously, so they stay untouched until its collect returns (pinned
 * host memory makes the copy asynchronous). The first submit allocates the staging and result
 * buffers. Do not mix with the plan's other execute calls while slots are in flight. */
int pg_pusch_plan_submit_host(pg_pusch_plan* plan, const uint32_t* grids);
int pg_pusch_plan_collect_host(pg_pusch_plan* plan, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results,
                               pg_port_result* port_results);

/* ---------------------------------------------------------------------------------------------
 * Open Fronthaul block-floating-point IQ (O-RAN.WG4.CUS Annex A.1.2): per PRB one exponent byte,
 * then the I and Q samples of the 12 subcarriers, data_width bits each, packed big-endian. */

/* Compressed bytes per PRB for data_width (1..16) bits: 1 + 3 * data_width; -1 when out of range. */
int pg_bfp_prb_bytes(int data_width);

/* Decompresses nof_prb consecutive PRBs (device bytes) into 12 * nof_prb complex bf16 words (device)
 * - iq_decompressor::decompress for compression_type::BFP (include/ocudu/ofh/compression/iq_decompressor.h;
 * lib/ofh/compression/iq_compression_bfp_impl.cpp:89-141, iq_compression_bfp_avx512.cpp:147-201),
 * with the rounding of the reference's x86 implementation for the width. A whole grid is one call:
 * its (port, symbol) rows are whole PRBs back to back. */
int pg_bfp_decompress_device(pg_context* ctx, const uint8_t* compressed, uint32_t nof_prb, int data_width,
                             uint32_t* iq, void* stream);

/* pg_pusch_plan_execute_host with the grids given as BFP-compressed PRBs (host bytes, the plan's
 * grid words / 12 PRBs in grid order): copies the compressed bytes, decompresses them on the GPU
 * into the plan's grid buffer and runs the plan. The first call allocates the plan's buffer for the
 * compressed bytes. */
int pg_pusch_plan_execute_host_bfp(pg_pusch_plan* plan, const uint8_t* compressed, size_t compressed_len,
                                   int data_width, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results,
                                   pg_port_result* port_results);

#ifdef __cplusplus
}
#endif

#endif /* PUSCH_B200_H */

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

/* Same, from and to host memory (H2D of the LLRs and D2H of bits and iterations inside the
 * call). This is what the ldpc_decoder / pusch_resident_codeblock_decoder::decode_batch
 * adapters call (include/ocudu/phy/upper/channel_processors/pusch/
 * pusch_resident_codeblock_decoder.h). */
int pg_ldpc_decode_batch_host(pg_context* ctx, const pg_ldpc_cb* cbs, int nof_cbs, const int8_t* llrs,
                              size_t nof_llrs_total, uint8_t* bits, size_t bits_bytes, int32_t* iterations);

/* Size in bytes of the decoded-bit output of one codeblock: ceil(K_b*Z/8). */
int pg_ldpc_output_bytes(int base_graph, int lifting_size);

/* Enables (1) or disables (0) CUDA-event timing of the decode kernel launches. */
int pg_set_kernel_timing(pg_context* ctx, int enabled);

/* Device time of the most recent decode kernel in milliseconds (CUDA events on its stream),
 * or a negative value when none was recorded. */
float pg_last_kernel_ms(pg_context* ctx);

#ifdef __cplusplus
}
#endif

#endif /* PUSCH_B200_H */

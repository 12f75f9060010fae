// Internal declarations shared by the pusch_b200 CUDA translation units.
#pragma once

#include "../../include/pusch_b200.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace pg {

// LDPC dimensions (TS 38.212 Section 5.3.2).
constexpr int kMaxZ          = 384;
constexpr int kBg1Rows       = 46;
constexpr int kBg2Rows       = 42;
constexpr int kBg1Edges      = 316;
constexpr int kBg2Edges      = 197;
constexpr int kMaxNodes      = 68;  // BG1 variable nodes before shortening
constexpr int kMaxRowDegree  = 19;
constexpr int kCrcPowLen     = 22 * kMaxZ + 64;  // x^e mod g for every exponent a codeblock CRC needs
constexpr int kC2vStride     = kBg1Edges * kMaxZ; // check-to-variable bytes per codeblock

inline int kb_of(int bg) { return bg == 1 ? 22 : 10; }
inline int nshort_of(int bg) { return bg == 1 ? 66 : 50; }

// Lifting-size set index (TS 38.212 Table 5.3.2-1), -1 when Z is not a lifting size.
int lifting_set_index(int Z);

// Polynomial and order of a pg_crc_poly.
void crc_poly_params(int poly, uint32_t* g, int* order);

struct device_buffers {
  int8_t*      c2v         = nullptr; // max_codeblocks * kC2vStride check-to-variable messages
  pg_ldpc_cb*  descs       = nullptr; // staged descriptors
  uint32_t*    crc_pow     = nullptr; // [3][kCrcPowLen]
  int8_t*      llrs        = nullptr; // staging for _host calls
  uint8_t*     bits        = nullptr;
  int32_t*     iterations  = nullptr;
  size_t       llr_cap     = 0;
  size_t       bits_cap    = 0;
};

} // namespace pg

struct pg_context {
  int                 device         = 0;
  int                 max_codeblocks = 0;
  int                 sm_count       = 0;
  pg::device_buffers  dev;
  pg_ldpc_cb*         host_descs     = nullptr; // pinned staging for descriptors
  void*               host_stage     = nullptr; // pinned staging for _host calls
  size_t              host_stage_cap = 0;
  cudaStream_t        stream         = nullptr; // stream of the _host calls
  cudaEvent_t         ev_start       = nullptr;
  cudaEvent_t         ev_stop        = nullptr;
  cudaEvent_t         ev_desc        = nullptr; // completion of the last descriptor upload
  bool                desc_pending   = false;
  bool                timed          = false;
  std::string         last_error;
};

namespace pg {

int set_error(pg_context* ctx, int code, const std::string& msg);
int check_cuda(pg_context* ctx, cudaError_t err, const char* what);

// Validates descriptors on the host; returns PG_OK or PG_ERR_INVALID with a message.
int validate_ldpc_descs(pg_context* ctx, const pg_ldpc_cb* cbs, int n, size_t nof_llrs_total, size_t bits_bytes);

// Uploads the constant base-graph tables (once per process and device).
int ldpc_upload_tables(pg_context* ctx);

// Enqueues the batched decoder; descs_dev holds n descriptors in device memory.
int ldpc_launch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                int32_t* iterations, cudaStream_t stream);

} // namespace pg

// Internal declarations shared by the pusch_b200 CUDA translation units.
#pragma once

#include "../../include/pusch_b200.h"

#include <cuda_runtime.h>
#include <array>
#include <cstdint>
#include <string>
#include <vector>

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
constexpr uint32_t kGoldWords = (14u * 3276u * 2u * 8u + 64u * 32u) / 32u + 2u; // Gold-sequence words per basis

inline int kb_of(int bg) { return bg == 1 ? 22 : 10; }
inline int nshort_of(int bg) { return bg == 1 ? 66 : 50; }

// Lifting-size set index (TS 38.212 Table 5.3.2-1), -1 when Z is not a lifting size.
int lifting_set_index(int Z);

// Polynomial (with its x^order term) and order of a pg_crc_poly (TS 38.212 Section 5.1).
__host__ __device__ inline void crc_poly_params(int poly, uint32_t* g, int* order)
{
  if (poly == PG_CRC16) {
    *g     = 0x11021u;
    *order = 16;
  } else if (poly == PG_CRC24A) {
    *g     = 0x1864cfbu;
    *order = 24;
  } else {
    *g     = 0x1800063u;
    *order = 24;
  }
}

// Host-to-device staging of one kind of descriptor list: pinned host copy, device copy and the
// event after which both may be reused (the last kernel that read them has completed).
struct staging_slot {
  void*       dev     = nullptr;
  void*       host    = nullptr;
  size_t      cap     = 0;
  cudaEvent_t ev      = nullptr;
  bool        pending = false;
};

struct device_buffers {
  int8_t*      c2v         = nullptr; // max_codeblocks * kC2vStride check-to-variable messages
  pg_ldpc_cb*  descs       = nullptr; // staged descriptors
  uint32_t*    crc_pow     = nullptr; // [3][kCrcPowLen]
  uint32_t*    crc_tabs    = nullptr; // [3][1024 + 2048]: x^k and x^(1024k) mod g
  uint32_t*    gold        = nullptr; // [32][kGoldWords]: x1 and the 31 unit-state x2 sequences
  int8_t*      llrs        = nullptr; // staging for _host calls
  uint8_t*     bits        = nullptr;
  int32_t*     iterations  = nullptr;
  int*         ldpc_counter = nullptr; // work counters of the persistent decoders (two ints)
  uint8_t*     ldpc_keys    = nullptr; // max_codeblocks work-order keys of the batch decodes
  uint32_t*    ldpc_order   = nullptr; // max_codeblocks work-order entries
  uint16_t*    ldpc_scale   = nullptr; // scale table of the two-lanes-per-thread decoder
  size_t       llr_cap     = 0;
  size_t       bits_cap    = 0;
};

} // namespace pg

struct pg_context {
  int                 device         = 0;
  int                 max_codeblocks = 0;
  int                 sm_count       = 0;
  int                 ldpc_ctas      = 1;       // resident decoder CTAs on the device
  pg::device_buffers  dev;
  pg_ldpc_cb*         host_descs     = nullptr; // pinned staging for descriptors
  void*               host_stage     = nullptr; // pinned staging for _host calls
  size_t              host_stage_cap = 0;
  cudaStream_t        stream         = nullptr; // stream of the _host calls
  cudaEvent_t         ev_start       = nullptr;
  cudaEvent_t         ev_stop        = nullptr;
  cudaEvent_t         ev_le_start    = nullptr; // learned-estimator stage of slot plans (timed contexts)
  cudaEvent_t         ev_le_stop     = nullptr;
  bool                le_recorded    = false;
  cudaEvent_t         ev_desc        = nullptr; // completion of the last descriptor upload
  bool                desc_pending   = false;
  pg::staging_slot    slots[8];                  // rate-dematch, CRC, TB, PUSCH, UE and UCI work lists
  void*               est_partials     = nullptr;  // partial sums of the batched channel estimation
  size_t              est_partials_cap = 0;
  void*               scratch_a      = nullptr;  // growable device scratch of the _host entries
  size_t              scratch_a_cap  = 0;
  void*               scratch_b      = nullptr;
  size_t              scratch_b_cap  = 0;
  bool                timed          = false;
  int8_t*             static_c2v     = nullptr;  // device address of the module-static LDPC scratch
  int                 ldpc_kernel    = PG_LDPC_KERNEL_Z384; // kernel of the batch decodes (pg_ldpc_kernel)
  int                 ldpc_ctas_per_sm = 0;   // resident CTAs per SM of the batch decodes (0: kernel limit)
  int                 ldpc_order_mode  = PG_LDPC_ORDER_LONGEST_FIRST; // work order of the batch decodes
  std::string         last_error;
};

namespace pg {

int set_error(pg_context* ctx, int code, const std::string& msg);
int check_cuda(pg_context* ctx, cudaError_t err, const char* what);

// Validates descriptors on the host; returns PG_OK or PG_ERR_INVALID with a message.
int validate_ldpc_descs(pg_context* ctx, const pg_ldpc_cb* cbs, int n, size_t nof_llrs_total, size_t bits_bytes);

// Uploads the constant base-graph tables (once per process and device).
int ldpc_upload_tables(pg_context* ctx);
int uci_upload_tables(pg_context* ctx);
// UL-SCH demultiplexing of n codewords (uci.cu): the device blob [UE table | symbol table | work
// items] that the kernel reads, built on the host; sizes (may be null) receives each codeword's
// UL-SCH, HARQ-ACK and CSI Part 1 soft bits. Returns an error text (empty: consistent).
struct uci_demux_work {
  size_t o_syms = 0, o_items = 0;
  int    nitems = 0;
};
std::string uci_demux_blob(const pg_ulsch_demux_config* cfgs, int n, std::vector<uint8_t>& blob, uci_demux_work& w,
                           std::vector<std::array<uint32_t, 3>>* sizes);
int uci_demux_launch(pg_context* ctx, const void* blob_dev, const uci_demux_work& w, const int8_t* llrs, int8_t* sch,
                     int8_t* harq_ack, int8_t* csi_part1, cudaStream_t s);
// Short-block UCI detection: the device items blob of n messages, and the launch.
std::string uci_short_blob(const pg_uci_short_block* items, int n, std::vector<uint8_t>& blob);
int uci_detect_launch(pg_context* ctx, const void* items_dev, int n, const int8_t* llrs, uint8_t* bits, uint8_t* valid,
                      cudaStream_t s);
// Polar-coded UCI: the device descriptors of n messages (codes built on the host; an error text for
// a message without a polar code), their launch, and both steps with the descriptors staged.
std::string uci_polar_blob(const pg_uci_polar* items, int n, std::vector<uint8_t>& blob);
int uci_polar_launch_dev(pg_context* ctx, const void* cbs_dev, int n, const int8_t* llrs, uint8_t* bits,
                         uint8_t* valid, cudaStream_t s);
int uci_polar_launch(pg_context* ctx, const pg_uci_polar* items, int n, const int8_t* llrs, uint8_t* bits,
                     uint8_t* valid, cudaStream_t s);
// Open Fronthaul BFP: compressed bytes per PRB, and decompression of nof_prb PRBs into cbf16.
int bfp_prb_bytes(int data_width);
int bfp_decompress_launch(pg_context* ctx, const uint8_t* in, uint32_t nof_prb, int data_width, uint32_t* out,
                          cudaStream_t s);

enum { SLOT_RM = 0, SLOT_CRC = 1, SLOT_TB = 2, SLOT_PUSCH = 3, SLOT_UE = 4, SLOT_UCI = 5, SLOT_UCI_SHORT = 6, SLOT_UCI_POLAR = 7 };

// Copies `bytes` of host descriptors to the slot's device buffer on stream s (growing it when
// needed); returns the device pointer in *dev. release_slot_after marks the slot busy until the
// work enqueued on s so far has completed.
int stage_slot(pg_context* ctx, int slot, const void* host, size_t bytes, cudaStream_t s, void** dev);
int release_slot_after(pg_context* ctx, int slot, cudaStream_t s);
void free_slots(pg_context* ctx);
int ensure_scratch(pg_context* ctx, void** buf, size_t* cap, size_t bytes, const char* what);

int validate_rm_descs(pg_context* ctx, const pg_rm_cb* cbs, int n, size_t in_total, size_t out_total);
int rate_dematch_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const int8_t* in, int8_t* out,
                        cudaStream_t stream);
// Same with ctas_per_cb CTAs per codeblock (1..32), over the n codeblocks list[0 .. n - 1] of
// descs_dev when list is not NULL (a plan's codeblocks that the demodulator does not store in place).
int rate_dematch_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const int8_t* in, int8_t* out,
                        cudaStream_t stream, int ctas_per_cb, const uint32_t* list = nullptr);
// Writes what rate dematching leaves at the positions no LLR reaches (+127 at the fillers, 0
// elsewhere) over the whole circular buffer of every codeblock with placed[c] = 1, to be done
// before the demodulator stores those codeblocks' LLRs in place.
int rm_prefill_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const uint8_t* placed, int8_t* out,
                      cudaStream_t stream);
void crc_tables_host(uint32_t* tab);
int crc_launch(pg_context* ctx, const pg_crc_item* items_dev, int n, const uint8_t* data, uint32_t* out,
               cudaStream_t stream);
// TB assembly and TB CRC. chunks_dev (may be NULL: a 2-D grid over every TB) lists the work items
// TB | chunk << 16 of tb_chunk_list, one CTA each.
int tb_assemble_launch(pg_context* ctx, const pg_tb_desc* tbs_dev, int n, const uint8_t* cb_bits,
                       const uint32_t* cb_bit_offsets, uint8_t* tb_out, uint32_t* tb_crc, cudaStream_t stream,
                       const uint32_t* chunks_dev = nullptr, int nof_chunks = 0);
// The 1,024-word chunks of every TB (n <= 65,535 TBs).
void tb_chunk_list(const pg_tb_desc* tbs, int n, std::vector<uint32_t>& out);

int demap_upload_tables(pg_context* ctx);
int est_upload_tables(pg_context* ctx);
int demod_upload_tables(pg_context* ctx, const void* slope, const void* intercept, const void* width);
uint32_t ue_codeword_bits(const pg_pusch_ue& u);
int demod_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t max_words, uint32_t total_tiles,
                 const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                 const pg_port_result* port_results, const uint32_t* seq_offsets_dev, uint32_t* seq_dev, int8_t* llrs,
                 cudaStream_t s);
// The batch's demodulation tiles (groups of consecutive subcarriers that one CTA demodulates over
// every data symbol), appended to `map` one word each: UE index | tile index within the UE's
// allocation << 16. Returns the number of tiles (the launchers refuse batches of more than
// kDemodMaxUes UEs).
constexpr int kDemodMaxUes = 65535;
uint32_t demod_tile_map(const pg_pusch_ue* ues, int n, std::vector<uint32_t>& map);
// Host-side work lists of a batch of transport blocks: one rate-dematch and one LDPC descriptor
// per codeblock, one TB descriptor per TB, the bit offset of each codeblock's decoded bits.
struct sch_work {
  std::vector<pg_rm_cb>   rm;
  std::vector<pg_ldpc_cb> ldpc;
  std::vector<pg_tb_desc> tbd;
  std::vector<uint32_t>   cb_bit_off;
  std::vector<int>        tb_first, tb_ncb;
  size_t                  rm_total = 0, bits_total = 0;
};
int build_sch_work(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, size_t nof_llrs_total, size_t tb_out_len,
                   sch_work& w);
// Scrambling sequences of every UE (c_init = RNTI * 2^15 + n_ID), words at seq_offsets_dev[u].
int scrambling_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t max_words,
                      const uint32_t* seq_offsets_dev, uint32_t* seq_dev, cudaStream_t s);
// Descrambling of n soft bits with the Gold sequence of c_init (in == out allowed).
int descramble_launch(pg_context* ctx, uint32_t c_init, const int8_t* in, int8_t* out, size_t n, cudaStream_t s);
// Demodulation with the scrambling sequences already generated.
int demod_only_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t total_tiles,
                      const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                      const pg_port_result* port_results, const uint32_t* seq_offsets_dev, const uint32_t* seq_dev,
                      int8_t* llrs, cudaStream_t s);
// Same with `block` threads per CTA (64, 128 or 256) and res_per_thread tiles per CTA (1..8), and
// the learned estimator's time-basis coefficients (basis, same layout as est; may be NULL) for the
// UEs with basis_use[u] != 0.
// Rate-dematch placement of one UE's codeword for the demodulator's direct stores (fused
// demodulation and rate dematching): the UE's codeblocks hold new data without repetition
// (E <= V = N_cb - F for each), so codeword bit g of codeblock r (E_r bits from off_r) lands in
// circular-buffer position pos(t), t = (g - off_r) mod Qm * (E_r / Qm) + (g - off_r) div Qm, with
// v = (v0 + t) mod V and pos = v < inf ? v : v + F (the placement of ldpc_rate_dematcher with
// new_data). The first n_small codeblocks carry e_small bits, the others e_large; codeblock r's
// buffer starts at out0 + r cb_len. enabled == 0: the UE's LLRs go to the codeword buffer instead.
struct rm_direct {
  uint32_t out0, cb_len, e_small, e_large, n_small, V, v0, inf, F, enabled;
};
int demod_only_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t total_tiles,
                      const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                      const pg_port_result* port_results, const uint32_t* seq_offsets_dev, const uint32_t* seq_dev,
                      int8_t* llrs, cudaStream_t s, int block, int res_per_thread, const float* basis = nullptr,
                      const uint8_t* basis_use = nullptr, const rm_direct* direct = nullptr, int8_t* rm_out = nullptr);
// Decodes transport blocks whose codeword LLRs are already in device memory (d_llrs, nof_llrs);
// uses scratch_b; results and TB payloads land in host memory.
int sch_decode_device_llrs(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* d_llrs,
                           size_t nof_llrs, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results);
int validate_ues(pg_context* ctx, const pg_pusch_ue* ues, int n);
// Channel estimation of a batch (pusch_estimate_chunk_kernel). est_work_build writes the work list
// of the UEs (one item per (UE, port, chunk of pilots)), then the first item of every (UE, port)
// (4 n + 1 entries), then each UE's offset in the pilot-bit rows of dmrs_bits_launch (n entries,
// *pilot_words words in total), and returns the item count. work_dev holds that blob on the device,
// partials nwork float4, arrivals 4 n ints that are zero before the launch (and again after it).
// pilot_bits (may be NULL: the kernel then forms the pilots from the Gold basis) holds the rows
// written by dmrs_bits_launch for the same UEs and blob.
int est_work_build(const pg_pusch_ue* ues, int n, std::vector<uint32_t>& blob, uint32_t* pilot_words = nullptr);
int estimate_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, const uint32_t* work_dev, int nwork,
                    void* partials, int* arrivals, const uint32_t* grids, float* est, float* ls,
                    pg_port_result* results, cudaStream_t s, const uint32_t* pilot_bits = nullptr);
// The DM-RS sequence bits of every UE (their slot, N_ID, n_SCID and symbols), once per plan.
int dmrs_bits_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, const uint32_t* work_dev, int nwork,
                     uint32_t* bits_dev, cudaStream_t s);
// The same from host UEs: stages the UEs and their work list (SLOT_UE), partials in the context.
int estimate_launch_host(pg_context* ctx, const pg_pusch_ue* ues, int n, const uint32_t* grids, float* est, float* ls,
                         pg_port_result* results, cudaStream_t s);
int max_nof_rb(const pg_pusch_ue* ues, int n);
int dmrs_count(const pg_pusch_ue& u, int* d0, int* d1);
int equalize_launch(pg_context* ctx, int nof_re, int nof_ports, int nof_layers, const uint32_t* y, const uint32_t* h,
                    const float* nvar_port_host, float tx, float2* out, float* out_var, cudaStream_t s);
int demap_launch(pg_context* ctx, int qm, int n, const float2* sym, const float* nvar, int8_t* llr, cudaStream_t s);

// Enqueues the batched decoder; descs_dev holds n descriptors in device memory.
int ldpc_launch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                int32_t* iterations, cudaStream_t stream);
// Same with a caller-provided check-to-variable scratch of min(n, ldpc_ctas) * kC2vStride bytes.
int ldpc_launch_scratch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                        int32_t* iterations, int8_t* c2v, cudaStream_t stream);
// Hardest-first work order (ldpc_score_kernel + ldpc_sort_kernel): keys n bytes, order n entries.
int ldpc_order_launch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* keys,
                      uint32_t* order, cudaStream_t stream);
// Persistent launch: min(n, ldpc_ctas) CTAs take codeblocks order[0..n) (identity when order is
// null) from *counter (device int, zeroed here on the stream); c2v holds one slab per CTA.
int ldpc_launch_persistent(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                           int32_t* iterations, int8_t* c2v, const uint32_t* order, int* counter,
                           cudaStream_t stream);
// Kinds of codeblocks a work list may hold: Z = 384 (two-lanes-per-thread decoder) and others.
// PG_LDPC_ROUTE_X2 routes the Z = 384 codeblocks to the two-lanes-per-thread decoder; without it
// ldpc_decode_kernel decodes every codeblock.
enum {
  PG_LDPC_KIND_OTHER  = 1,
  PG_LDPC_KIND_Z384   = 2,
  PG_LDPC_KIND_ALL    = 3,
  PG_LDPC_ROUTE_X2    = 4,
  PG_LDPC_ROUTE_SPLIT = 8,
  PG_LDPC_ROUTE_Z     = 16,
  PG_LDPC_ROUTE_ZS    = 32
};
// Route flags of a pg_ldpc_kernel value.
inline int ldpc_route(int kernel)
{
  return kernel == PG_LDPC_KERNEL_TWO_LANES ? PG_LDPC_ROUTE_X2
         : kernel == PG_LDPC_KERNEL_SPLIT   ? PG_LDPC_ROUTE_SPLIT
         : kernel == PG_LDPC_KERNEL_Z384    ? PG_LDPC_ROUTE_Z
         : kernel == PG_LDPC_KERNEL_Z384_SPLIT ? PG_LDPC_ROUTE_ZS
                                            : 0;
}
// Same with at most max_ctas CTAs per decoder kernel, launching only the decoders of `kinds`.
// counter: two device ints; c2v: one slab (kC2vStride bytes) per CTA.
int ldpc_launch_persistent(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                           int32_t* iterations, int8_t* c2v, const uint32_t* order, int* counter,
                           cudaStream_t stream, int max_ctas, int kinds);
// CTAs of ldpc_decode_kernel resident on the whole device.
int ldpc_resident_ctas(pg_context* ctx);

// Tensor-core 1-D convolutions (tc_conv1d.cu): kernel attributes, the forward launch over an
// activation buffer of R rows ([C/8][R][8] bf16; bias, res and mask may be null) and the weight
// gradient (adds to dw[5][cin][cout] and, when db is not null, to db[cout]).
int conv_setup(pg_context* ctx);
int conv_forward_launch(pg_context* ctx, int cin, int cout, const void* x, const void* w, const float* bias,
                        const void* res, const void* mask, void* y, const uint8_t* row_valid, int R, int relu,
                        int* err, cudaStream_t s);
int conv_wgrad_launch(pg_context* ctx, int cin, int cout, const void* x, const void* dy, int R, float* dw, float* db,
                      int* err, cudaStream_t s);

// Learned channel estimator (learned_est.cu): one allocation sequence of the network's row layout
// (a (UE, receive port, layer) allocation of 12 nof_rb rows).
struct le_seq {
  uint32_t row0;    // first row
  uint32_t len;     // rows = 12 nof_rb
  uint32_t est0;    // complex-float offset of (port, DM-RS symbol 0, layer) in est / ls / h_true
  uint32_t dstride; // complex floats from DM-RS symbol 0 to 1 (layers x 12 nof_rb)
  uint32_t pr;      // port-result index (u * 4 + port)
  float    beta;    // DM-RS amplitude
  uint32_t h0;      // complex-float offset of (port, OFDM symbol 0, layer) in the full-grid truth of training
                    // ([port][14][layer][12 nof_rb] per UE, UEs back to back); symbol stride dstride
  uint8_t  layer, nof_layers, nd;
  uint8_t  dsym;    // DM-RS symbols: first in bits 0-3, second in bits 4-7
};
static_assert(sizeof(le_seq) == 32, "le_seq layout");

// Sequences of the UEs with use[u] != 0 (all when use is null), est_offset already assigned;
// returns the rows of the layout (0 without sequences) and, in *terms, the loss terms (two per
// subcarrier and data symbol).
size_t le_build_seqs(const pg_pusch_ue* ues, int n, const uint8_t* use, std::vector<le_seq>& out, size_t* terms);
// PG_OK when the net's buffers hold `rows` rows and `nseq` sequences, else PG_ERR_CAPACITY.
int le_capacity(const pg_le_net* net, size_t rows, int nseq);
pg_context* le_context(const pg_le_net* net);
// Features -> network -> est += correction, for sequences already in device memory.
int le_refine_launch(pg_le_net* net, const le_seq* seqs_dev, int nseq, int R, const float* ls, float* est, float* basis,
                     const pg_port_result* pr, cudaStream_t s);
// Event-record flags for timing events on stream s: under stream capture the records become event
// nodes of the graph (external records).
unsigned int timing_record_flags(pg_context* ctx, cudaStream_t s);

} // namespace pg

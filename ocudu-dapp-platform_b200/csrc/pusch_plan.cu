// Slot plans: the PUSCH receive path of a batch of UEs (any number of cells) prepared once on the
// host and executed per slot as a fixed sequence of launches on one stream, with no host
// synchronisation in between (pusch_processor_impl::process / process_data,
// lib/phy/upper/channel_processors/pusch/pusch_processor_impl.cpp:349-900, for a whole slot of
// PDUs at once).
//
// Creation does everything that depends only on the PDUs: segmentation and the work lists of every
// stage (UE, rate-dematch, LDPC and TB descriptors, uploaded once), the device workspace (one
// allocation: frequency responses, LLRs, dematched codeblocks, decoded bits, check-to-variable
// scratch) and the descrambling sequences, which depend only on RNTI and n_ID.
// Execution per slot: DM-RS estimation -> demodulation (equalise, demap, descramble) -> rate
// dematching -> LDPC -> TB assembly and CRC -> per-UE results, optionally replayed as a CUDA graph
// captured on the first execution.
#include "pg_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

using namespace pg;

constexpr int kPlanInFlight = 3; // slots pg_pusch_plan_submit_host may hold before a collect

// The part of one cell's grid ([port][symbol][subcarrier] words from `offset`) that the plan's UEs
// occupy: subcarriers [sc0, sc0 + width) of every port and symbol. Host executions copy only these
// spans; no kernel reads a grid word outside them.
struct grid_span {
  size_t offset; // first word copied: the grid's offset + sc0
  size_t width;  // words per row
  size_t pitch;  // words between rows (subcarriers of the grid)
  size_t rows;   // ports x 14 symbols
};
extern "C" {
static int copy_grid_spans(pg_pusch_plan* plan, uint32_t* dst, const uint32_t* src, cudaStream_t s);
}

struct pg_pusch_plan {
  pg_context*              ctx = nullptr;
  int                      nof_ues = 0, nof_cbs = 0;
  size_t                   grid_words = 0, tb_bytes = 0, nof_llrs = 0, dev_bytes = 0, est_total = 0;
  uint32_t                 total_tiles = 0; // demodulation tiles
  int                      max_rb   = 1;
  int                      ldpc_kinds = 0; // PG_LDPC_KIND_* present in the plan
  std::vector<pg_pusch_ue> ues;
  std::vector<pg_rm_cb>    rm;                 // rate-dematch descriptors (host copy, for HARQ updates)
  std::vector<int>         tb_first, tb_ncb;   // codeblocks of each UE
  std::vector<rm_direct>   direct;             // host copies of d_direct / d_placed (rebuilt by set_harq)
  std::vector<uint8_t>     placed;
  std::vector<uint32_t>    unplaced;           // the other codeblocks: the rate-dematch launch's list
  size_t                   rm_total = 0;       // bytes of dematched codeblocks (the soft buffers)
  // Device: descriptors, then workspace.
  void*           dev      = nullptr;
  pg_pusch_ue*    d_ues    = nullptr;
  // UCI on PUSCH: the demultiplexer's device blob and work shape, the detector's message items,
  // the UCI soft bits, detected bits (pg_pusch_uci_result layout per UE) and validity per message.
  void*           d_uci_blob  = nullptr;
  uci_demux_work  uci_w;
  void*           d_uci_items = nullptr;
  int             uci_nmsg    = 0;
  int8_t*         d_uci_llr   = nullptr;
  uint8_t*        d_uci_bits  = nullptr;
  uint8_t*        d_uci_valid = nullptr;
  std::vector<int> uci_msg_ue, uci_msg_kind; // per message: UE and 0 HARQ-ACK / 1 CSI Part 1
  // Polar-coded messages (after the short-block ones in the message order): their descriptors,
  // their decoded bits, and per message the bit offset (in the short-block results or the polar
  // bits) and the size.
  int              uci_nshort   = 0;
  int              polar_n      = 0;
  void*            d_polar_cbs  = nullptr;
  uint8_t*         d_polar_bits = nullptr;
  std::vector<uint32_t> uci_msg_off, uci_msg_nbits;
  rm_direct*      d_direct   = nullptr; // per UE: fused rate-dematch placement of the demodulator
  uint8_t*        d_placed   = nullptr; // per codeblock: 1 when the demodulator places its LLRs
  uint32_t*       d_unplaced = nullptr; // capacity nof_cbs
  uint32_t*       d_pilot_bits = nullptr; // DM-RS sequence bits of every UE (dmrs_bits_launch)
  // Side branch of every execution: the in-place codeblocks' circular buffers are prefilled on
  // `aux` (forked from and joined back into the execution's stream) beside the channel estimation.
  cudaStream_t    aux        = nullptr;
  cudaEvent_t     ev_fork    = nullptr;
  cudaEvent_t     ev_join    = nullptr;
  cudaEvent_t     ev_ufork   = nullptr; // polar UCI decoding on the aux stream, beside the UL-SCH stages
  cudaEvent_t     ev_ujoin   = nullptr;
  uint32_t*       d_est_work = nullptr; // channel-estimation work list and per-(UE, port) first items
  void*           d_est_part = nullptr; // its partial sums
  int*            d_est_arr  = nullptr; // per-(UE, port) arrival counters, zero between executions
  int             est_nwork  = 0;
  pg_rm_cb*       d_rm     = nullptr;
  pg_ldpc_cb*     d_ldpc   = nullptr;
  pg_tb_desc*     d_tb     = nullptr;
  uint32_t*       d_cb_off = nullptr;
  uint32_t*       d_seq_off = nullptr;
  uint32_t*       d_tile_map = nullptr;
  uint32_t*       d_seq    = nullptr;
  float*          d_est    = nullptr;
  pg_port_result* d_pr     = nullptr;
  int8_t*         d_llr    = nullptr;
  int8_t*         d_rm_out = nullptr;
  uint8_t*        d_cb_bits = nullptr;
  uint32_t*       d_tb_crc = nullptr;
  int32_t*        d_iters  = nullptr;
  int8_t*         d_c2v    = nullptr;
  uint32_t*       d_order  = nullptr; // per-execution work order (device ordering)
  uint32_t*       d_order_static = nullptr; // largest codeblocks first, fixed at creation
  uint32_t*       d_tb_chunks    = nullptr; // TB-assembly work items (TB | chunk << 16)
  int             tb_nchunks     = 0;
  uint8_t*        d_keys   = nullptr; // work-order keys of the codeblocks // LDPC work order: largest codeblocks first
  int*            d_counter = nullptr; // work counter of the persistent decoder
  uint32_t*       d_grid   = nullptr; // grids of execute_host
  uint8_t*        d_tb_out = nullptr; // TBs of execute_host
  pg_sch_result*  d_res    = nullptr; // results of execute_host
  // Pinned host buffers of execute_host: [results | port results | TBs].
  void*           host     = nullptr;
  // Compressed grids of execute_host_bfp (allocated on its first call).
  uint8_t*        d_bfp     = nullptr;
  size_t          d_bfp_cap = 0;
  // Pipelined host execution (submit_host / collect_host; allocated on the first submit): two
  // staging buffers the next slots' grids are copied into while the current slot runs (each free
  // again once its grids moved into the grid buffer), the copy stream, and a pinned result slot per
  // slot in flight.
  uint32_t*       d_stage[2]                  = {nullptr, nullptr};
  cudaStream_t    copy_stream                 = nullptr;
  cudaEvent_t     ev_h2d                      = nullptr;
  cudaEvent_t     ev_stage_free[2]            = {nullptr, nullptr};
  cudaEvent_t     ev_done[kPlanInFlight]      = {nullptr, nullptr, nullptr};
  void*           host_slot[kPlanInFlight]    = {nullptr, nullptr, nullptr};
  uint64_t        submitted     = 0;
  uint64_t        collected     = 0;
  std::vector<grid_span> grid_spans;
  size_t                 h2d_grid_bytes = 0;
  // Learned estimator: the net, the LS estimates, the time-basis coefficients (same layout as
  // d_est) with the per-UE flags of the UEs that use them, and the sequences of the refined UEs.
  pg_le_net*      le_net      = nullptr;
  void*           le_dev      = nullptr;
  float*          d_ls        = nullptr;
  float*          d_basis     = nullptr;
  uint8_t*        d_basis_use = nullptr;
  le_seq*         d_le_seqs = nullptr;
  int             le_nseq   = 0;
  int             le_rows   = 0;
  // Launch shapes (defaults, or the autotuner's choice).
  pg_pusch_plan_tuning tuning = {8, 1, 256, 2, PG_LDPC_KERNEL_Z384, 1};
  // CUDA graph of execute_device.
  bool            use_graph = false;
  cudaGraphExec_t exec      = nullptr;
  const void*     key[5]    = {};
};

namespace {

// Per-UE pusch_decoder_result from the codeblock iteration counts and the TB CRC remainder:
// C == 1: the codeblock CRC is the TB CRC; C > 1: every codeblock CRC and the TB CRC. A failed
// codeblock counts max_iterations (pusch_decoder_impl.cpp:612-710).
__global__ void sch_results_kernel(const pg_tb_desc* __restrict__ tbs, const pg_pusch_ue* __restrict__ ues, int n,
                                   const int32_t* __restrict__ iters, const uint32_t* __restrict__ tb_crc,
                                   pg_sch_result* __restrict__ out)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) {
    return;
  }
  const pg_tb_desc d     = tbs[t];
  const uint32_t   maxit = ues[t].max_iterations;
  uint32_t         ok = 0, mx = 0;
  float            sum = 0.f;
  for (uint32_t c = 0; c < d.nof_cbs; ++c) {
    const int32_t  it  = iters[d.cb_first + c];
    const uint32_t run = it > 0 ? (uint32_t)it : maxit;
    ok += it > 0 ? 1u : 0u;
    sum += (float)run;
    mx = run > mx ? run : mx;
  }
  pg_sch_result r;
  r.tb_crc_ok          = (ok == d.nof_cbs && (d.nof_cbs == 1 || tb_crc[t] == 0)) ? 1u : 0u;
  r.nof_cbs            = d.nof_cbs;
  r.nof_cbs_crc_ok     = ok;
  r.mean_iterations    = sum / (float)d.nof_cbs;
  r.max_iterations_run = mx;
  out[t]               = r;
}

size_t al(size_t x)
{
  return (x + 255) & ~(size_t)255;
}

// Fused demodulation and rate dematching: per UE the placement of its codeword in the codeblock
// buffers when every codeblock holds new data without repetition (E <= N_cb - F), as a
// consecutive run of E values with the smaller ones first and buffers a constant stride apart;
// other UEs keep the codeword buffer and the rate-dematch kernel. placed[c] = 1 for the codeblocks
// of the enabled UEs (prefilled with rm_prefill_launch, left alone by the rate-dematch kernel).
void build_direct(const std::vector<pg_pusch_ue>& ues, const std::vector<pg_rm_cb>& rm, const std::vector<int>& first,
                  const std::vector<int>& ncb, std::vector<rm_direct>& direct, std::vector<uint8_t>& placed)
{
  direct.assign(ues.size(), rm_direct{});
  placed.assign(rm.size(), 0);
  for (size_t u = 0; u < ues.size(); ++u) {
    const int c0 = first[u], n = ncb[u];
    if (n <= 0) {
      continue;
    }
    const pg_rm_cb& a   = rm[c0];
    const int       bg  = a.base_graph;
    const int       Z   = a.lifting_size;
    const int       Kb  = bg == 1 ? 22 : 10;
    const int       N   = (bg == 1 ? 66 : 50) * Z;
    const int       Ncb = (a.nref > 0 && (int)a.nref < N) ? (int)a.nref : N;
    const int       F   = a.nof_filler_bits;
    const int       sys = (Kb - 2) * Z;
    const int       inf = sys - F;
    const int       V   = Ncb - F;
    const int       sh  = bg == 1 ? (a.rv == 0 ? 0 : a.rv == 1 ? 17 : a.rv == 2 ? 33 : 56)
                                  : (a.rv == 0 ? 0 : a.rv == 1 ? 13 : a.rv == 2 ? 25 : 43);
    const int       k0  = (int)(((long long)sh * Ncb) / N) * Z;
    const int       v0  = k0 < inf ? k0 : (k0 < sys ? inf : k0 - F);
    const uint32_t  es  = a.rm_length;
    const uint32_t  el  = rm[c0 + n - 1].rm_length;
    uint32_t        ns  = 0;
    while ((int)ns < n && rm[c0 + ns].rm_length == es) {
      ++ns;
    }
    const pg_pusch_ue& ue = ues[u];
    bool ok = ue.modulation_order == a.modulation_order && el <= (uint32_t)V && es <= el;
    for (int k = 0; k < n && ok; ++k) {
      const pg_rm_cb& c  = rm[c0 + k];
      const uint32_t  e  = (uint32_t)k < ns ? es : el;
      const uint32_t  in = ue.llr_offset + ((uint32_t)k < ns ? (uint32_t)k * es : ns * es + ((uint32_t)k - ns) * el);
      ok = c.new_data != 0 && c.base_graph == a.base_graph && c.lifting_size == a.lifting_size &&
           c.nof_filler_bits == a.nof_filler_bits && c.nref == a.nref && c.rv == a.rv &&
           c.modulation_order == a.modulation_order && c.rm_length == e && c.in_offset == in &&
           c.out_offset == a.out_offset + (uint32_t)k * (uint32_t)N &&
           e % (uint32_t)(ue.nof_layers * ue.modulation_order) == 0;
    }
    if (!ok) {
      continue;
    }
    rm_direct& d = direct[u];
    d.out0       = a.out_offset;
    d.cb_len     = (uint32_t)N;
    d.e_small    = es;
    d.e_large    = el;
    d.n_small    = ns;
    d.V          = (uint32_t)V;
    d.v0         = (uint32_t)v0;
    d.inf        = (uint32_t)inf;
    d.F          = (uint32_t)F;
    d.enabled    = 1;
    for (int k = 0; k < n; ++k) {
      placed[c0 + k] = 1;
    }
  }
}

// The codeblocks that the demodulator does not store in place, in codeblock order.
std::vector<uint32_t> unplaced_list(const std::vector<uint8_t>& placed)
{
  std::vector<uint32_t> list;
  for (size_t c = 0; c < placed.size(); ++c) {
    if (placed[c] == 0) {
      list.push_back((uint32_t)c);
    }
  }
  return list;
}

int enqueue(pg_pusch_plan* p, const uint32_t* grids, uint8_t* tb_out, pg_sch_result* results,
            pg_port_result* port_results, cudaStream_t s)
{
  pg_context* ctx = p->ctx;
  // Fork: the in-place codeblocks' prefill depends on nothing of this execution (the previous
  // execution on this stream, whose decoder read the buffers, precedes the fork).
  int rc = check_cuda(ctx, cudaEventRecord(p->ev_fork, s), "cudaEventRecord(fork)");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamWaitEvent(p->aux, p->ev_fork, 0), "cudaStreamWaitEvent(fork)");
  }
  if (rc == PG_OK) {
    rc = rm_prefill_launch(ctx, p->d_rm, p->nof_cbs, p->d_placed, p->d_rm_out, p->aux);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventRecord(p->ev_join, p->aux), "cudaEventRecord(join)");
  }
  if (rc == PG_OK) {
    rc = estimate_launch(ctx, p->d_ues, p->nof_ues, p->d_est_work, p->est_nwork, p->d_est_part, p->d_est_arr, grids,
                         p->d_est, p->le_net != nullptr ? p->d_ls : nullptr, port_results, s, p->d_pilot_bits);
  }
  if (rc == PG_OK && p->le_net != nullptr) {
    const unsigned int flags = timing_record_flags(ctx, s);
    if (ctx->timed) {
      cudaEventRecordWithFlags(ctx->ev_le_start, s, flags);
    }
    rc = le_refine_launch(p->le_net, p->d_le_seqs, p->le_nseq, p->le_rows, p->d_ls, p->d_est, p->d_basis,
                          port_results, s);
    if (ctx->timed) {
      cudaEventRecordWithFlags(ctx->ev_le_stop, s, flags);
      ctx->le_recorded = true;
    }
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent(join)");
  }
  if (rc == PG_OK) {
    rc = demod_only_launch(ctx, p->d_ues, p->nof_ues, p->total_tiles, p->d_tile_map, grids, p->d_est, port_results,
                           p->d_seq_off, p->d_seq, p->d_llr, s, p->tuning.demod_block, p->tuning.demod_res_per_thread,
                           p->le_net != nullptr ? p->d_basis : nullptr,
                           p->le_net != nullptr ? p->d_basis_use : nullptr, p->d_direct, p->d_rm_out);
  }
  if (rc == PG_OK && p->uci_w.nitems > 0) {
    // UCI UEs: their codewords into the UL-SCH stream (in the codeword buffer, after the codewords)
    // and the HARQ-ACK / CSI Part 1 streams, then the short-block detection of the messages.
    rc = uci_demux_launch(ctx, p->d_uci_blob, p->uci_w, p->d_llr, p->d_llr, p->d_uci_llr, p->d_uci_llr, s);
    if (rc == PG_OK) {
      rc = uci_detect_launch(ctx, p->d_uci_items, p->uci_nshort, p->d_uci_llr, p->d_uci_bits, p->d_uci_valid, s);
    }
    if (rc == PG_OK && p->polar_n > 0) {
      // The polar decoders read only the demultiplexed UCI streams: a branch of their own that
      // overlaps rate dematching and LDPC decoding, joined at the end.
      rc = check_cuda(ctx, cudaEventRecord(p->ev_ufork, s), "cudaEventRecord(UCI fork)");
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaStreamWaitEvent(p->aux, p->ev_ufork, 0), "cudaStreamWaitEvent(UCI fork)");
      }
      if (rc == PG_OK) {
        rc = uci_polar_launch_dev(ctx, p->d_polar_cbs, p->polar_n, p->d_uci_llr, p->d_polar_bits,
                                  p->d_uci_valid + p->uci_nshort, p->aux);
      }
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaEventRecord(p->ev_ujoin, p->aux), "cudaEventRecord(UCI join)");
      }
    }
  }
  if (rc == PG_OK && !p->unplaced.empty()) {
    rc = rate_dematch_launch(ctx, p->d_rm, (int)p->unplaced.size(), p->d_llr, p->d_rm_out, s,
                             p->tuning.rm_ctas_per_cb, p->d_unplaced);
  }
  const uint32_t* order = p->d_order_static;
  if (rc == PG_OK && p->nof_cbs > 1 && p->tuning.ldpc_order != 0) {
    // Longest first: the decoders take the codeblocks by the predicted decoding time of their input.
    rc    = ldpc_order_launch(ctx, p->d_ldpc, p->nof_cbs, p->d_rm_out, p->d_keys, p->d_order, s);
    order = p->d_order;
  }
  if (rc == PG_OK) {
    rc = ldpc_launch_persistent(ctx, p->d_ldpc, p->nof_cbs, p->d_rm_out, p->d_cb_bits, p->d_iters, p->d_c2v,
                                order, p->d_counter, s, p->tuning.ldpc_ctas_per_sm * ctx->sm_count,
                                p->ldpc_kinds | ldpc_route(p->tuning.ldpc_kernel));
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemsetAsync(tb_out, 0, p->tb_bytes, s), "cudaMemsetAsync(tb)");
  }
  if (rc == PG_OK) {
    rc = tb_assemble_launch(ctx, p->d_tb, p->nof_ues, p->d_cb_bits, p->d_cb_off, tb_out, p->d_tb_crc, s, p->d_tb_chunks,
                            p->tb_nchunks);
  }
  if (rc == PG_OK) {
    sch_results_kernel<<<(p->nof_ues + 127) / 128, 128, 0, s>>>(p->d_tb, p->d_ues, p->nof_ues, p->d_iters, p->d_tb_crc,
                                                                 results);
    rc = check_cuda(ctx, cudaGetLastError(), "sch_results_kernel launch");
  }
  if (rc == PG_OK && p->uci_w.nitems > 0 && p->polar_n > 0) {
    rc = check_cuda(ctx, cudaStreamWaitEvent(s, p->ev_ujoin, 0), "cudaStreamWaitEvent(UCI join)");
  }
  return rc;
}

void release(pg_pusch_plan* p)
{
  if (p->exec) {
    cudaGraphExecDestroy(p->exec);
  }
  cudaFree(p->dev);
  cudaFree(p->le_dev);
  cudaFree(p->d_bfp);
  cudaFree(p->d_stage[0]);
  cudaFree(p->d_stage[1]);
  if (p->copy_stream) {
    cudaStreamDestroy(p->copy_stream);
  }
  if (p->aux) {
    cudaStreamDestroy(p->aux);
  }
  for (cudaEvent_t e : {p->ev_h2d, p->ev_stage_free[0], p->ev_stage_free[1], p->ev_done[0], p->ev_done[1],
                        p->ev_done[2], p->ev_fork, p->ev_join, p->ev_ufork, p->ev_ujoin}) {
    if (e) {
      cudaEventDestroy(e);
    }
  }
  for (void* h : p->host_slot) {
    if (h) {
      cudaFreeHost(h);
    }
  }
  if (p->host) {
    cudaFreeHost(p->host);
  }
  delete p;
}

} // namespace

extern "C" {

int pg_pusch_plan_create(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, size_t grid_words, pg_pusch_plan** out)
{
  return pg_pusch_plan_create_uci(ctx, ues, nullptr, nof_ues, grid_words, out);
}

int pg_pusch_plan_create_uci(pg_context* ctx, const pg_pusch_ue* ues, const pg_pusch_uci* uci, int nof_ues,
                             size_t grid_words, pg_pusch_plan** out)
{
  if (ctx == nullptr || out == nullptr) {
    return PG_ERR_INVALID;
  }
  *out = nullptr;
  if (int rc = validate_ues(ctx, ues, nof_ues)) {
    return rc;
  }
  if (nof_ues == 0) {
    return set_error(ctx, PG_ERR_INVALID, "a plan needs at least one UE");
  }
  pg_pusch_plan* p = new (std::nothrow) pg_pusch_plan();
  if (p == nullptr) {
    return set_error(ctx, PG_ERR_CAPACITY, "out of host memory");
  }
  p->ctx        = ctx;
  p->nof_ues    = nof_ues;
  p->grid_words = grid_words;
  p->ues.assign(ues, ues + nof_ues);

  // UE layout: frequency responses, codeword LLRs and descrambling sequences back to back.
  std::vector<uint32_t>  seq_off(nof_ues);
  std::vector<pg_sch_tb> tbs(nof_ues);
  size_t                 est_total = 0, seq_total = 0;
  uint32_t               max_words = 0;
  for (int i = 0; i < nof_ues; ++i) {
    pg_pusch_ue& u = p->ues[i];
    if ((size_t)u.grid_offset + (size_t)u.nof_rx_ports * 14 * u.grid_nof_subc > grid_words) {
      release(p);
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(i) + ": grid beyond the buffer");
    }
    const uint32_t g = ue_codeword_bits(u);
    u.est_offset     = (uint32_t)est_total;
    p->nof_llrs      = (p->nof_llrs + 15) & ~(size_t)15; // 16-byte aligned codewords: vector LLR stores
    u.llr_offset     = (uint32_t)p->nof_llrs;
    est_total += pg_pusch_est_size(&u);
    p->nof_llrs += g;
    seq_off[i]           = (uint32_t)seq_total;
    const uint32_t words = (g + 31) / 32 + 2;
    seq_total += words;
    max_words = std::max(max_words, words);
    p->tb_bytes  = std::max(p->tb_bytes, (size_t)u.tb_out_offset + u.tbs_bits / 8);
    pg_sch_tb& t = tbs[i];
    t            = pg_sch_tb{};
    t.llr_offset       = u.llr_offset;
    t.nof_ch_symbols   = g / u.modulation_order;
    t.tbs_bits         = u.tbs_bits;
    t.tb_out_offset    = u.tb_out_offset;
    t.nref             = u.nref;
    t.base_graph       = u.base_graph;
    t.modulation_order = u.modulation_order;
    t.nof_layers       = u.nof_layers;
    t.rv               = u.rv;
    t.max_iterations   = u.max_iterations;
  }
  // UCI UEs: the demultiplexer's configuration, the UL-SCH stream in the codeword buffer after
  // the codewords (the TB decodes from there), the HARQ-ACK and CSI Part 1 streams in their own
  // buffer, one short-block message per field.
  std::vector<pg_ulsch_demux_config> ucfg;
  std::vector<pg_uci_short_block>    umsg;
  std::vector<pg_uci_polar>          pmsg;
  std::vector<int>                   pmsg_ue, pmsg_kind;
  size_t                             uci_llr_total = 0, polar_bits_total = 0;
  for (int i = 0; uci != nullptr && i < nof_ues; ++i) {
    const pg_pusch_uci& q = uci[i];
    if (q.nof_harq_ack_bits == 0 && q.nof_csi_part1_bits == 0) {
      continue;
    }
    const pg_pusch_ue&    u = p->ues[i];
    pg_ulsch_demux_config c = {};
    c.llr_offset            = u.llr_offset;
    c.nof_llrs              = ue_codeword_bits(u);
    c.c_init                = ((uint32_t)u.rnti << 15) + u.n_id_data;
    c.nof_harq_ack_rvd      = q.nof_harq_ack_rvd;
    c.nof_enc_harq_ack_bits = q.nof_enc_harq_ack_bits;
    c.nof_enc_csi_part1_bits = q.nof_enc_csi_part1_bits;
    c.nof_prb               = u.nof_rb;
    c.dmrs_symbol_mask      = u.dmrs_symbol_mask;
    c.modulation_order      = u.modulation_order;
    c.nof_layers            = u.nof_layers;
    c.start_symbol_index    = u.first_symbol;
    c.nof_symbols           = u.nof_symbols;
    c.dmrs_type             = 1;
    c.nof_cdm_groups_without_data = q.nof_cdm_groups_without_data;
    c.nof_harq_ack_bits     = q.nof_harq_ack_bits;
    c.nof_csi_part1_bits    = q.nof_csi_part1_bits;
    uint32_t sz[3]          = {0, 0, 0};
    if (pg_ulsch_demultiplex_sizes(&c, sz) != PG_OK) {
      release(p);
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(i) + ": inconsistent UCI configuration");
    }
    if ((q.nof_harq_ack_bits > 1706) || (q.nof_csi_part1_bits > 1706)) {
      release(p);
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(i) + ": UCI fields of 1 to 1706 bits");
    }
    p->nof_llrs      = (p->nof_llrs + 15) & ~(size_t)15;
    c.sch_offset     = (uint32_t)p->nof_llrs;
    p->nof_llrs += sz[0];
    c.harq_ack_offset  = (uint32_t)uci_llr_total;
    c.csi_part1_offset = (uint32_t)(uci_llr_total + sz[1]);
    for (int k = 0; k < 2; ++k) {
      const unsigned nbits = k == 0 ? q.nof_harq_ack_bits : q.nof_csi_part1_bits;
      if (nbits > 11) {
        pg_uci_polar m = {};
        m.llr_offset   = k == 0 ? c.harq_ack_offset : c.csi_part1_offset;
        m.nof_llrs     = sz[1 + k];
        m.out_offset   = (uint32_t)polar_bits_total;
        m.nof_bits     = (uint16_t)nbits;
        pmsg.push_back(m);
        pmsg_ue.push_back(i);
        pmsg_kind.push_back(k);
        polar_bits_total += nbits;
      } else if (nbits > 0) {
        pg_uci_short_block m = {};
        m.llr_offset         = k == 0 ? c.harq_ack_offset : c.csi_part1_offset;
        m.nof_llrs           = sz[1 + k];
        m.out_offset         = (uint32_t)(i * sizeof(pg_pusch_uci_result)) + (k == 0 ? 0u : 11u);
        m.nof_bits           = (uint8_t)nbits;
        m.modulation_order   = u.modulation_order;
        umsg.push_back(m);
        p->uci_msg_ue.push_back(i);
        p->uci_msg_kind.push_back(k);
        p->uci_msg_off.push_back(m.out_offset);
        p->uci_msg_nbits.push_back(nbits);
      }
    }
    uci_llr_total += sz[1] + sz[2];
    tbs[i].llr_offset     = c.sch_offset;
    tbs[i].nof_ch_symbols = sz[0] / u.modulation_order;
    ucfg.push_back(c);
  }
  std::vector<uint8_t> uci_blob, uci_items, polar_blob;
  if (!ucfg.empty()) {
    std::string err = uci_demux_blob(ucfg.data(), (int)ucfg.size(), uci_blob, p->uci_w, nullptr);
    if (err.empty()) {
      err = uci_short_blob(umsg.data(), (int)umsg.size(), uci_items);
    }
    if (err.empty()) {
      err = uci_polar_blob(pmsg.data(), (int)pmsg.size(), polar_blob);
    }
    if (!err.empty()) {
      release(p);
      return set_error(ctx, PG_ERR_INVALID, err);
    }
    p->uci_nshort = (int)umsg.size();
    p->polar_n    = (int)pmsg.size();
    for (size_t m = 0; m < pmsg.size(); ++m) {
      p->uci_msg_ue.push_back(pmsg_ue[m]);
      p->uci_msg_kind.push_back(pmsg_kind[m]);
      p->uci_msg_off.push_back(pmsg[m].out_offset);
      p->uci_msg_nbits.push_back(pmsg[m].nof_bits);
    }
    p->uci_nmsg = p->uci_nshort + p->polar_n;
  }
  {
    // Per cell grid (UEs sharing grid_offset), the span of the subcarriers its UEs occupy.
    std::vector<std::pair<uint32_t, grid_span>> cells;
    for (int i = 0; i < nof_ues; ++i) {
      const pg_pusch_ue& u   = p->ues[i];
      const size_t       sc0 = 12u * (size_t)u.rb_start, sc1 = 12u * ((size_t)u.rb_start + u.nof_rb);
      auto it = std::find_if(cells.begin(), cells.end(), [&](const auto& c) { return c.first == u.grid_offset; });
      if (it == cells.end()) {
        cells.push_back({u.grid_offset, grid_span{sc0, sc1 - sc0, u.grid_nof_subc, (size_t)u.nof_rx_ports * 14u}});
        continue;
      }
      grid_span&   g   = it->second;
      const size_t lo  = std::min(g.offset, sc0), hi = std::max(g.offset + g.width, sc1);
      g.offset         = lo;
      g.width          = hi - lo;
      g.pitch          = std::max<size_t>(g.pitch, u.grid_nof_subc);
      g.rows           = std::max<size_t>(g.rows, (size_t)u.nof_rx_ports * 14u);
    }
    for (auto& c : cells) {
      grid_span g = c.second;
      g.offset += c.first;
      if (g.width > g.pitch || g.offset + (g.rows - 1) * g.pitch + g.width > grid_words) {
        g = grid_span{c.first, c.second.pitch, c.second.pitch, c.second.rows}; // whole rows
      }
      p->grid_spans.push_back(g);
      p->h2d_grid_bytes += 4 * g.width * g.rows;
    }
  }
  p->max_rb    = max_nof_rb(p->ues.data(), nof_ues);
  p->est_total = est_total;
  std::vector<uint32_t> tile_map;
  p->total_tiles = demod_tile_map(p->ues.data(), nof_ues, tile_map);
  sch_work w;
  if (int rc = build_sch_work(ctx, tbs.data(), nof_ues, p->nof_llrs, p->tb_bytes, w)) {
    release(p);
    return rc;
  }
  p->nof_cbs  = (int)w.ldpc.size();
  p->rm       = w.rm;
  p->tb_first = w.tb_first;
  p->tb_ncb   = w.tb_ncb;
  p->rm_total = w.rm_total;
  // LDPC work order, largest first: a codeblock's cost grows with Z times the LLR positions it
  // fills (E + F, at most N), which fix the check rows it runs.
  std::vector<uint32_t> order(p->nof_cbs);
  std::vector<uint64_t> cost(p->nof_cbs);
  for (int c = 0; c < p->nof_cbs; ++c) {
    const pg_ldpc_cb& l = w.ldpc[c];
    order[c]            = (uint32_t)c;
    cost[c]             = (uint64_t)l.lifting_size * std::min<uint64_t>(w.rm[c].rm_length + l.nof_filler_bits, l.nof_llrs);
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  p->ldpc_kinds = 0;
  for (const pg_ldpc_cb& l : w.ldpc) {
    p->ldpc_kinds |= l.lifting_size == 384 ? PG_LDPC_KIND_Z384 : PG_LDPC_KIND_OTHER;
  }
  // One check-to-variable slab per decoder CTA: up to four per SM, at most one per codeblock.
  const int ldpc_slabs = std::max(1, std::min(p->nof_cbs, 4 * ctx->sm_count));

  // Device image: descriptors first (uploaded once), then the workspace.
  const size_t o_ues    = 0;
  const size_t o_rm     = o_ues + al((size_t)nof_ues * sizeof(pg_pusch_ue));
  const size_t o_ldpc   = o_rm + al(w.rm.size() * sizeof(pg_rm_cb));
  const size_t o_tb     = o_ldpc + al(w.ldpc.size() * sizeof(pg_ldpc_cb));
  const size_t o_cb_off = o_tb + al(w.tbd.size() * sizeof(pg_tb_desc));
  const size_t o_order  = o_cb_off + al(w.cb_bit_off.size() * 4);
  const size_t o_ostat  = o_order + al(order.size() * 4);
  std::vector<uint32_t> tb_chunks;
  tb_chunk_list(w.tbd.data(), (int)w.tbd.size(), tb_chunks);
  p->tb_nchunks         = (int)tb_chunks.size();
  const size_t o_tbch   = o_ostat + al(order.size() * 4);
  const size_t o_seqoff = o_tbch + al(tb_chunks.size() * 4);
  const size_t o_reoff  = o_seqoff + al((size_t)nof_ues * 4);
  std::vector<uint32_t> est_work;
  uint32_t              pilot_words = 0;
  p->est_nwork          = est_work_build(p->ues.data(), nof_ues, est_work, &pilot_words);
  std::vector<rm_direct> direct;
  std::vector<uint8_t>   placed;
  build_direct(p->ues, w.rm, w.tb_first, w.tb_ncb, direct, placed);
  p->direct     = direct;
  p->placed     = placed;
  p->unplaced   = unplaced_list(placed);
  const size_t o_ework  = o_reoff + al(tile_map.size() * 4);
  const size_t o_ublob  = o_ework + al(est_work.size() * 4);
  const size_t o_uitems = o_ublob + al(uci_blob.size());
  const size_t o_pcbs   = o_uitems + al(uci_items.size());
  const size_t o_direct = o_pcbs + al(polar_blob.size());
  const size_t o_fill   = o_direct + al(direct.size() * sizeof(rm_direct));
  const size_t o_unpl   = o_fill + al(placed.size());
  const size_t desc_end = o_unpl + al((size_t)p->nof_cbs * 4);
  const size_t o_seq    = desc_end;
  const size_t o_est    = o_seq + al(seq_total * 4);
  const size_t o_pr     = o_est + al(est_total * 8);
  const size_t o_llr    = o_pr + al((size_t)nof_ues * 4 * sizeof(pg_port_result));
  const size_t o_rmout  = o_llr + al(p->nof_llrs);
  const size_t o_bits   = o_rmout + al(w.rm_total);
  const size_t o_crc    = o_bits + al(w.bits_total);
  const size_t o_it     = o_crc + al((size_t)nof_ues * 4);
  const size_t o_keys   = o_it + al((size_t)p->nof_cbs * 4);
  const size_t o_cnt    = o_keys + al((size_t)p->nof_cbs);
  const size_t o_c2v    = o_cnt + al(sizeof(int));
  const size_t o_grid   = o_c2v + al((size_t)ldpc_slabs * kC2vStride);
  const size_t o_tbout  = o_grid + al(grid_words * 4);
  const size_t o_res    = o_tbout + al(p->tb_bytes);
  const size_t o_epart  = o_res + al((size_t)nof_ues * sizeof(pg_sch_result));
  const size_t o_earr   = o_epart + al((size_t)std::max(1, p->est_nwork) * 16);
  const size_t o_ullr   = o_earr + al((size_t)nof_ues * 16);
  const size_t o_ubits  = o_ullr + al(uci_llr_total);
  const size_t o_uvalid = o_ubits + al((size_t)nof_ues * sizeof(pg_pusch_uci_result));
  const size_t o_polb   = o_uvalid + al((size_t)std::max(1, p->uci_nmsg));
  const size_t o_pbits  = o_polb + al(polar_bits_total);
  p->dev_bytes          = o_pbits + al((size_t)pilot_words * 4);

  const size_t h_res  = 0;
  const size_t h_pr   = h_res + al((size_t)nof_ues * sizeof(pg_sch_result));
  const size_t h_tb   = h_pr + al((size_t)nof_ues * 4 * sizeof(pg_port_result));
  const size_t h_size = std::max(h_tb + al(p->tb_bytes), desc_end);

  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&p->dev, p->dev_bytes), "cudaMalloc(plan)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMallocHost(&p->host, h_size), "cudaMallocHost(plan)");
  }
  if (rc != PG_OK) {
    release(p);
    return rc;
  }
  uint8_t* b   = static_cast<uint8_t*>(p->dev);
  p->d_ues     = reinterpret_cast<pg_pusch_ue*>(b + o_ues);
  p->d_rm      = reinterpret_cast<pg_rm_cb*>(b + o_rm);
  p->d_ldpc    = reinterpret_cast<pg_ldpc_cb*>(b + o_ldpc);
  p->d_tb      = reinterpret_cast<pg_tb_desc*>(b + o_tb);
  p->d_cb_off  = reinterpret_cast<uint32_t*>(b + o_cb_off);
  p->d_seq_off = reinterpret_cast<uint32_t*>(b + o_seqoff);
  p->d_tile_map = reinterpret_cast<uint32_t*>(b + o_reoff);
  p->d_seq     = reinterpret_cast<uint32_t*>(b + o_seq);
  p->d_est     = reinterpret_cast<float*>(b + o_est);
  p->d_pr      = reinterpret_cast<pg_port_result*>(b + o_pr);
  p->d_llr     = reinterpret_cast<int8_t*>(b + o_llr);
  p->d_rm_out  = reinterpret_cast<int8_t*>(b + o_rmout);
  p->d_cb_bits = b + o_bits;
  p->d_tb_crc  = reinterpret_cast<uint32_t*>(b + o_crc);
  p->d_iters   = reinterpret_cast<int32_t*>(b + o_it);
  p->d_c2v     = reinterpret_cast<int8_t*>(b + o_c2v);
  p->d_order   = reinterpret_cast<uint32_t*>(b + o_order);
  p->d_order_static = reinterpret_cast<uint32_t*>(b + o_ostat);
  p->d_tb_chunks    = reinterpret_cast<uint32_t*>(b + o_tbch);
  p->d_counter = reinterpret_cast<int*>(b + o_cnt);
  p->d_keys    = b + o_keys;
  p->d_grid    = reinterpret_cast<uint32_t*>(b + o_grid);
  p->d_tb_out  = b + o_tbout;
  p->d_res     = reinterpret_cast<pg_sch_result*>(b + o_res);
  p->d_est_work = reinterpret_cast<uint32_t*>(b + o_ework);
  p->d_direct   = reinterpret_cast<rm_direct*>(b + o_direct);
  p->d_placed   = b + o_fill;
  p->d_unplaced = reinterpret_cast<uint32_t*>(b + o_unpl);
  p->d_pilot_bits = reinterpret_cast<uint32_t*>(b + o_pbits);
  p->d_est_part = b + o_epart;
  p->d_est_arr  = reinterpret_cast<int*>(b + o_earr);
  p->d_uci_blob  = b + o_ublob;
  p->d_uci_items = b + o_uitems;
  p->d_uci_llr   = reinterpret_cast<int8_t*>(b + o_ullr);
  p->d_uci_bits  = b + o_ubits;
  p->d_uci_valid = b + o_uvalid;
  p->d_polar_cbs  = b + o_pcbs;
  p->d_polar_bits = b + o_polb;

  // Descriptor image in pinned memory, one upload.
  uint8_t* h = static_cast<uint8_t*>(p->host);
  std::memset(h, 0, desc_end);
  std::memcpy(h + o_ues, p->ues.data(), (size_t)nof_ues * sizeof(pg_pusch_ue));
  std::memcpy(h + o_rm, w.rm.data(), w.rm.size() * sizeof(pg_rm_cb));
  std::memcpy(h + o_ldpc, w.ldpc.data(), w.ldpc.size() * sizeof(pg_ldpc_cb));
  std::memcpy(h + o_tb, w.tbd.data(), w.tbd.size() * sizeof(pg_tb_desc));
  std::memcpy(h + o_cb_off, w.cb_bit_off.data(), w.cb_bit_off.size() * 4);
  std::memcpy(h + o_order, order.data(), order.size() * 4);
  std::memcpy(h + o_ostat, order.data(), order.size() * 4);
  std::memcpy(h + o_tbch, tb_chunks.data(), tb_chunks.size() * 4);
  std::memcpy(h + o_seqoff, seq_off.data(), (size_t)nof_ues * 4);
  std::memcpy(h + o_reoff, tile_map.data(), tile_map.size() * 4);
  std::memcpy(h + o_ework, est_work.data(), est_work.size() * 4);
  if (!uci_blob.empty()) {
    std::memcpy(h + o_ublob, uci_blob.data(), uci_blob.size());
    std::memcpy(h + o_uitems, uci_items.data(), uci_items.size());
    std::memcpy(h + o_pcbs, polar_blob.data(), polar_blob.size());
  }
  std::memcpy(h + o_direct, direct.data(), direct.size() * sizeof(rm_direct));
  std::memcpy(h + o_fill, placed.data(), placed.size());
  std::memcpy(h + o_unpl, p->unplaced.data(), p->unplaced.size() * 4);
  cudaStream_t s = ctx->stream;
  rc = check_cuda(ctx, cudaMemcpyAsync(p->dev, h, desc_end, cudaMemcpyHostToDevice, s), "H2D plan descriptors");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking), "cudaStreamCreate(aux)");
  }
  for (cudaEvent_t* e : {&p->ev_fork, &p->ev_join, &p->ev_ufork, &p->ev_ujoin}) {
    if (rc == PG_OK) {
      rc = check_cuda(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate(fork/join)");
    }
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemsetAsync(b + o_seq, 0, al(seq_total * 4), s), "cudaMemsetAsync(sequences)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemsetAsync(b + o_earr, 0, (size_t)nof_ues * 16, s), "cudaMemsetAsync(arrivals)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemsetAsync(b + o_ubits, 0, (size_t)nof_ues * sizeof(pg_pusch_uci_result), s),
                    "cudaMemsetAsync(UCI results)");
  }
  if (rc == PG_OK) {
    rc = scrambling_launch(ctx, p->d_ues, nof_ues, max_words, p->d_seq_off, p->d_seq, s);
  }
  if (rc == PG_OK) {
    rc = dmrs_bits_launch(ctx, p->d_ues, nof_ues, p->d_est_work, p->est_nwork, p->d_pilot_bits, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize(plan)");
  }
  if (rc != PG_OK) {
    release(p);
    return rc;
  }
  *out = p;
  return PG_OK;
}

void pg_pusch_plan_destroy(pg_pusch_plan* plan)
{
  if (plan == nullptr) {
    return;
  }
  cudaStreamSynchronize(plan->ctx->stream);
  release(plan);
}

int pg_pusch_plan_info(const pg_pusch_plan* plan, pg_pusch_plan_info_t* info)
{
  if (plan == nullptr || info == nullptr) {
    return PG_ERR_INVALID;
  }
  info->nof_ues        = (uint32_t)plan->nof_ues;
  info->nof_codeblocks = (uint32_t)plan->nof_cbs;
  info->tb_bytes       = plan->tb_bytes;
  info->nof_llrs       = plan->nof_llrs;
  info->grid_words     = plan->grid_words;
  info->device_bytes   = plan->dev_bytes;
  // The kernels enqueue() launches: prefill, estimation, [learned: features, network, corrections],
  // demodulation, [UCI: demultiplexing, detection], [rate dematching of the codeblocks not placed],
  // [device work order: score, sort], LDPC, TB assembly, results.
  info->nof_kernels = 2u + (plan->le_net != nullptr ? 3u : 0u) + 1u + (plan->uci_w.nitems > 0 ? 1u : 0u) +
                      (plan->uci_nshort > 0 ? 1u : 0u) + (plan->polar_n > 0 ? 1u : 0u) +
                      (plan->unplaced.empty() ? 0u : 1u) + (plan->nof_cbs > 1 && plan->tuning.ldpc_order != 0 ? 2u : 0u) +
                      3u;
  info->h2d_grid_bytes = (uint32_t)std::min<size_t>(plan->h2d_grid_bytes, 0xffffffffu);
  return PG_OK;
}

int pg_pusch_plan_set_graph(pg_pusch_plan* plan, int enabled)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  plan->use_graph = enabled != 0;
  return PG_OK;
}

int pg_pusch_plan_set_learned(pg_pusch_plan* plan, pg_le_net* net, const uint8_t* use)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (net != nullptr && le_context(net) != ctx) {
    return set_error(ctx, PG_ERR_INVALID, "the learned estimator belongs to another context");
  }
  if (int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize")) {
    return rc;
  }
  if (plan->exec != nullptr) {
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  cudaFree(plan->le_dev);
  plan->le_dev      = nullptr;
  plan->le_net      = nullptr;
  plan->d_ls        = nullptr;
  plan->d_basis     = nullptr;
  plan->d_basis_use = nullptr;
  plan->d_le_seqs   = nullptr;
  plan->le_nseq = plan->le_rows = 0;
  if (net == nullptr) {
    return PG_OK;
  }
  std::vector<le_seq> seqs;
  const size_t        rows = le_build_seqs(plan->ues.data(), plan->nof_ues, use, seqs, nullptr);
  if (le_capacity(net, rows, (int)seqs.size()) != PG_OK) {
    return set_error(ctx, PG_ERR_CAPACITY,
                     "learned estimator: the plan needs " + std::to_string(rows) + " rows, more than the net holds");
  }
  const size_t o_basis = al(plan->est_total * 8);
  const size_t o_use   = o_basis + al(plan->est_total * 8);
  const size_t o_seq   = o_use + al((size_t)plan->nof_ues);
  const size_t bytes   = o_seq + al(std::max<size_t>(1, seqs.size()) * sizeof(le_seq));
  int          rc      = check_cuda(ctx, cudaMalloc(&plan->le_dev, bytes), "cudaMalloc(plan learned estimator)");
  std::vector<uint8_t> use_flags(plan->nof_ues);
  for (int u = 0; u < plan->nof_ues; ++u) {
    use_flags[u] = (use == nullptr || use[u] != 0) ? 1 : 0;
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemset(static_cast<uint8_t*>(plan->le_dev) + o_basis, 0, plan->est_total * 8),
                    "cudaMemset(plan time-basis coefficients)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaMemcpy(static_cast<uint8_t*>(plan->le_dev) + o_use, use_flags.data(), use_flags.size(),
                               cudaMemcpyHostToDevice),
                    "H2D plan learned-estimator flags");
  }
  if (rc == PG_OK && !seqs.empty()) {
    rc = check_cuda(ctx,
                    cudaMemcpy(static_cast<uint8_t*>(plan->le_dev) + o_seq, seqs.data(), seqs.size() * sizeof(le_seq),
                               cudaMemcpyHostToDevice),
                    "H2D plan learned-estimator sequences");
  }
  if (rc != PG_OK) {
    cudaFree(plan->le_dev);
    plan->le_dev = nullptr;
    return rc;
  }
  plan->d_ls        = static_cast<float*>(plan->le_dev);
  plan->d_basis     = reinterpret_cast<float*>(static_cast<uint8_t*>(plan->le_dev) + o_basis);
  plan->d_basis_use = static_cast<uint8_t*>(plan->le_dev) + o_use;
  plan->d_le_seqs   = reinterpret_cast<le_seq*>(static_cast<uint8_t*>(plan->le_dev) + o_seq);
  plan->le_nseq   = (int)seqs.size();
  plan->le_rows   = (int)rows;
  plan->le_net    = net;
  return PG_OK;
}

int pg_pusch_plan_uci_results(pg_pusch_plan* plan, pg_pusch_uci_result* out)
{
  if (plan == nullptr || out == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  std::vector<pg_pusch_uci_result> r(plan->nof_ues);
  std::vector<uint8_t>             valid(std::max(1, plan->uci_nmsg));
  int rc = check_cuda(ctx,
                      cudaMemcpy(r.data(), plan->d_uci_bits, r.size() * sizeof(pg_pusch_uci_result),
                                 cudaMemcpyDeviceToHost),
                      "D2H UCI bits");
  if (rc == PG_OK && plan->uci_nmsg > 0) {
    rc = check_cuda(ctx, cudaMemcpy(valid.data(), plan->d_uci_valid, (size_t)plan->uci_nmsg, cudaMemcpyDeviceToHost),
                    "D2H UCI validity");
  }
  if (rc != PG_OK) {
    return rc;
  }
  for (int u = 0; u < plan->nof_ues; ++u) {
    r[u].harq_ack_valid  = 0;
    r[u].csi_part1_valid = 0;
  }
  for (int m = 0; m < plan->uci_nmsg; ++m) {
    pg_pusch_uci_result& x = r[plan->uci_msg_ue[m]];
    (plan->uci_msg_kind[m] == 0 ? x.harq_ack_valid : x.csi_part1_valid) = valid[m];
  }
  std::memcpy(out, r.data(), r.size() * sizeof(pg_pusch_uci_result));
  return PG_OK;
}

int pg_pusch_plan_uci_message(pg_pusch_plan* plan, int ue, int field, uint8_t* bits, size_t len, uint8_t* valid)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (bits == nullptr || valid == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null argument");
  }
  int m = 0;
  while (m < plan->uci_nmsg && !(plan->uci_msg_ue[m] == ue && plan->uci_msg_kind[m] == field)) {
    ++m;
  }
  if (m == plan->uci_nmsg) {
    return set_error(ctx, PG_ERR_INVALID, "the UE carries no such UCI message");
  }
  const size_t nbits = plan->uci_msg_nbits[m];
  if (len < nbits) {
    return set_error(ctx, PG_ERR_INVALID, "bit buffer shorter than the message");
  }
  const uint8_t* src = (m < plan->uci_nshort ? plan->d_uci_bits : plan->d_polar_bits) + plan->uci_msg_off[m];
  int            rc  = check_cuda(ctx, cudaMemcpy(bits, src, nbits, cudaMemcpyDeviceToHost), "D2H UCI message");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpy(valid, plan->d_uci_valid + m, 1, cudaMemcpyDeviceToHost), "D2H UCI validity");
  }
  return rc;
}

int pg_pusch_plan_set_harq(pg_pusch_plan* plan, const uint8_t* new_data, const uint8_t* rv)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  for (int u = 0; u < plan->nof_ues && rv != nullptr; ++u) {
    if (rv[u] > 3) {
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(u) + ": redundancy version above 3");
    }
  }
  for (int u = 0; u < plan->nof_ues; ++u) {
    if (rv != nullptr) {
      plan->ues[u].rv = rv[u];
    }
    for (int c = plan->tb_first[u]; c < plan->tb_first[u] + plan->tb_ncb[u]; ++c) {
      if (rv != nullptr) {
        plan->rm[c].rv = rv[u];
      }
      if (new_data != nullptr) {
        plan->rm[c].new_data = new_data[u] != 0 ? 1 : 0;
      }
    }
  }
  // Soft combining (new_data == 0) takes a UE off the fused demodulation and rate dematching.
  build_direct(plan->ues, plan->rm, plan->tb_first, plan->tb_ncb, plan->direct, plan->placed);
  std::vector<uint32_t> unplaced = unplaced_list(plan->placed);
  if (unplaced.size() != plan->unplaced.size() && plan->exec != nullptr) {
    // The rate-dematch launch changes shape: the next execution captures a new graph.
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  plan->unplaced = unplaced;
  // Otherwise the kernels read the descriptors when they run, so a captured graph stays valid.
  cudaStream_t s  = ctx->stream;
  int          rc = check_cuda(ctx,
                               cudaMemcpyAsync(plan->d_rm, plan->rm.data(), plan->rm.size() * sizeof(pg_rm_cb),
                                               cudaMemcpyHostToDevice, s),
                               "H2D HARQ rate-dematch descriptors");
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(plan->d_direct, plan->direct.data(), plan->direct.size() * sizeof(rm_direct),
                                    cudaMemcpyHostToDevice, s),
                    "H2D HARQ demodulator placement");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(plan->d_placed, plan->placed.data(), plan->placed.size(), cudaMemcpyHostToDevice, s),
                    "H2D HARQ in-place flags");
  }
  if (rc == PG_OK && !plan->unplaced.empty()) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(plan->d_unplaced, plan->unplaced.data(), plan->unplaced.size() * 4,
                                    cudaMemcpyHostToDevice, s),
                    "H2D HARQ rate-dematch list");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(plan->d_ues, plan->ues.data(), plan->ues.size() * sizeof(pg_pusch_ue),
                                    cudaMemcpyHostToDevice, s),
                    "H2D HARQ UE descriptors");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

static bool tuning_valid(const pg_pusch_plan_tuning& t, const pg_context* ctx)
{
  return t.rm_ctas_per_cb >= 1 && t.rm_ctas_per_cb <= 32 && t.demod_res_per_thread >= 1 &&
         t.demod_res_per_thread <= 8 && (t.demod_block == 64 || t.demod_block == 128 || t.demod_block == 256) &&
         t.ldpc_ctas_per_sm >= 1 && t.ldpc_ctas_per_sm <= 4 &&
         t.ldpc_kernel >= PG_LDPC_KERNEL_ONE_LANE && t.ldpc_kernel <= PG_LDPC_KERNEL_Z384_SPLIT &&
         (t.ldpc_order == 0 || t.ldpc_order == 1);
}

int pg_pusch_plan_get_tuning(const pg_pusch_plan* plan, pg_pusch_plan_tuning* out)
{
  if (plan == nullptr || out == nullptr) {
    return PG_ERR_INVALID;
  }
  *out = plan->tuning;
  return PG_OK;
}

int pg_pusch_plan_set_tuning(pg_pusch_plan* plan, const pg_pusch_plan_tuning* t)
{
  if (plan == nullptr || t == nullptr) {
    return PG_ERR_INVALID;
  }
  if (!tuning_valid(*t, plan->ctx)) {
    return set_error(plan->ctx, PG_ERR_INVALID, "launch shapes out of range");
  }
  if (int rc = check_cuda(plan->ctx, cudaStreamSynchronize(plan->ctx->stream), "cudaStreamSynchronize")) {
    return rc;
  }
  plan->tuning = *t;
  if (plan->exec != nullptr) {
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  return PG_OK;
}

// Device time of `reps` executions (enqueued directly, no graph) with the plan's current shapes:
// the minimum over the repetitions, after one untimed execution.
static int time_plan(pg_pusch_plan* p, const uint32_t* grids, uint8_t* tb, pg_sch_result* res, int reps, float* best)
{
  pg_context*  ctx = p->ctx;
  cudaStream_t s   = ctx->stream;
  cudaEvent_t  a = nullptr, b = nullptr;
  int          rc = check_cuda(ctx, cudaEventCreate(&a), "cudaEventCreate");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreate(&b), "cudaEventCreate");
  }
  const bool timed = ctx->timed;
  ctx->timed       = false;
  *best            = 1e30f;
  for (int r = -1; r < reps && rc == PG_OK; ++r) {
    rc = check_cuda(ctx, cudaEventRecord(a, s), "cudaEventRecord");
    if (rc == PG_OK) {
      rc = enqueue(p, grids, tb, res, p->d_pr, s);
    }
    if (rc == PG_OK) {
      rc = check_cuda(ctx, cudaEventRecord(b, s), "cudaEventRecord");
    }
    if (rc == PG_OK) {
      rc = check_cuda(ctx, cudaEventSynchronize(b), "cudaEventSynchronize");
    }
    float ms = 0.f;
    if (rc == PG_OK && r >= 0 && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
      *best = std::min(*best, ms);
    }
  }
  ctx->timed = timed;
  if (a) {
    cudaEventDestroy(a);
  }
  if (b) {
    cudaEventDestroy(b);
  }
  return rc;
}

int pg_pusch_plan_autotune(pg_pusch_plan* plan, const uint32_t* grids, int reps, pg_pusch_plan_tuning* best_out,
                           float* best_ms)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (grids == nullptr || reps < 1) {
    return set_error(ctx, PG_ERR_INVALID, "autotune: null grids or no repetitions");
  }
  // Candidate shapes per stage; coordinate descent over the stages, two passes, each candidate
  // timed on the plan's own slot (the outputs land in the plan's execute_host buffers).
  static const int rm_c[]    = {2, 4, 8, 16, 32};
  static const int res_c[]   = {1, 2, 4};
  static const int blk_c[]   = {64, 128, 256};
  static const int ldpc_c[]  = {1, 2, 3, 4};
  pg_pusch_plan_tuning cur   = plan->tuning;
  float                cur_ms = 0.f;
  // UEs set to combine would accumulate every timed execution into their soft buffers: keep a
  // copy of the buffers and put it back afterwards.
  bool combining = false;
  for (const pg_rm_cb& c : plan->rm) {
    combining = combining || c.new_data == 0;
  }
  int8_t* saved = nullptr;
  int     rc    = PG_OK;
  if (combining) {
    rc = check_cuda(ctx, cudaMalloc(&saved, plan->rm_total), "cudaMalloc(soft-buffer copy)");
    if (rc == PG_OK) {
      rc = check_cuda(ctx,
                      cudaMemcpyAsync(saved, plan->d_rm_out, plan->rm_total, cudaMemcpyDeviceToDevice, ctx->stream),
                      "D2D soft buffers");
    }
    if (rc != PG_OK) {
      cudaFree(saved);
      return rc;
    }
  }
  rc = time_plan(plan, grids, plan->d_tb_out, plan->d_res, reps, &cur_ms);
  auto try_set = [&](pg_pusch_plan_tuning cand) -> int {
    if (!tuning_valid(cand, ctx)) {
      return PG_OK;
    }
    const pg_pusch_plan_tuning keep = plan->tuning;
    plan->tuning                    = cand;
    float ms                        = 0.f;
    const int r                     = time_plan(plan, grids, plan->d_tb_out, plan->d_res, reps, &ms);
    if (r == PG_OK && ms < cur_ms) {
      cur_ms = ms;
      cur    = cand;
    }
    plan->tuning = keep;
    return r;
  };
  for (int pass = 0; pass < 2 && rc == PG_OK; ++pass) {
    for (int v : rm_c) {
      pg_pusch_plan_tuning c = cur;
      c.rm_ctas_per_cb       = v;
      if (rc == PG_OK) rc = try_set(c);
    }
    for (int v : res_c) {
      pg_pusch_plan_tuning c = cur;
      c.demod_res_per_thread = v;
      if (rc == PG_OK) rc = try_set(c);
    }
    for (int v : blk_c) {
      pg_pusch_plan_tuning c = cur;
      c.demod_block          = v;
      if (rc == PG_OK) rc = try_set(c);
    }
    for (int v : ldpc_c) {
      pg_pusch_plan_tuning c = cur;
      c.ldpc_ctas_per_sm     = v;
      if (rc == PG_OK) rc = try_set(c);
    }
    for (int v : {PG_LDPC_KERNEL_ONE_LANE, PG_LDPC_KERNEL_TWO_LANES, PG_LDPC_KERNEL_SPLIT, PG_LDPC_KERNEL_Z384,
                  PG_LDPC_KERNEL_Z384_SPLIT}) {
      pg_pusch_plan_tuning c = cur;
      c.ldpc_kernel          = v;
      if (rc == PG_OK) rc = try_set(c);
    }
    for (int v : {0, 1}) {
      pg_pusch_plan_tuning c = cur;
      c.ldpc_order           = v;
      if (rc == PG_OK) rc = try_set(c);
    }
  }
  if (saved != nullptr) {
    const int r = check_cuda(
      ctx, cudaMemcpyAsync(plan->d_rm_out, saved, plan->rm_total, cudaMemcpyDeviceToDevice, ctx->stream),
      "D2D soft buffers");
    const int r2 = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
    cudaFree(saved);
    rc = rc != PG_OK ? rc : (r != PG_OK ? r : r2);
  }
  if (rc != PG_OK) {
    return rc;
  }
  plan->tuning = cur;
  if (plan->exec != nullptr) {
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  if (best_out != nullptr) {
    *best_out = cur;
  }
  if (best_ms != nullptr) {
    *best_ms = cur_ms;
  }
  return PG_OK;
}

int pg_pusch_plan_execute_device(pg_pusch_plan* plan, const uint32_t* grids, uint8_t* tb_out, pg_sch_result* results,
                                 pg_port_result* port_results, void* stream)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (grids == nullptr || tb_out == nullptr || results == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null device buffer");
  }
  pg_port_result* pr = port_results != nullptr ? port_results : plan->d_pr;
  cudaStream_t    s  = static_cast<cudaStream_t>(stream);
  if (!plan->use_graph || s == nullptr) {
    return enqueue(plan, grids, tb_out, results, pr, s);
  }
  const void* key[5] = {grids, tb_out, results, pr, stream};
  if (plan->exec == nullptr || !std::equal(key, key + 5, plan->key)) {
    if (plan->exec != nullptr) {
      cudaGraphExecDestroy(plan->exec);
      plan->exec = nullptr;
    }
    int rc = check_cuda(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    if (rc != PG_OK) {
      return rc;
    }
    const int   rc_enq = enqueue(plan, grids, tb_out, results, pr, s);
    cudaGraph_t graph  = nullptr;
    rc                 = check_cuda(ctx, cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture");
    if (rc_enq != PG_OK || rc != PG_OK) {
      if (graph != nullptr) {
        cudaGraphDestroy(graph);
      }
      return rc_enq != PG_OK ? rc_enq : rc;
    }
    rc = check_cuda(ctx, cudaGraphInstantiate(&plan->exec, graph, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(graph);
    if (rc != PG_OK) {
      plan->exec = nullptr;
      return rc;
    }
    std::copy(key, key + 5, plan->key);
  }
  return check_cuda(ctx, cudaGraphLaunch(plan->exec, s), "cudaGraphLaunch");
}

// The part of the host entries after the grids are on the device: the plan on plan->d_grid, the
// results and TBs back to the host.
static int execute_host_tail(pg_pusch_plan* plan, uint8_t* tb_out, pg_sch_result* results,
                             pg_port_result* port_results, int rc);

int pg_pusch_plan_execute_host(pg_pusch_plan* plan, const uint32_t* grids, uint8_t* tb_out, size_t tb_out_len,
                               pg_sch_result* results, pg_port_result* port_results)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (grids == nullptr || results == nullptr || (tb_out == nullptr && plan->tb_bytes > 0)) {
    return set_error(ctx, PG_ERR_INVALID, "null host buffer");
  }
  if (tb_out_len < plan->tb_bytes) {
    return set_error(ctx, PG_ERR_INVALID, "transport-block buffer smaller than the plan's TBs");
  }
  const int rc = copy_grid_spans(plan, plan->d_grid, grids, ctx->stream);
  return execute_host_tail(plan, tb_out, results, port_results, rc);
}

int pg_pusch_plan_execute_host_bfp(pg_pusch_plan* plan, const uint8_t* compressed, size_t compressed_len,
                                   int data_width, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results,
                                   pg_port_result* port_results)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (compressed == nullptr || results == nullptr || (tb_out == nullptr && plan->tb_bytes > 0)) {
    return set_error(ctx, PG_ERR_INVALID, "null host buffer");
  }
  if (tb_out_len < plan->tb_bytes) {
    return set_error(ctx, PG_ERR_INVALID, "transport-block buffer smaller than the plan's TBs");
  }
  if (data_width < 1 || data_width > 16) {
    return set_error(ctx, PG_ERR_INVALID, "BFP data width must be 1 to 16 bits");
  }
  if (plan->grid_words % 12 != 0) {
    return set_error(ctx, PG_ERR_INVALID, "the plan's grids are not whole PRBs");
  }
  const uint32_t nof_prb = (uint32_t)(plan->grid_words / 12);
  const size_t   bytes   = (size_t)nof_prb * (size_t)bfp_prb_bytes(data_width);
  if (compressed_len < bytes) {
    return set_error(ctx, PG_ERR_INVALID, "compressed grids shorter than the plan's PRBs (" + std::to_string(bytes) +
                                              " bytes)");
  }
  cudaStream_t s = ctx->stream;
  if (plan->d_bfp_cap < bytes) {
    if (int rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize")) {
      return rc;
    }
    cudaFree(plan->d_bfp);
    plan->d_bfp     = nullptr;
    plan->d_bfp_cap = 0;
    if (int rc = check_cuda(ctx, cudaMalloc(&plan->d_bfp, bytes), "cudaMalloc(compressed grids)")) {
      return rc;
    }
    plan->d_bfp_cap = bytes;
  }
  int rc = check_cuda(ctx, cudaMemcpyAsync(plan->d_bfp, compressed, bytes, cudaMemcpyHostToDevice, s),
                      "H2D compressed grids");
  if (rc == PG_OK) {
    rc = bfp_decompress_launch(ctx, plan->d_bfp, nof_prb, data_width, plan->d_grid, s);
  }
  return execute_host_tail(plan, tb_out, results, port_results, rc);
}

// Results of one slot from the pinned host buffer h (layout of plan->host) to the caller's buffers.
static void copy_results_out(const pg_pusch_plan* plan, const uint8_t* h, uint8_t* tb_out, pg_sch_result* results,
                             pg_port_result* port_results)
{
  const int             n    = plan->nof_ues;
  const pg_sch_result*  hres = reinterpret_cast<const pg_sch_result*>(h);
  const pg_port_result* hpr  = reinterpret_cast<const pg_port_result*>(h + al((size_t)n * sizeof(pg_sch_result)));
  const uint8_t*        htb  = h + al((size_t)n * sizeof(pg_sch_result)) + al((size_t)n * 4 * sizeof(pg_port_result));
  std::memcpy(results, hres, (size_t)n * sizeof(pg_sch_result));
  if (port_results != nullptr) {
    std::memcpy(port_results, hpr, (size_t)n * 4 * sizeof(pg_port_result));
  }
  // The reference writes a TB's payload only when its CRC passes.
  for (int i = 0; i < n; ++i) {
    if (hres[i].tb_crc_ok) {
      const pg_pusch_ue& u = plan->ues[i];
      std::memcpy(tb_out + u.tb_out_offset, htb + u.tb_out_offset, u.tbs_bits / 8);
    }
  }
}

// D2H of one slot's results, port results and TBs into the pinned host buffer h.
static int enqueue_results_d2h(pg_pusch_plan* plan, uint8_t* h, cudaStream_t s)
{
  pg_context* ctx = plan->ctx;
  const int   n   = plan->nof_ues;
  uint8_t*    hpr = h + al((size_t)n * sizeof(pg_sch_result));
  uint8_t*    htb = hpr + al((size_t)n * 4 * sizeof(pg_port_result));
  int rc = check_cuda(ctx, cudaMemcpyAsync(h, plan->d_res, (size_t)n * sizeof(pg_sch_result), cudaMemcpyDeviceToHost, s),
                      "D2H results");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(hpr, plan->d_pr, (size_t)n * 4 * sizeof(pg_port_result), cudaMemcpyDeviceToHost, s),
                    "D2H port results");
  }
  if (rc == PG_OK && plan->tb_bytes > 0) {
    rc = check_cuda(ctx, cudaMemcpyAsync(htb, plan->d_tb_out, plan->tb_bytes, cudaMemcpyDeviceToHost, s), "D2H TBs");
  }
  return rc;
}

// Host grids to a device grid buffer of the plan's layout: one 2-D copy per cell span.
static int copy_grid_spans(pg_pusch_plan* plan, uint32_t* dst, const uint32_t* src, cudaStream_t s)
{
  for (const grid_span& g : plan->grid_spans) {
    if (int rc = check_cuda(plan->ctx,
                            cudaMemcpy2DAsync(dst + g.offset, g.pitch * 4, src + g.offset, g.pitch * 4, g.width * 4,
                                              g.rows, cudaMemcpyHostToDevice, s),
                            "H2D grids")) {
      return rc;
    }
  }
  return PG_OK;
}

int pg_pusch_plan_submit_host(pg_pusch_plan* plan, const uint32_t* grids)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (grids == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null host buffer");
  }
  if (plan->submitted - plan->collected >= (uint64_t)kPlanInFlight) {
    return set_error(ctx, PG_ERR_INVALID, "three slots in flight: collect one before submitting another");
  }
  const size_t grid_bytes = plan->grid_words * 4;
  const size_t n          = (size_t)plan->nof_ues;
  const size_t h_bytes    = al(n * sizeof(pg_sch_result)) + al(n * 4 * sizeof(pg_port_result)) + al(plan->tb_bytes);
  int          rc         = PG_OK;
  if (plan->copy_stream == nullptr) {
    rc = check_cuda(ctx, cudaStreamCreateWithFlags(&plan->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (cudaEvent_t* e : {&plan->ev_h2d, &plan->ev_stage_free[0], &plan->ev_stage_free[1], &plan->ev_done[0],
                           &plan->ev_done[1], &plan->ev_done[2]}) {
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
      }
    }
    for (uint32_t** d : {&plan->d_stage[0], &plan->d_stage[1]}) {
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(d), std::max<size_t>(grid_bytes, 4)),
                        "cudaMalloc(staging grids)");
      }
    }
    for (void** h : {&plan->host_slot[0], &plan->host_slot[1], &plan->host_slot[2]}) {
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaMallocHost(h, std::max<size_t>(h_bytes, 64)), "cudaMallocHost(result slot)");
      }
    }
    if (rc != PG_OK) {
      return rc;
    }
  }
  cudaStream_t s    = ctx->stream;
  const int    slot  = (int)(plan->submitted % (uint64_t)kPlanInFlight);
  const int    stage = (int)(plan->submitted & 1u);
  // Copy stream: a staging buffer is free once the slot two submissions back has moved it into the
  // grid buffer; the H2D then overlaps whatever the compute stream runs, up to two slots ahead.
  rc = check_cuda(ctx, cudaStreamWaitEvent(plan->copy_stream, plan->ev_stage_free[stage], 0), "cudaStreamWaitEvent");
  if (rc == PG_OK) {
    rc = copy_grid_spans(plan, plan->d_stage[stage], grids, plan->copy_stream);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventRecord(plan->ev_h2d, plan->copy_stream), "cudaEventRecord");
  }
  // Compute stream: the grids into the plan's grid buffer (after the previous slot's plan, same
  // stream), the plan, the results back.
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamWaitEvent(s, plan->ev_h2d, 0), "cudaStreamWaitEvent");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(plan->d_grid, plan->d_stage[stage], grid_bytes, cudaMemcpyDeviceToDevice, s),
                    "D2D grids");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventRecord(plan->ev_stage_free[stage], s), "cudaEventRecord");
  }
  if (rc == PG_OK) {
    rc = pg_pusch_plan_execute_device(plan, plan->d_grid, plan->d_tb_out, plan->d_res, plan->d_pr, s);
  }
  if (rc == PG_OK) {
    rc = enqueue_results_d2h(plan, static_cast<uint8_t*>(plan->host_slot[slot]), s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventRecord(plan->ev_done[slot], s), "cudaEventRecord");
  }
  if (rc == PG_OK) {
    ++plan->submitted;
  }
  return rc;
}

int pg_pusch_plan_collect_host(pg_pusch_plan* plan, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results,
                               pg_port_result* port_results)
{
  if (plan == nullptr) {
    return PG_ERR_INVALID;
  }
  pg_context* ctx = plan->ctx;
  if (results == nullptr || (tb_out == nullptr && plan->tb_bytes > 0)) {
    return set_error(ctx, PG_ERR_INVALID, "null host buffer");
  }
  if (tb_out_len < plan->tb_bytes) {
    return set_error(ctx, PG_ERR_INVALID, "transport-block buffer smaller than the plan's TBs");
  }
  if (plan->collected == plan->submitted) {
    return set_error(ctx, PG_ERR_INVALID, "no slot submitted");
  }
  const int slot = (int)(plan->collected % (uint64_t)kPlanInFlight);
  if (int rc = check_cuda(ctx, cudaEventSynchronize(plan->ev_done[slot]), "cudaEventSynchronize")) {
    return rc;
  }
  copy_results_out(plan, static_cast<const uint8_t*>(plan->host_slot[slot]), tb_out, results, port_results);
  ++plan->collected;
  return PG_OK;
}

static int execute_host_tail(pg_pusch_plan* plan, uint8_t* tb_out, pg_sch_result* results,
                             pg_port_result* port_results, int rc)
{
  pg_context*     ctx  = plan->ctx;
  const int       n    = plan->nof_ues;
  cudaStream_t    s    = ctx->stream;
  uint8_t*        h    = static_cast<uint8_t*>(plan->host);
  pg_sch_result*  hres = reinterpret_cast<pg_sch_result*>(h);
  pg_port_result* hpr  = reinterpret_cast<pg_port_result*>(h + al((size_t)n * sizeof(pg_sch_result)));
  uint8_t*        htb  = h + al((size_t)n * sizeof(pg_sch_result)) + al((size_t)n * 4 * sizeof(pg_port_result));
  if (rc == PG_OK) {
    rc = pg_pusch_plan_execute_device(plan, plan->d_grid, plan->d_tb_out, plan->d_res, plan->d_pr, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(hres, plan->d_res, (size_t)n * sizeof(pg_sch_result), cudaMemcpyDeviceToHost, s),
                    "D2H results");
  }
  if (rc == PG_OK && port_results != nullptr) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(hpr, plan->d_pr, (size_t)n * 4 * sizeof(pg_port_result), cudaMemcpyDeviceToHost, s),
                    "D2H port results");
  }
  if (rc == PG_OK && plan->tb_bytes > 0) {
    rc = check_cuda(ctx, cudaMemcpyAsync(htb, plan->d_tb_out, plan->tb_bytes, cudaMemcpyDeviceToHost, s), "D2H TBs");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  if (rc != PG_OK) {
    return rc;
  }
  std::memcpy(results, hres, (size_t)n * sizeof(pg_sch_result));
  if (port_results != nullptr) {
    std::memcpy(port_results, hpr, (size_t)n * 4 * sizeof(pg_port_result));
  }
  // The reference writes a TB's payload only when its CRC passes.
  for (int i = 0; i < n; ++i) {
    if (hres[i].tb_crc_ok) {
      const pg_pusch_ue& u = plan->ues[i];
      std::memcpy(tb_out + u.tb_out_offset, htb + u.tb_out_offset, u.tbs_bits / 8);
    }
  }
  return PG_OK;
}

} // extern "C"

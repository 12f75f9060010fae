// C ABI of the PUSCH slot entry points: demodulation and the whole receive path.
#include "pg_internal.h"

#include <algorithm>
#include <vector>

using namespace pg;

namespace {

struct slot_layout {
  std::vector<pg_pusch_ue> ues;
  std::vector<uint32_t>    seq_off;
  std::vector<uint32_t>    offs; // [seq offsets (n) | demodulation tile offsets (n + 1)]
  size_t                   est_total = 0, llr_total = 0, seq_total = 0;
  uint32_t                 max_words = 0, total_tiles = 0;
};

// Assigns est/llr offsets and scrambling-sequence offsets.
void plan(const pg_pusch_ue* ues, int n, slot_layout& L, bool assign_offsets)
{
  L.ues.assign(ues, ues + n);
  L.seq_off.resize(n);
  for (int i = 0; i < n; ++i) {
    pg_pusch_ue&   u = L.ues[i];
    const uint32_t g = ue_codeword_bits(u);
    if (assign_offsets) {
      u.est_offset = (uint32_t)L.est_total;
      L.llr_total  = (L.llr_total + 15) & ~(size_t)15; // 16-byte aligned codewords: vector LLR stores
      u.llr_offset = (uint32_t)L.llr_total;
    }
    L.est_total += pg_pusch_est_size(&u);
    L.llr_total = std::max(L.llr_total, (size_t)u.llr_offset + g);
    L.seq_off[i] = (uint32_t)L.seq_total;
    const uint32_t words = (g + 31) / 32 + 2;
    L.seq_total += words;
    L.max_words = std::max(L.max_words, words);
  }
  // [sequence offsets (n) | demodulation tile map]
  L.offs.assign(L.seq_off.begin(), L.seq_off.end());
  L.total_tiles = demod_tile_map(L.ues.data(), n, L.offs);
}

} // namespace

extern "C" {

int pg_descramble_device(pg_context* ctx, uint32_t c_init, const int8_t* llrs_in, int8_t* llrs_out, size_t n,
                         void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (n > 0 && (llrs_in == nullptr || llrs_out == nullptr)) {
    return set_error(ctx, PG_ERR_INVALID, "null soft-bit buffer");
  }
  return descramble_launch(ctx, c_init, llrs_in, llrs_out, n, static_cast<cudaStream_t>(stream));
}

int pg_descramble_host(pg_context* ctx, uint32_t c_init, const int8_t* llrs_in, int8_t* llrs_out, size_t n)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (n == 0) {
    return PG_OK;
  }
  if (llrs_in == nullptr || llrs_out == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null soft-bit buffer");
  }
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(n, 256), "cudaMalloc(descramble)");
  }
  int8_t*      d = static_cast<int8_t*>(ctx->scratch_a);
  cudaStream_t s = ctx->stream;
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(d, llrs_in, n, cudaMemcpyHostToDevice, s), "H2D soft bits");
  }
  if (rc == PG_OK) {
    rc = descramble_launch(ctx, c_init, d, d, n, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(llrs_out, d, n, cudaMemcpyDeviceToHost, s), "D2H soft bits");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

int pg_pusch_demodulate_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                               const float* est, const pg_port_result* port_results, int8_t* llrs, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ues(ctx, ues, nof_ues)) {
    return rc;
  }
  if (nof_ues == 0) {
    return PG_OK;
  }
  slot_layout L;
  plan(ues, nof_ues, L, false);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Scratch: [sequence offsets | demodulation tile map | sequences].
  const size_t noffs = L.offs.size();
  const size_t bytes = 256 + noffs * 4 + L.seq_total * 4;
  if (int rc = ensure_scratch(ctx, &ctx->scratch_b, &ctx->scratch_b_cap, bytes, "cudaMalloc(demod scratch)")) {
    return rc;
  }
  uint32_t* d_off = static_cast<uint32_t*>(ctx->scratch_b);
  uint32_t* d_seq = d_off + ((noffs + 63) / 64) * 64;
  void*     d_ues = nullptr;
  int       rc    = check_cuda(ctx, cudaMemcpyAsync(d_off, L.offs.data(), noffs * 4, cudaMemcpyHostToDevice, s),
                               "cudaMemcpyAsync(offsets)");
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_UE, L.ues.data(), (size_t)nof_ues * sizeof(pg_pusch_ue), s, &d_ues);
  }
  if (rc == PG_OK) {
    rc = demod_launch(ctx, static_cast<const pg_pusch_ue*>(d_ues), nof_ues, L.max_words, L.total_tiles,
                      d_off + nof_ues, grids, est, port_results, d_off, d_seq, llrs, s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_UE, s);
  }
  if (rc == PG_OK) {
    // The offsets were copied from a host vector that goes out of scope.
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

int pg_pusch_process_host(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                          size_t grid_words, uint8_t* tb_out, size_t tb_out_len, pg_port_result* port_results,
                          pg_sch_result* results)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ues(ctx, ues, nof_ues)) {
    return rc;
  }
  if (nof_ues == 0) {
    return PG_OK;
  }
  if (grids == nullptr || results == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null buffer");
  }
  slot_layout L;
  plan(ues, nof_ues, L, true);
  for (int i = 0; i < nof_ues; ++i) {
    const pg_pusch_ue& u = L.ues[i];
    if ((size_t)u.grid_offset + (size_t)u.nof_rx_ports * 14 * u.grid_nof_subc > grid_words) {
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(i) + ": grid beyond the buffer");
    }
  }
  auto         al     = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_grid = 0;
  const size_t o_est  = o_grid + al(grid_words * 4);
  const size_t o_pr   = o_est + al(L.est_total * 8);
  const size_t o_off  = o_pr + al((size_t)nof_ues * 4 * sizeof(pg_port_result));
  const size_t o_seq  = o_off + al(L.offs.size() * 4);
  const size_t o_llr  = o_seq + al(L.seq_total * 4);
  const size_t total  = o_llr + al(L.llr_total);
  cudaStream_t s      = ctx->stream;
  int          rc     = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, total, "cudaMalloc(slot scratch)");
  }
  if (rc != PG_OK) {
    return rc;
  }
  uint8_t*        b     = static_cast<uint8_t*>(ctx->scratch_a);
  uint32_t*       d_grid = reinterpret_cast<uint32_t*>(b + o_grid);
  float*          d_est  = reinterpret_cast<float*>(b + o_est);
  pg_port_result* d_pr   = reinterpret_cast<pg_port_result*>(b + o_pr);
  uint32_t*       d_off  = reinterpret_cast<uint32_t*>(b + o_off);
  uint32_t*       d_seq  = reinterpret_cast<uint32_t*>(b + o_seq);
  int8_t*         d_llr  = reinterpret_cast<int8_t*>(b + o_llr);
  rc = check_cuda(ctx, cudaMemcpyAsync(d_grid, grids, grid_words * 4, cudaMemcpyHostToDevice, s), "H2D grids");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(d_off, L.offs.data(), L.offs.size() * 4, cudaMemcpyHostToDevice, s),
                    "H2D offsets");
  }
  if (rc == PG_OK) {
    rc = estimate_launch_host(ctx, L.ues.data(), nof_ues, d_grid, d_est, nullptr, d_pr, s);
  }
  void* d_ues = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_UE, L.ues.data(), (size_t)nof_ues * sizeof(pg_pusch_ue), s, &d_ues);
  }
  if (rc == PG_OK) {
    rc = demod_launch(ctx, static_cast<const pg_pusch_ue*>(d_ues), nof_ues, L.max_words, L.total_tiles, d_off + nof_ues,
                      d_grid, d_est, d_pr, d_off, d_seq, d_llr, s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_UE, s);
  }
  std::vector<pg_sch_tb> tbs(nof_ues);
  for (int i = 0; i < nof_ues; ++i) {
    const pg_pusch_ue& u = L.ues[i];
    pg_sch_tb&         t = tbs[i];
    t                    = pg_sch_tb{};
    t.llr_offset         = u.llr_offset;
    t.nof_ch_symbols     = ue_codeword_bits(u) / u.modulation_order;
    t.tbs_bits           = u.tbs_bits;
    t.tb_out_offset      = u.tb_out_offset;
    t.nref               = u.nref;
    t.base_graph         = u.base_graph;
    t.modulation_order   = u.modulation_order;
    t.nof_layers         = u.nof_layers;
    t.rv                 = u.rv;
    t.max_iterations     = u.max_iterations;
  }
  if (rc == PG_OK) {
    rc = sch_decode_device_llrs(ctx, tbs.data(), nof_ues, d_llr, L.llr_total, tb_out, tb_out_len, results);
  }
  if (rc == PG_OK && port_results != nullptr) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(port_results, d_pr, (size_t)nof_ues * 4 * sizeof(pg_port_result),
                                    cudaMemcpyDeviceToHost, s),
                    "D2H port results");
    if (rc == PG_OK) {
      rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
  }
  return rc;
}

} // extern "C"

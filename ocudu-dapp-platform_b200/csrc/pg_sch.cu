// C ABI of the rate-dematching, CRC, TB-assembly and TB-decoding entry points, and the UL-SCH
// segmentation (host code).
#include "pg_internal.h"
#include "pg_device.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace {

// Descrambling of n soft bits: out[i] = -in[i] where c(bit_offset + i) = 1 (TS 38.211 Section 6.3.1.1,
// the Gold sequence of Section 5.2.1 with initialisation c_init), one 32-bit sequence word per thread.
__global__ void descramble_kernel(const int8_t* __restrict__ in, int8_t* __restrict__ out, uint32_t n, uint32_t c_init,
                                  uint32_t bit_offset, const uint32_t* __restrict__ gold, uint32_t gold_words)
{
  const uint32_t words = (n + 31) / 32;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    const uint32_t seq = pg::gold_word(gold, gold_words, c_init, bit_offset + 32u * w);
#pragma unroll 4
    for (uint32_t b = 0; b < 32; ++b) {
      const uint32_t k = 32u * w + b;
      if (k < n) {
        const int v = in[k];
        out[k]      = (int8_t)(((seq >> b) & 1u) ? -v : v);
      }
    }
  }
}

} // namespace

namespace pg {

static const int kLiftingSizes[51] = {2,  3,  4,  5,  6,  7,   8,   9,   10,  11,  12,  13,  14,  15,  16,  18,  20,
                                      22, 24, 26, 28, 30, 32,  36,  40,  44,  48,  52,  56,  60,  64,  72,  80,  88,
                                      96, 104, 112, 120, 128, 144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};

// TS 38.212 Section 5.2.2 code block segmentation with the reference's rounding
// (include/ocudu/ran/sch/sch_segmentation.h:40-118,
//  lib/phy/upper/channel_coding/ldpc/ldpc_segmenter_rx_impl.cpp:33-85 and
//  lib/phy/upper/channel_coding/ldpc/ldpc_segmenter_helpers.h:63-95).
int segment(uint32_t tbs, int bg, int qm, int layers, uint32_t nof_ch_symbols, pg_sch_segmentation* o)
{
  if ((bg != 1 && bg != 2) || tbs == 0 || layers < 1 || layers > 4 || !(qm == 1 || qm == 2 || qm == 4 || qm == 6 || qm == 8)) {
    return PG_ERR_INVALID;
  }
  const uint32_t tb_crc = tbs <= 3824 ? 16 : 24;
  const uint32_t b      = tbs + tb_crc;
  const uint32_t kcb    = bg == 1 ? 8448 : 3840;
  const uint32_t c      = b <= kcb ? 1 : (b + (kcb - 24) - 1) / (kcb - 24);
  const uint32_t l      = c > 1 ? 24 : 0;
  const uint32_t bout   = b + c * l;
  uint32_t       kb     = 22;
  if (bg == 2) {
    kb = b > 640 ? 10 : (b > 560 ? 9 : (b > 192 ? 8 : 6));
  }
  uint32_t z = 0;
  for (int ls : kLiftingSizes) {
    if ((uint32_t)ls * c * kb >= bout) {
      z = ls;
      break;
    }
  }
  if (z == 0) {
    return PG_ERR_INVALID;
  }
  const uint32_t k        = (bg == 1 ? 22 : 10) * z;
  const uint32_t max_info = (bout + c - 1) / c - l;
  if (layers == 0 || nof_ch_symbols % (uint32_t)layers != 0) {
    return PG_ERR_INVALID;
  }
  const uint32_t per_layer = nof_ch_symbols / layers;
  o->nof_cbs               = c;
  o->lifting_size          = z;
  o->cb_length             = k;
  o->nof_filler_bits       = k - (max_info + l);
  o->cb_crc_bits           = l;
  o->tb_crc_bits           = tb_crc;
  o->nof_short_cbs         = c - (per_layer % c);
  o->e_short               = (per_layer / c) * layers * qm;
  o->e_long                = ((per_layer + c - 1) / c) * layers * qm;
  return PG_OK;
}

} // namespace pg

using namespace pg;

extern "C" {

int pg_sch_segment(uint32_t tbs_bits, int base_graph, int modulation_order, int nof_layers, uint32_t nof_ch_symbols,
                   pg_sch_segmentation* out)
{
  if (out == nullptr) {
    return PG_ERR_INVALID;
  }
  return segment(tbs_bits, base_graph, modulation_order, nof_layers, nof_ch_symbols, out);
}

int pg_rate_dematch_batch_device(pg_context* ctx, const pg_rm_cb* cbs, int nof_cbs, const int8_t* in, int8_t* out,
                                 void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_rm_descs(ctx, cbs, nof_cbs, 0, 0)) {
    return rc;
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  void*        dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_RM, cbs, (size_t)nof_cbs * sizeof(pg_rm_cb), s, &dev)) {
    return rc;
  }
  if (int rc = rate_dematch_launch(ctx, static_cast<const pg_rm_cb*>(dev), nof_cbs, in, out, s)) {
    return rc;
  }
  return release_slot_after(ctx, SLOT_RM, s);
}

int pg_rate_dematch_batch_host(pg_context* ctx, const pg_rm_cb* cbs, int nof_cbs, const int8_t* in, size_t in_len,
                               int8_t* out, size_t out_len)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_rm_descs(ctx, cbs, nof_cbs, in_len, out_len)) {
    return rc;
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  cudaStream_t s = ctx->stream;
  void*        d_in  = nullptr;
  void*        d_out = nullptr;
  int          rc    = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, in_len, "cudaMalloc(rm input)");
  }
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_b, &ctx->scratch_b_cap, out_len, "cudaMalloc(rm output)");
  }
  if (rc != PG_OK) {
    return rc;
  }
  d_in  = ctx->scratch_a;
  d_out = ctx->scratch_b;
  rc    = check_cuda(ctx, cudaMemcpyAsync(d_in, in, in_len, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(in)");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(d_out, out, out_len, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(out)");
  }
  void* dev = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_RM, cbs, (size_t)nof_cbs * sizeof(pg_rm_cb), s, &dev);
  }
  if (rc == PG_OK) {
    rc = rate_dematch_launch(ctx, static_cast<const pg_rm_cb*>(dev), nof_cbs, static_cast<const int8_t*>(d_in),
                             static_cast<int8_t*>(d_out), s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_RM, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(out, d_out, out_len, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync(out)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

static int validate_crc_items(pg_context* ctx, const pg_crc_item* items, int n, size_t data_len)
{
  if (n < 0 || (n > 0 && items == nullptr)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid CRC item list");
  }
  for (int i = 0; i < n; ++i) {
    if (items[i].poly > PG_CRC24B) {
      return set_error(ctx, PG_ERR_INVALID, "CRC item " + std::to_string(i) + ": polynomial");
    }
    if (items[i].nof_bits > (1u << 21) - 64) {
      return set_error(ctx, PG_ERR_INVALID, "CRC item " + std::to_string(i) + ": longer than 2^21 bits");
    }
    if (data_len != 0 && ((size_t)items[i].bit_offset + items[i].nof_bits + 7) / 8 > data_len) {
      return set_error(ctx, PG_ERR_INVALID, "CRC item " + std::to_string(i) + ": beyond the buffer");
    }
  }
  return PG_OK;
}

int pg_crc_calculate_device(pg_context* ctx, const pg_crc_item* items, int nof_items, const uint8_t* data,
                            uint32_t* crcs, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_crc_items(ctx, items, nof_items, 0)) {
    return rc;
  }
  if (nof_items == 0) {
    return PG_OK;
  }
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  void*        dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_CRC, items, (size_t)nof_items * sizeof(pg_crc_item), s, &dev)) {
    return rc;
  }
  if (int rc = crc_launch(ctx, static_cast<const pg_crc_item*>(dev), nof_items, data, crcs, s)) {
    return rc;
  }
  return release_slot_after(ctx, SLOT_CRC, s);
}

int pg_crc_calculate_host(pg_context* ctx, const pg_crc_item* items, int nof_items, const uint8_t* data,
                          size_t data_len, uint32_t* crcs)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_crc_items(ctx, items, nof_items, data_len)) {
    return rc;
  }
  if (nof_items == 0) {
    return PG_OK;
  }
  cudaStream_t s  = ctx->stream;
  int          rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(data_len, 1), "cudaMalloc(crc data)");
  }
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_b, &ctx->scratch_b_cap, (size_t)nof_items * 4, "cudaMalloc(crc out)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(ctx->scratch_a, data, data_len, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
  }
  void* dev = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_CRC, items, (size_t)nof_items * sizeof(pg_crc_item), s, &dev);
  }
  if (rc == PG_OK) {
    rc = crc_launch(ctx, static_cast<const pg_crc_item*>(dev), nof_items, static_cast<const uint8_t*>(ctx->scratch_a),
                    static_cast<uint32_t*>(ctx->scratch_b), s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_CRC, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(crcs, ctx->scratch_b, (size_t)nof_items * 4, cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

int pg_tb_assemble_device(pg_context* ctx, const pg_tb_desc* tbs, int nof_tbs, const uint8_t* cb_bits,
                          const uint32_t* cb_bit_offsets, uint8_t* tb_out, uint32_t* tb_crc, void* stream)
{
  if (ctx == nullptr || nof_tbs < 0 || (nof_tbs > 0 && tbs == nullptr)) {
    return PG_ERR_INVALID;
  }
  for (int i = 0; i < nof_tbs; ++i) {
    const pg_tb_desc& d = tbs[i];
    if (d.nof_cbs == 0 || d.cb_payload_bits == 0 || d.tbs_bits % 8 != 0 || d.crc_poly > PG_CRC24A ||
        (uint64_t)d.cb_payload_bits * d.nof_cbs < d.tbs_bits || (uint64_t)d.cb_payload_bits * d.nof_cbs > (1u << 21) - 64) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(i) + ": invalid sizes");
    }
  }
  if (nof_tbs == 0) {
    return PG_OK;
  }
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  void*        dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_TB, tbs, (size_t)nof_tbs * sizeof(pg_tb_desc), s, &dev)) {
    return rc;
  }
  if (int rc = tb_assemble_launch(ctx, static_cast<const pg_tb_desc*>(dev), nof_tbs, cb_bits, cb_bit_offsets, tb_out,
                                  tb_crc, s)) {
    return rc;
  }
  return release_slot_after(ctx, SLOT_TB, s);
}

int pg_sch_decode_batch_host(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* llrs,
                             size_t nof_llrs_total, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results)
{
  if (ctx == nullptr || nof_tbs < 0 || (nof_tbs > 0 && (tbs == nullptr || results == nullptr || llrs == nullptr))) {
    return ctx ? set_error(ctx, PG_ERR_INVALID, "invalid arguments") : PG_ERR_INVALID;
  }
  if (nof_tbs == 0) {
    return PG_OK;
  }
  if (int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
    return rc;
  }
  if (int rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(nof_llrs_total, 256),
                              "cudaMalloc(llrs)")) {
    return rc;
  }
  if (int rc = check_cuda(ctx, cudaMemcpyAsync(ctx->scratch_a, llrs, nof_llrs_total, cudaMemcpyHostToDevice, ctx->stream),
                          "cudaMemcpyAsync(llrs)")) {
    return rc;
  }
  return sch_decode_device_llrs(ctx, tbs, nof_tbs, static_cast<const int8_t*>(ctx->scratch_a), nof_llrs_total, tb_out,
                                tb_out_len, results);
}

int pg_sch_decode_batch_resident(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* llrs,
                                 size_t nof_llrs_total, const uint32_t* c_init, const uint32_t* bit_offset,
                                 uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results)
{
  if (ctx == nullptr || nof_tbs < 0 || (nof_tbs > 0 && (tbs == nullptr || results == nullptr || llrs == nullptr))) {
    return ctx ? set_error(ctx, PG_ERR_INVALID, "invalid arguments") : PG_ERR_INVALID;
  }
  if (nof_tbs == 0) {
    return PG_OK;
  }
  if (int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
    return rc;
  }
  const int8_t* d_llrs = llrs;
  if (c_init != nullptr) {
    // Descrambled copy of every TB's soft bits (the caller's buffer stays untouched).
    for (int t = 0; t < nof_tbs; ++t) {
      const uint64_t g   = (uint64_t)tbs[t].nof_ch_symbols * tbs[t].modulation_order;
      const uint64_t off = bit_offset != nullptr ? bit_offset[t] : 0;
      if (tbs[t].llr_offset + g > nof_llrs_total || off + g + 64 > 32ull * (kGoldWords - 2)) {
        return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": soft bits out of range");
      }
    }
    if (int rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(nof_llrs_total, 256),
                                "cudaMalloc(descrambled llrs)")) {
      return rc;
    }
    int8_t* d = static_cast<int8_t*>(ctx->scratch_a);
    for (int t = 0; t < nof_tbs; ++t) {
      const uint32_t g = tbs[t].nof_ch_symbols * tbs[t].modulation_order;
      descramble_kernel<<<(g / 32 + 255) / 256 + 1, 256, 0, ctx->stream>>>(
          llrs + tbs[t].llr_offset, d + tbs[t].llr_offset, g, c_init[t], bit_offset != nullptr ? bit_offset[t] : 0,
          ctx->dev.gold, kGoldWords);
      if (int rc = check_cuda(ctx, cudaGetLastError(), "descramble_kernel launch")) {
        return rc;
      }
    }
    d_llrs = d;
  }
  return sch_decode_device_llrs(ctx, tbs, nof_tbs, d_llrs, nof_llrs_total, tb_out, tb_out_len, results);
}

} // extern "C"

namespace pg {

int build_sch_work(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, size_t nof_llrs_total, size_t tb_out_len,
                   sch_work& w)
{
  // Work lists: one rate-dematch and one LDPC descriptor per codeblock, one TB descriptor per TB.
  w = sch_work();
  w.tb_first.resize(nof_tbs);
  w.tb_ncb.resize(nof_tbs);
  for (int t = 0; t < nof_tbs; ++t) {
    const pg_sch_tb&    tb = tbs[t];
    pg_sch_segmentation sg;
    if (segment(tb.tbs_bits, tb.base_graph, tb.modulation_order, tb.nof_layers, tb.nof_ch_symbols, &sg) != PG_OK ||
        tb.max_iterations == 0 || tb.tbs_bits % 8 != 0) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": invalid configuration");
    }
    const uint32_t tb_llrs = tb.nof_ch_symbols * tb.modulation_order;
    if ((size_t)tb.llr_offset + tb_llrs > nof_llrs_total) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": LLRs beyond the buffer");
    }
    if ((size_t)tb.tb_out_offset + tb.tbs_bits / 8 > tb_out_len) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": output beyond the buffer");
    }
    const uint32_t bout = tb.tbs_bits + sg.tb_crc_bits + sg.nof_cbs * sg.cb_crc_bits;
    if (bout % sg.nof_cbs != 0) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": TBS not segmentable evenly");
    }
    w.tb_first[t]    = (int)w.ldpc.size();
    w.tb_ncb[t]      = (int)sg.nof_cbs;
    const uint32_t N = (tb.base_graph == 1 ? 66 : 50) * sg.lifting_size;
    uint32_t       cw_off = 0;
    for (uint32_t c = 0; c < sg.nof_cbs; ++c) {
      const uint32_t e = c < sg.nof_short_cbs ? sg.e_short : sg.e_long;
      pg_rm_cb       r{};
      r.in_offset        = tb.llr_offset + cw_off;
      r.rm_length        = e;
      r.out_offset       = (uint32_t)w.rm_total;
      r.nref             = tb.nref;
      r.lifting_size     = (uint16_t)sg.lifting_size;
      r.nof_filler_bits  = (uint16_t)sg.nof_filler_bits;
      r.base_graph       = tb.base_graph;
      r.rv               = tb.rv;
      r.modulation_order = tb.modulation_order;
      r.new_data         = 1;
      w.rm.push_back(r);
      pg_ldpc_cb l{};
      l.llr_offset      = (uint32_t)w.rm_total;
      l.nof_llrs        = N;
      l.out_offset      = (uint32_t)w.bits_total;
      l.lifting_size    = (uint16_t)sg.lifting_size;
      l.nof_filler_bits = (uint16_t)sg.nof_filler_bits;
      l.base_graph      = tb.base_graph;
      l.crc_poly        = sg.nof_cbs > 1 ? PG_CRC24B : (tb.tbs_bits <= 3824 ? PG_CRC16 : PG_CRC24A);
      l.max_iterations  = tb.max_iterations;
      w.ldpc.push_back(l);
      w.cb_bit_off.push_back((uint32_t)(w.bits_total * 8));
      w.rm_total += (N + 15u) & ~15u; // 16-byte aligned codeblocks: vector loads in the decoder
      w.bits_total += (sg.cb_length + 7) / 8;
      cw_off += e;
    }
    if (cw_off != tb_llrs) {
      return set_error(ctx, PG_ERR_INVALID, "transport block " + std::to_string(t) + ": E_r do not sum to G");
    }
    pg_tb_desc d{};
    d.cb_first        = (uint32_t)w.tb_first[t];
    d.nof_cbs         = sg.nof_cbs;
    d.cb_payload_bits = bout / sg.nof_cbs - sg.cb_crc_bits;
    d.tbs_bits        = tb.tbs_bits;
    d.tb_out_offset   = tb.tb_out_offset;
    d.crc_poly        = tb.tbs_bits <= 3824 ? PG_CRC16 : PG_CRC24A;
    w.tbd.push_back(d);
  }
  return PG_OK;
}

int sch_decode_device_llrs(pg_context* ctx, const pg_sch_tb* tbs, int nof_tbs, const int8_t* d_llrs,
                           size_t nof_llrs_total, uint8_t* tb_out, size_t tb_out_len, pg_sch_result* results)
{
  sch_work w;
  if (int rc = build_sch_work(ctx, tbs, nof_tbs, nof_llrs_total, tb_out_len, w)) {
    return rc;
  }
  std::vector<pg_rm_cb>&   rm         = w.rm;
  std::vector<pg_ldpc_cb>& ldpc       = w.ldpc;
  std::vector<pg_tb_desc>& tbd        = w.tbd;
  std::vector<uint32_t>&   cb_bit_off = w.cb_bit_off;
  std::vector<int>&        tb_first   = w.tb_first;
  std::vector<int>&        tb_ncb     = w.tb_ncb;
  const size_t             rm_total   = w.rm_total;
  const size_t             bits_total = w.bits_total;
  const int ncb = (int)ldpc.size();
  if (ncb > ctx->max_codeblocks) {
    return set_error(ctx, PG_ERR_CAPACITY, "batch of " + std::to_string(ncb) + " codeblocks exceeds max_codeblocks");
  }
  if (nof_tbs == 0) {
    return PG_OK;
  }
  // Device buffers (scratch_b): [rm buffers | cb bits | cb bit offsets | tb out | tb crc | iterations].
  auto   al       = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t o_rm     = 0;
  size_t o_bits   = o_rm + al(rm_total);
  size_t o_offs   = o_bits + al(bits_total);
  size_t o_tb     = o_offs + al((size_t)ncb * 4);
  size_t o_crc    = o_tb + al(tb_out_len);
  size_t o_it     = o_crc + al((size_t)nof_tbs * 4);
  size_t total    = o_it + al((size_t)ncb * 4);
  cudaStream_t s  = ctx->stream;
  int          rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_b, &ctx->scratch_b_cap, total, "cudaMalloc(sch scratch)");
  }
  if (rc != PG_OK) {
    return rc;
  }
  uint8_t* base = static_cast<uint8_t*>(ctx->scratch_b);
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(base + o_offs, cb_bit_off.data(), (size_t)ncb * 4, cudaMemcpyHostToDevice, s),
                    "cudaMemcpyAsync(offsets)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemsetAsync(base + o_tb, 0, tb_out_len, s), "cudaMemsetAsync(tb)");
  }
  void* d_rm = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_RM, rm.data(), rm.size() * sizeof(pg_rm_cb), s, &d_rm);
  }
  if (rc == PG_OK) {
    rc = rate_dematch_launch(ctx, static_cast<const pg_rm_cb*>(d_rm), ncb, d_llrs,
                             reinterpret_cast<int8_t*>(base + o_rm), s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_RM, s);
  }
  void* d_ldpc = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_PUSCH, ldpc.data(), ldpc.size() * sizeof(pg_ldpc_cb), s, &d_ldpc);
  }
  if (rc == PG_OK) {
    rc = ldpc_launch(ctx, static_cast<const pg_ldpc_cb*>(d_ldpc), ncb, reinterpret_cast<const int8_t*>(base + o_rm),
                     base + o_bits, reinterpret_cast<int32_t*>(base + o_it), s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_PUSCH, s);
  }
  void* d_tb = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_TB, tbd.data(), tbd.size() * sizeof(pg_tb_desc), s, &d_tb);
  }
  if (rc == PG_OK) {
    rc = tb_assemble_launch(ctx, static_cast<const pg_tb_desc*>(d_tb), nof_tbs, base + o_bits,
                            reinterpret_cast<const uint32_t*>(base + o_offs), base + o_tb,
                            reinterpret_cast<uint32_t*>(base + o_crc), s);
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_TB, s);
  }
  std::vector<uint8_t>  tb_host(tb_out_len);
  std::vector<uint32_t> crc_host(nof_tbs);
  std::vector<int32_t>  it_host(ncb);
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(tb_host.data(), base + o_tb, tb_out_len, cudaMemcpyDeviceToHost, s), "D2H tb");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(crc_host.data(), base + o_crc, (size_t)nof_tbs * 4, cudaMemcpyDeviceToHost, s),
                    "D2H crc");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(it_host.data(), base + o_it, (size_t)ncb * 4, cudaMemcpyDeviceToHost, s),
                    "D2H iterations");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  if (rc != PG_OK) {
    return rc;
  }
  for (int t = 0; t < nof_tbs; ++t) {
    pg_sch_result& r    = results[t];
    int            okcb = 0;
    double         sum  = 0;
    uint32_t       mx   = 0;
    for (int c = 0; c < tb_ncb[t]; ++c) {
      const int32_t it  = it_host[tb_first[t] + c];
      const uint32_t run = it > 0 ? (uint32_t)it : tbs[t].max_iterations;
      okcb += it > 0;
      sum += run;
      mx = std::max(mx, run);
    }
    r.nof_cbs            = (uint32_t)tb_ncb[t];
    r.nof_cbs_crc_ok     = (uint32_t)okcb;
    r.mean_iterations    = (float)(sum / tb_ncb[t]);
    r.max_iterations_run = mx;
    // C == 1: the codeblock CRC is the TB CRC; C > 1: every codeblock CRC and the TB CRC.
    r.tb_crc_ok = (okcb == tb_ncb[t]) && (tb_ncb[t] == 1 || crc_host[t] == 0);
    // The reference writes the payload only for a passing TB.
    if (r.tb_crc_ok) {
      std::memcpy(tb_out + tbs[t].tb_out_offset, tb_host.data() + tbs[t].tb_out_offset, tbs[t].tbs_bits / 8);
    }
  }
  return PG_OK;
}

} // namespace pg

// Test infrastructure only (checker, never shipped): a flat C ABI over the reference's own
// CPU implementation of the PUSCH receive-path stages, so tests and the CPU-baseline arm
// can call it through ctypes. Every function builds the reference object through the
// reference's public factory (the same factories upper_phy_factories.cpp wires) and calls
// the reference interface unchanged:
//   ldpc_decoder::decode            include/ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h:57
//   ldpc_encoder::encode            include/ocudu/phy/upper/channel_coding/ldpc/ldpc_encoder.h
//   ldpc_rate_matcher::rate_match   include/ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_matcher.h
//   ldpc_rate_dematcher::rate_dematch include/ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h:36
//   crc_calculator::calculate       include/ocudu/phy/upper/channel_coding/crc_calculator.h:67-77
//   demodulation_mapper::demodulate_soft include/ocudu/phy/upper/channel_modulation/demodulation_mapper.h:48
// The base-graph accessors expose the lifted shift table (TS 38.212 Tables 5.3.2-2/-3) so the
// product's own compact table can be checked against it entry by entry.

#include "ocudu/phy/upper/channel_coding/channel_coding_factories.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_encoder.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_encoder_buffer.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_matcher.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_segmenter_buffer.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_segmenter_tx.h"
#include "ocudu/phy/upper/channel_modulation/channel_modulation_factories.h"
#include "ocudu/phy/upper/channel_modulation/demodulation_mapper.h"
#include "ocudu/phy/generic_functions/generic_functions_factories.h"
#include "ocudu/phy/support/re_buffer.h"
#include "ocudu/phy/support/resource_grid_reader.h"
#include "ocudu/phy/support/time_alignment_estimator/time_alignment_estimator_factories.h"
#include "ocudu/phy/upper/sequence_generators/sequence_generator_factories.h"
#include "ocudu/phy/upper/signal_processors/channel_estimator/factories.h"
#include "lib/phy/upper/signal_processors/dmrs_helper.h"
// The estimator's FP32 frequency response (before the conversion to bf16 of its public
// interface) is a private member; the checker reads it directly.
#define private public
#include "lib/phy/upper/signal_processors/channel_estimator/port_channel_estimator_average_impl.h"
#undef private
#include "ocudu/phy/upper/equalization/dynamic_ch_est_list.h"
#include "ocudu/phy/upper/equalization/equalization_factories.h"
#include "ocudu/ran/sch/sch_segmentation.h"
#include "ocudu/ran/pusch/pusch_mcs.h"
#include "ocudu/ran/sch/ldpc_base_graph.h"
#include "ocudu/ran/sch/tbs_calculator.h"
#include "lib/phy/upper/channel_coding/ldpc/ldpc_graph_impl.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_segmenter_rx.h"
#include "ocudu/ocuduvec/bit.h"
#include "../include/pusch_b200.h"
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <atomic>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

using namespace ocudu;

namespace {

ldpc_base_graph_type to_bg(int bg)
{
  return bg == 2 ? ldpc_base_graph_type::BG2 : ldpc_base_graph_type::BG1;
}

crc_generator_poly to_poly(int p)
{
  switch (p) {
    case 0:
      return crc_generator_poly::CRC16;
    case 1:
      return crc_generator_poly::CRC24A;
    case 2:
      return crc_generator_poly::CRC24B;
    case 3:
      return crc_generator_poly::CRC24C;
    case 4:
      return crc_generator_poly::CRC11;
    default:
      return crc_generator_poly::CRC6;
  }
}

modulation_scheme to_mod(int qm)
{
  switch (qm) {
    case 1:
      return modulation_scheme::BPSK;
    case 2:
      return modulation_scheme::QPSK;
    case 4:
      return modulation_scheme::QAM16;
    case 6:
      return modulation_scheme::QAM64;
    default:
      return modulation_scheme::QAM256;
  }
}

// One decoder per (thread, variant): the reference objects are not thread safe.
thread_local std::map<std::string, std::unique_ptr<ldpc_decoder>>   tl_decoders;
thread_local std::map<int, std::unique_ptr<crc_calculator>>         tl_crc;
thread_local std::unique_ptr<ldpc_rate_dematcher>                   tl_dematcher;
thread_local std::unique_ptr<ldpc_encoder>                          tl_encoder;
thread_local std::unique_ptr<ldpc_rate_matcher>                     tl_matcher;
thread_local std::unique_ptr<demodulation_mapper>                   tl_demapper;

crc_calculator* get_crc(int poly)
{
  auto it = tl_crc.find(poly);
  if (it == tl_crc.end()) {
    auto factory = create_crc_calculator_factory_sw("auto");
    it           = tl_crc.emplace(poly, factory->create(to_poly(poly))).first;
  }
  return it->second.get();
}

ldpc_decoder* get_decoder(const char* variant)
{
  std::string key(variant);
  auto        it = tl_decoders.find(key);
  if (it == tl_decoders.end()) {
    ldpc_decoder_factory::ldpc_decoder_factory_configuration cfg;
    cfg.force_decoding      = false;
    cfg.early_stop_syndrome = false;
    auto factory            = create_ldpc_decoder_factory_sw(key, cfg);
    if (!factory) {
      return nullptr;
    }
    auto dec = factory->create();
    if (!dec) {
      return nullptr;
    }
    it = tl_decoders.emplace(key, std::move(dec)).first;
  }
  return it->second.get();
}

unsigned bg_k(int bg)
{
  return bg == 2 ? 10 : 22;
}

unsigned bg_n_short(int bg)
{
  return bg == 2 ? 50 : 66;
}

} // namespace

extern "C" {

/// Decodes one codeblock with the reference decoder of the given variant ("avx512", "avx2",
/// "generic", "auto"). crc_poly < 0 disables CRC early stop. Output bits are packed MSB first
/// (K*Z bits). Returns the iteration count (> 0) when the decoder reports success, 0 when it
/// returns no value, and -1 when the variant is unavailable on this CPU.
int ref_ldpc_decode(const char*   variant,
                    int           bg,
                    int           Z,
                    int           nof_filler_bits,
                    int           nof_crc_bits,
                    int           crc_poly,
                    int           max_iterations,
                    const int8_t* llrs,
                    int           nof_llrs,
                    uint8_t*      out_packed)
{
  ldpc_decoder* dec = get_decoder(variant);
  if (dec == nullptr) {
    return -1;
  }
  ldpc_decoder::configuration cfg;
  cfg.base_graph      = to_bg(bg);
  cfg.lifting_size    = static_cast<ldpc::lifting_size_t>(Z);
  cfg.nof_filler_bits = nof_filler_bits;
  cfg.nof_crc_bits    = nof_crc_bits;
  cfg.max_iterations  = max_iterations;

  unsigned   K     = bg_k(bg) * Z;
  bit_buffer out   = bit_buffer::from_bytes(span<uint8_t>(out_packed, (K + 7) / 8));
  bit_buffer out_k = out.first(K);
  span<const log_likelihood_ratio> in(reinterpret_cast<const log_likelihood_ratio*>(llrs), nof_llrs);
  crc_calculator*                  crc = crc_poly < 0 ? nullptr : get_crc(crc_poly);
  std::optional<unsigned>          res = dec->decode(out_k, in, crc, cfg);
  return res.has_value() ? static_cast<int>(res.value()) : 0;
}

/// Returns the name of the decoder variant the reference's "auto" factory selects here.
const char* ref_ldpc_auto_variant()
{
  static std::string name;
  name = get_ldpc_decoder_type_str("auto");
  return name.c_str();
}

/// CRC of nof_bits bits packed MSB first (crc_calculator::calculate on a bit_buffer).
unsigned ref_crc_calculate(int crc_poly, const uint8_t* packed, int nof_bits)
{
  crc_calculator* crc = get_crc(crc_poly);
  std::vector<uint8_t> tmp(packed, packed + (nof_bits + 7) / 8);
  bit_buffer           buf = bit_buffer::from_bytes(span<uint8_t>(tmp)).first(nof_bits);
  return crc->calculate(buf);
}

/// CRC of whole bytes (crc_calculator::calculate_byte).
unsigned ref_crc_calculate_byte(int crc_poly, const uint8_t* bytes, int nof_bytes)
{
  return get_crc(crc_poly)->calculate_byte(span<const uint8_t>(bytes, nof_bytes));
}

/// Encodes K*Z message bits (packed MSB first; filler bits must be zero) into the full
/// N = N_short*Z codeword, unpacked one bit per byte.
int ref_ldpc_encode(int bg, int Z, const uint8_t* msg_packed, uint8_t* cw_unpacked)
{
  if (!tl_encoder) {
    tl_encoder = create_ldpc_encoder_factory_sw("generic")->create();
  }
  unsigned               K = bg_k(bg) * Z;
  std::vector<uint8_t>   tmp(msg_packed, msg_packed + (K + 7) / 8);
  bit_buffer             msg = bit_buffer::from_bytes(span<uint8_t>(tmp)).first(K);
  ldpc_encoder::configuration cfg;
  cfg.base_graph   = to_bg(bg);
  cfg.lifting_size = static_cast<ldpc::lifting_size_t>(Z);
  cfg.Nref         = 0;
  const ldpc_encoder_buffer& eb = tl_encoder->encode(msg, cfg);
  unsigned                   N  = eb.get_codeblock_length();
  eb.write_codeblock(span<uint8_t>(cw_unpacked, N), 0);
  return static_cast<int>(N);
}

/// Encodes K*Z message bits and rate matches them to E bits (unpacked, one bit per byte),
/// with the reference encoder and rate matcher.
int ref_ldpc_encode_rm(int            bg,
                       int            Z,
                       int            rv,
                       int            qm,
                       int            Nref,
                       int            nof_filler_bits,
                       int            E,
                       const uint8_t* msg_packed,
                       uint8_t*       out_unpacked)
{
  if (!tl_encoder) {
    tl_encoder = create_ldpc_encoder_factory_sw("generic")->create();
  }
  if (!tl_matcher) {
    tl_matcher = create_ldpc_rate_matcher_factory_sw()->create();
  }
  unsigned             K = bg_k(bg) * Z;
  std::vector<uint8_t> tmp(msg_packed, msg_packed + (K + 7) / 8);
  bit_buffer           msg = bit_buffer::from_bytes(span<uint8_t>(tmp)).first(K);
  ldpc_encoder::configuration cfg;
  cfg.base_graph                 = to_bg(bg);
  cfg.lifting_size               = static_cast<ldpc::lifting_size_t>(Z);
  cfg.Nref                       = Nref;
  const ldpc_encoder_buffer& eb  = tl_encoder->encode(msg, cfg);
  codeblock_metadata         md  = {};
  md.tb_common.base_graph        = to_bg(bg);
  md.tb_common.lifting_size      = static_cast<ldpc::lifting_size_t>(Z);
  md.tb_common.rv                = rv;
  md.tb_common.mod               = to_mod(qm);
  md.tb_common.Nref              = Nref;
  md.cb_specific.full_length     = bg_n_short(bg) * Z;
  md.cb_specific.rm_length       = E;
  md.cb_specific.nof_filler_bits = nof_filler_bits;
  std::vector<uint8_t> packed((E + 7) / 8);
  bit_buffer           out = bit_buffer::from_bytes(span<uint8_t>(packed)).first(E);
  tl_matcher->rate_match(out, eb, md);
  for (int i = 0; i < E; ++i) {
    out_unpacked[i] = out.extract(i, 1);
  }
  return 0;
}

/// Rate dematching of E LLRs into the N-LLR circular buffer (ldpc_rate_dematcher::rate_dematch).
/// The output buffer is read before the call (soft combining when new_data == 0).
int ref_rate_dematch(int           bg,
                     int           Z,
                     int           rv,
                     int           qm,
                     int           Nref,
                     int           nof_filler_bits,
                     int           new_data,
                     const int8_t* in,
                     int           E,
                     int8_t*       out)
{
  if (!tl_dematcher) {
    tl_dematcher = create_ldpc_rate_dematcher_factory_sw("auto")->create();
  }
  codeblock_metadata md          = {};
  md.tb_common.base_graph        = to_bg(bg);
  md.tb_common.lifting_size      = static_cast<ldpc::lifting_size_t>(Z);
  md.tb_common.rv                = rv;
  md.tb_common.mod               = to_mod(qm);
  md.tb_common.Nref              = Nref;
  md.cb_specific.full_length     = bg_n_short(bg) * Z;
  md.cb_specific.rm_length       = E;
  md.cb_specific.nof_filler_bits = nof_filler_bits;
  unsigned N                     = bg_n_short(bg) * Z;
  tl_dematcher->rate_dematch(span<log_likelihood_ratio>(reinterpret_cast<log_likelihood_ratio*>(out), N),
                             span<const log_likelihood_ratio>(reinterpret_cast<const log_likelihood_ratio*>(in), E),
                             new_data != 0,
                             md);
  return 0;
}

/// Soft demapping (demodulation_mapper::demodulate_soft): symbols are interleaved (re, im)
/// float pairs; one noise variance per symbol; qm LLRs per symbol.
int ref_demodulate_soft(int qm, const float* symbols, const float* noise_vars, int nof_symbols, int8_t* llrs)
{
  if (!tl_demapper) {
    tl_demapper = create_demodulation_mapper_factory()->create();
  }
  tl_demapper->demodulate_soft(
      span<log_likelihood_ratio>(reinterpret_cast<log_likelihood_ratio*>(llrs), nof_symbols * qm),
      span<const cf_t>(reinterpret_cast<const cf_t*>(symbols), nof_symbols),
      span<const float>(noise_vars, nof_symbols),
      to_mod(qm));
  return 0;
}

/// Lifted shift of base-graph edge (row, col) for lifting size Z, or -1 when there is no edge.
int ref_ldpc_graph_shift(int bg, int Z, int row, int col)
{
  ldpc_graph_impl g(to_bg(bg), static_cast<ldpc::lifting_size_t>(Z));
  uint16_t        v = g.get_lifted_node(row, col);
  return v == ldpc::NO_EDGE ? -1 : static_cast<int>(v);
}

/// Writes the variable-node list of base-graph row `row` (in the decoder's edge order) and
/// returns its length.
int ref_ldpc_graph_row(int bg, int row, int* out_vars)
{
  ldpc_graph_impl                 g(to_bg(bg), ldpc::LS384);
  const ldpc::BG_adjacency_row_t& r = g.get_adjacency_row(row);
  int                             n = 0;
  for (uint16_t v : r) {
    if (v == ldpc::NO_EDGE) {
      break;
    }
    out_vars[n++] = v;
  }
  return n;
}

/// TS 38.212 segmentation quantities as computed by the reference (sch_segmentation.h).
/// Writes {C, Z, K(segment length), nof_tb_crc_bits}.
int ref_sch_segmentation(int tbs_bits, int bg, int* out4)
{
  units::bits          tbs(tbs_bits);
  ldpc_base_graph_type g   = to_bg(bg);
  unsigned             C   = compute_nof_codeblocks(tbs, g);
  unsigned             Zc  = compute_lifting_size(tbs, g, C);
  unsigned             K   = compute_codeblock_size(g, Zc).value();
  unsigned             crc = compute_tb_crc_size(tbs).value();
  out4[0]                  = C;
  out4[1]                  = Zc;
  out4[2]                  = K;
  out4[3]                  = crc;
  return 0;
}

/// Decodes a batch of codeblocks on nof_threads host threads (one reference decoder per thread,
/// codeblocks claimed dynamically), as the reference's per-codeblock executor tasks do
/// (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:466-470). meta holds six ints
/// per codeblock {bg, Z, filler, crc_poly, max_iterations, nof_llrs}; llr_offsets gives each
/// codeblock's first LLR. Writes iterations (0 = failure) and returns the wall time in seconds.
double ref_ldpc_decode_batch_mt(const char*    variant,
                                int            nof_cbs,
                                const int*     meta,
                                const int64_t* llr_offsets,
                                const int8_t*  llrs,
                                int*           iterations,
                                int            nof_threads)
{
  std::atomic<int> next{0};
  auto             worker = [&]() {
    std::vector<uint8_t> out((22 * 384 + 7) / 8);
    for (int i = next.fetch_add(1); i < nof_cbs; i = next.fetch_add(1)) {
      const int* m    = meta + 6 * i;
      int        poly = m[3] == 255 ? -1 : m[3];
      iterations[i]   = ref_ldpc_decode(variant,
                                      m[0],
                                      m[1],
                                      m[2],
                                      poly == 0 ? 16 : 24,
                                      poly,
                                      m[4],
                                      llrs + llr_offsets[i],
                                      m[5],
                                      out.data());
    }
  };
  // Create the per-thread decoders before the clock starts.
  auto                     t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (int t = 0; t < nof_threads; ++t) {
    pool.emplace_back(worker);
  }
  for (auto& th : pool) {
    th.join();
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

/// Channel equalisation with the reference's generic equaliser
/// (channel_equalizer::equalize, include/ocudu/phy/upper/equalization/channel_equalizer.h:71-76).
/// algorithm: 0 = ZF, 1 = MMSE. ch_symbols: cbf16 [port][re] as uint32 (real in the low half);
/// ch_estimates: cbf16 [port][layer][re]; outputs layer-interleaved [re][layer].
int ref_equalize(int             algorithm,
                 int             nof_re,
                 int             nof_ports,
                 int             nof_layers,
                 const uint32_t* ch_symbols,
                 const uint32_t* ch_estimates,
                 const float*    noise_var_per_port,
                 float           tx_scaling,
                 float*          eq_symbols,
                 float*          eq_noise_vars)
{
  auto factory = create_channel_equalizer_generic_factory(algorithm == 0 ? channel_equalizer_algorithm_type::zf
                                                                         : channel_equalizer_algorithm_type::mmse);
  auto eq      = factory->create();
  dynamic_re_buffer<cbf16_t> syms(nof_ports, nof_re);
  dynamic_ch_est_list        est(nof_re, nof_ports, nof_layers);
  for (int p = 0; p < nof_ports; ++p) {
    std::memcpy(syms.get_slice(p).data(), ch_symbols + (size_t)p * nof_re, (size_t)nof_re * 4);
    for (int l = 0; l < nof_layers; ++l) {
      std::memcpy(est.get_channel(p, l).data(), ch_estimates + ((size_t)p * nof_layers + l) * nof_re,
                  (size_t)nof_re * 4);
    }
  }
  eq->equalize(span<cf_t>(reinterpret_cast<cf_t*>(eq_symbols), (size_t)nof_re * nof_layers),
               span<float>(eq_noise_vars, (size_t)nof_re * nof_layers),
               syms,
               est,
               span<const float>(noise_var_per_port, nof_ports),
               tx_scaling);
  return 0;
}

} // extern "C"

namespace {

/// Read-only resource grid over caller memory: cbf16 [port][symbol][subcarrier].
class array_grid_reader : public resource_grid_reader
{
public:
  array_grid_reader(const uint32_t* data, unsigned nports, unsigned nsymb, unsigned nsubc) :
    data_(reinterpret_cast<const cbf16_t*>(data)), nports_(nports), nsymb_(nsymb), nsubc_(nsubc)
  {
  }
  unsigned     get_nof_ports() const override { return nports_; }
  unsigned     get_nof_subc() const override { return nsubc_; }
  unsigned     get_nof_symbols() const override { return nsymb_; }
  bool         is_empty(unsigned) const override { return false; }
  bool         is_empty() const override { return false; }
  crb_interval get_allocation_range(unsigned, unsigned) const override { return {0, nsubc_ / 12}; }
  span<cf_t>   get(span<cf_t> symbols, unsigned port, unsigned l, unsigned k_init, const bounded_bitset<MAX_NOF_SUBCARRIERS>& mask) const override
  {
    mask.for_each(0, mask.size(), [&](unsigned k) {
      symbols.front() = to_cf(view(port, l)[k_init + k]);
      symbols         = symbols.last(symbols.size() - 1);
    });
    return symbols;
  }
  span<cbf16_t> get(span<cbf16_t> symbols, unsigned port, unsigned l, unsigned k_init, const bounded_bitset<MAX_NOF_SUBCARRIERS>& mask) const override
  {
    mask.for_each(0, mask.size(), [&](unsigned k) {
      symbols.front() = view(port, l)[k_init + k];
      symbols         = symbols.last(symbols.size() - 1);
    });
    return symbols;
  }
  void get(span<cf_t> symbols, unsigned port, unsigned l, unsigned k_init, unsigned stride) const override
  {
    for (unsigned i = 0; i != symbols.size(); ++i) {
      symbols[i] = to_cf(view(port, l)[k_init + i * stride]);
    }
  }
  void get(span<cbf16_t> symbols, unsigned port, unsigned l, unsigned k_init) const override
  {
    std::copy_n(view(port, l).begin() + k_init, symbols.size(), symbols.begin());
  }
  span<const cbf16_t> get_view(unsigned port, unsigned l) const override { return view(port, l); }

private:
  span<const cbf16_t> view(unsigned port, unsigned l) const
  {
    return span<const cbf16_t>(data_ + ((size_t)port * nsymb_ + l) * nsubc_, nsubc_);
  }
  const cbf16_t* data_;
  unsigned       nports_, nsymb_, nsubc_;
};

} // namespace

extern "C" {

/// One receive port of the reference's DM-RS PUSCH channel estimator
/// (port_channel_estimator::compute, FD "filter", TD "interpolate", no CFO compensation), type-1
/// DM-RS on layers 0..nof_layers-1, pilots generated as dmrs_pusch_estimator_impl does
/// (pseudo-random c_init per symbol, OCC of port 1). grid: cbf16 [nports][14][nsubc].
/// Outputs: freq (complex float [nof_dmrs][nof_layers][12*nof_rb], the FP32 response),
/// sym_est (cbf16 [14][nof_layers][12*nof_rb], the public per-symbol estimates) and
/// scalars {noise_var, epre, snr, rsrp[layer]...}.
static int port_estimate_impl(const uint32_t* grid,
                              int             nports,
                              int             nsubc,
                              int             port,
                              int             slot,
                              int             n_id,
                              int             n_scid,
                              int             rb_start,
                              int             nof_rb,
                              int             nof_layers,
                              uint32_t        dmrs_symbol_mask,
                              float           scaling,
                              float*          freq,
                              uint32_t*       sym_est,
                              float*          scalars,
                              float*          pilots_out,
                              double*         cfo_ta)
{
  array_grid_reader reader(grid, nports, 14, nsubc);
  auto              prg = create_pseudo_random_generator_sw_factory()->create();

  port_channel_estimator::configuration cfg;
  cfg.scs          = subcarrier_spacing::kHz30;
  cfg.cp           = cyclic_prefix::NORMAL;
  cfg.first_symbol = 0;
  cfg.nof_symbols  = 14;
  cfg.scaling      = scaling;
  cfg.rx_ports.push_back(static_cast<uint8_t>(port));
  bounded_bitset<MAX_NSYMB_PER_SLOT> symbols(14);
  for (int s = 0; s < 14; ++s) {
    if ((dmrs_symbol_mask >> s) & 1u) {
      symbols.set(s);
    }
  }
  crb_bitmap rb_mask(rb_start + nof_rb);
  rb_mask.fill(rb_start, rb_start + nof_rb);
  unsigned nof_dmrs = symbols.count();
  unsigned npil     = 6 * nof_rb;

  dmrs_symbol_list pilots({npil, nof_dmrs, static_cast<unsigned>(nof_layers)});
  for (int s = 0, i = 0; s < 14; ++s) {
    if (!symbols.test(s)) {
      continue;
    }
    unsigned c_init = ((14 * slot + s + 1) * (2 * n_id + 1) * (1U << 17) + (2 * n_id + n_scid)) % (1U << 31);
    prg->init(c_init);
    dmrs_sequence_generate(pilots.get_symbol(i, 0), *prg, M_SQRT1_2, 0, 6, rb_mask);
    ++i;
  }
  for (int l = 1; l < nof_layers; ++l) {
    dmrs_pxsch_parameters params = get_pxsch_dmrs_params(dmrs_config_type::type1, l);
    for (unsigned i = 0; i != nof_dmrs; ++i) {
      span<cf_t>       d  = pilots.get_symbol(i, l);
      span<const cf_t> d0 = pilots.get_symbol(i, 0);
      std::copy(d0.begin(), d0.end(), d.begin());
      if (params.w_f[0] != params.w_f[1]) {
        for (unsigned k = 1; k < d.size(); k += 2) {
          d[k] *= params.w_f[1];
        }
      }
    }
  }
  for (int l = 0; l < nof_layers; ++l) {
    dmrs_pxsch_parameters params = get_pxsch_dmrs_params(dmrs_config_type::type1, l);
    cfg.dmrs_pattern.push_back({symbols, rb_mask, {}, std::nullopt, params.re_pattern});
  }

  auto ta_factory = create_time_alignment_estimator_dft_factory(create_dft_processor_factory_generic());
  auto factory    = create_port_channel_estimator_factory_sw(ta_factory);
  auto est        = factory->create(port_channel_estimator_fd_smoothing_strategy::filter,
                             port_channel_estimator_td_interpolation_strategy::interpolate,
                             false);
  const port_channel_estimator_results& res = est->compute(reader, 0, pilots, cfg);

  auto* impl = dynamic_cast<port_channel_estimator_average_impl*>(est.get());
  for (unsigned d = 0; d != nof_dmrs; ++d) {
    for (int l = 0; l < nof_layers; ++l) {
      span<const cf_t> fr = impl->freq_response_hop0.get_symbol(d, l);
      std::memcpy(freq + ((size_t)d * nof_layers + l) * 2 * fr.size(), fr.data(), fr.size() * sizeof(cf_t));
    }
  }
  unsigned nsc = 12 * nof_rb;
  for (int s = 0; s < 14; ++s) {
    for (int l = 0; l < nof_layers; ++l) {
      res.get_symbol_ch_estimate(
          span<cbf16_t>(reinterpret_cast<cbf16_t*>(sym_est) + ((size_t)s * nof_layers + l) * nsc, nsc), s, l);
    }
  }
  scalars[0] = res.get_noise_variance();
  scalars[1] = res.get_epre();
  scalars[2] = res.get_snr();
  for (int l = 0; l < nof_layers; ++l) {
    scalars[3 + l] = res.get_rsrp(l);
  }
  if (pilots_out != nullptr) {
    for (unsigned d = 0; d != nof_dmrs; ++d) {
      for (int l = 0; l < nof_layers; ++l) {
        span<const cf_t> pl = pilots.get_symbol(d, l);
        std::memcpy(pilots_out + ((size_t)d * nof_layers + l) * 2 * npil, pl.data(), npil * sizeof(cf_t));
      }
    }
  }
  if (cfo_ta != nullptr) {
    std::optional<float> cfo = res.get_cfo_Hz();
    cfo_ta[0]                = cfo.has_value() ? static_cast<double>(*cfo) : std::nan("");
    cfo_ta[1]                = res.get_time_alignment().to_seconds();
  }
  return 0;
}

int ref_port_estimate(const uint32_t* grid,
                      int             nports,
                      int             nsubc,
                      int             port,
                      int             slot,
                      int             n_id,
                      int             n_scid,
                      int             rb_start,
                      int             nof_rb,
                      int             nof_layers,
                      uint32_t        dmrs_symbol_mask,
                      float           scaling,
                      float*          freq,
                      uint32_t*       sym_est,
                      float*          scalars)
{
  return port_estimate_impl(grid, nports, nsubc, port, slot, n_id, n_scid, rb_start, nof_rb, nof_layers,
                            dmrs_symbol_mask, scaling, freq, sym_est, scalars, nullptr, nullptr);
}

/// ref_port_estimate that also returns the pilots it used (cf32 [nof_dmrs][nof_layers][6*nof_rb],
/// dmrs_pusch_estimator_impl's sequences) and the reference's CFO in Hz (NaN when it has none) and
/// time alignment in seconds (cfo_ta[0], cfo_ta[1]).
int ref_port_estimate_full(const uint32_t* grid,
                           int             nports,
                           int             nsubc,
                           int             port,
                           int             slot,
                           int             n_id,
                           int             n_scid,
                           int             rb_start,
                           int             nof_rb,
                           int             nof_layers,
                           uint32_t        dmrs_symbol_mask,
                           float           scaling,
                           float*          freq,
                           uint32_t*       sym_est,
                           float*          scalars,
                           float*          pilots_out,
                           double*         cfo_ta)
{
  return port_estimate_impl(grid, nports, nsubc, port, slot, n_id, n_scid, rb_start, nof_rb, nof_layers,
                            dmrs_symbol_mask, scaling, freq, sym_est, scalars, pilots_out, cfo_ta);
}

/// PUSCH MCS (TS 38.214 Tables 5.1.3.1-1/2; table 0 = qam64, 1 = qam256), no transform
/// precoding: returns Qm and writes the target code rate x 1024 (pusch_mcs_get_config).
int ref_pusch_mcs(int table, int index, float* rate_x1024)
{
  const sch_mcs_description d = pusch_mcs_get_config(table == 0 ? pusch_mcs_table::qam64 : pusch_mcs_table::qam256,
                                                     sch_mcs_index(static_cast<uint8_t>(index)), false, false);
  *rate_x1024 = d.target_code_rate;
  return static_cast<int>(get_bits_per_symbol(d.modulation));
}

/// Transport block size in bits (tbs_calculator_calculate, TS 38.214 Section 5.1.3.2).
unsigned ref_tbs(int nof_symb_sh, int nof_dmrs_prb, int nof_oh_prb, int qm, float rate_x1024, int nof_layers, int n_prb)
{
  tbs_calculator_configuration cfg = {};
  cfg.nof_symb_sh                  = nof_symb_sh;
  cfg.nof_dmrs_prb                 = nof_dmrs_prb;
  cfg.nof_oh_prb                   = nof_oh_prb;
  cfg.mcs_descr.modulation         = to_mod(qm);
  cfg.mcs_descr.target_code_rate   = rate_x1024;
  cfg.nof_layers                   = nof_layers;
  cfg.tb_scaling_field             = 0;
  cfg.n_prb                        = n_prb;
  return static_cast<unsigned>(units::bits(tbs_calculator_calculate(cfg)).value());
}

/// LDPC base graph (1 or 2) for a target code rate and payload size (TS 38.212 Section 7.2.2).
int ref_base_graph(float rate, unsigned tbs_bits)
{
  return get_ldpc_base_graph(rate, units::bits(tbs_bits)) == ldpc_base_graph_type::BG1 ? 1 : 2;
}

/// The reference's CPU receive path for a batch of PUSCH PDUs, one UE at a time per thread, with
/// the reference's own stage objects in the order pusch_processor_impl::process runs them
/// (lib/phy/upper/channel_processors/pusch/pusch_processor_impl.cpp:349-900): DM-RS pilots and
/// port_channel_estimator (FD filter, TD interpolate) per receive port, per data symbol
/// get_symbol_ch_estimate + channel_equalizer (MMSE) + demodulation_mapper, descrambling with the
/// pseudo-random generator, ldpc_segmenter_rx, then per codeblock ldpc_rate_dematcher and
/// ldpc_decoder with CRC early stop, and the TB join of pusch_decoder_impl::join_and_notify
/// (pusch_decoder_impl.cpp:612-710). No UCI, no HARQ combining. Threads claim UEs from a shared
/// counter (independent UE-level work, as the reference's PUSCH processor pool runs them).
/// ues: pg_pusch_ue array (include/pusch_b200.h layout); grids: cbf16 words; tb_out: TB bytes at
/// each UE's tb_out_offset (written when the TB CRC passes); ok / iters: per UE. Returns wall s.
static double pusch_decode_impl(const pg_pusch_ue* ues,
                                int                nof_ues,
                                const uint32_t*    grids,
                                uint8_t*           tb_out,
                                int32_t*           ok,
                                float*             mean_iters,
                                int                nof_threads,
                                const int32_t*     cb_first,
                                int32_t*           cb_iters,
                                int32_t*           nof_cbs,
                                int8_t*            llr_out)
{
  std::atomic<int> next{0};
  auto worker = [&]() {
    auto prg        = create_pseudo_random_generator_sw_factory()->create();
    auto ta_factory = create_time_alignment_estimator_dft_factory(create_dft_processor_factory_generic());
    auto est        = create_port_channel_estimator_factory_sw(ta_factory)
                   ->create(port_channel_estimator_fd_smoothing_strategy::filter,
                            port_channel_estimator_td_interpolation_strategy::interpolate,
                            false);
    auto eq    = create_channel_equalizer_generic_factory(channel_equalizer_algorithm_type::mmse)->create();
    auto demap = create_demodulation_mapper_factory()->create();
    auto seg   = create_ldpc_segmenter_rx_factory_sw()->create();
    auto dem   = create_ldpc_rate_dematcher_factory_sw("auto")->create();
    ldpc_decoder_factory::ldpc_decoder_factory_configuration dcfg_f = {false, false};
    auto dec   = create_ldpc_decoder_factory_sw("auto", dcfg_f)->create();
    auto crcf  = create_crc_calculator_factory_sw("auto");
    auto crc16 = crcf->create(crc_generator_poly::CRC16);
    auto crc24a = crcf->create(crc_generator_poly::CRC24A);
    auto crc24b = crcf->create(crc_generator_poly::CRC24B);

    for (int i = next++; i < nof_ues; i = next++) {
      const pg_pusch_ue& u   = ues[i];
      const unsigned     np  = u.nof_rx_ports;
      const unsigned     nl  = u.nof_layers;
      const unsigned     nsc = 12u * u.nof_rb;
      const unsigned     qm  = u.modulation_order;
      array_grid_reader  reader(grids + u.grid_offset, np, 14, u.grid_nof_subc);

      // DM-RS pilots of every layer and the estimator configuration.
      port_channel_estimator::configuration cfg;
      cfg.scs          = subcarrier_spacing::kHz30;
      cfg.cp           = cyclic_prefix::NORMAL;
      cfg.first_symbol = u.first_symbol;
      cfg.nof_symbols  = u.nof_symbols;
      cfg.scaling      = u.dmrs_scaling;
      for (unsigned p = 0; p < np; ++p) {
        cfg.rx_ports.push_back(static_cast<uint8_t>(p));
      }
      bounded_bitset<MAX_NSYMB_PER_SLOT> symbols(14);
      for (int s = 0; s < 14; ++s) {
        if ((u.dmrs_symbol_mask >> s) & 1u) {
          symbols.set(s);
        }
      }
      crb_bitmap rb_mask(u.rb_start + u.nof_rb);
      rb_mask.fill(u.rb_start, u.rb_start + u.nof_rb);
      const unsigned   nof_dmrs = symbols.count();
      dmrs_symbol_list pilots({6u * u.nof_rb, nof_dmrs, nl});
      for (int s = 0, d = 0; s < 14; ++s) {
        if (!symbols.test(s)) {
          continue;
        }
        unsigned c_init =
            ((14 * u.slot + s + 1) * (2 * u.n_id + 1) * (1U << 17) + (2 * u.n_id + u.n_scid)) % (1U << 31);
        prg->init(c_init);
        dmrs_sequence_generate(pilots.get_symbol(d, 0), *prg, M_SQRT1_2, 0, 6, rb_mask);
        ++d;
      }
      for (unsigned l = 1; l < nl; ++l) {
        dmrs_pxsch_parameters params = get_pxsch_dmrs_params(dmrs_config_type::type1, l);
        for (unsigned d = 0; d != nof_dmrs; ++d) {
          span<cf_t>       dst = pilots.get_symbol(d, l);
          span<const cf_t> src = pilots.get_symbol(d, 0);
          std::copy(src.begin(), src.end(), dst.begin());
          if (params.w_f[0] != params.w_f[1]) {
            for (unsigned k = 1; k < dst.size(); k += 2) {
              dst[k] *= params.w_f[1];
            }
          }
        }
      }
      for (unsigned l = 0; l < nl; ++l) {
        dmrs_pxsch_parameters params = get_pxsch_dmrs_params(dmrs_config_type::type1, l);
        cfg.dmrs_pattern.push_back({symbols, rb_mask, {}, std::nullopt, params.re_pattern});
      }

      // Channel estimates of every data symbol, layer and port; port noise variances.
      std::vector<unsigned> data_syms;
      for (unsigned s = u.first_symbol; s < u.first_symbol + u.nof_symbols; ++s) {
        if (!symbols.test(s)) {
          data_syms.push_back(s);
        }
      }
      std::vector<cbf16_t> h((size_t)np * data_syms.size() * nl * nsc);
      std::vector<float>   nvar(np);
      for (unsigned p = 0; p < np; ++p) {
        const port_channel_estimator_results& res = est->compute(reader, p, pilots, cfg);
        nvar[p]                                   = res.get_noise_variance();
        for (unsigned k = 0; k < data_syms.size(); ++k) {
          for (unsigned l = 0; l < nl; ++l) {
            res.get_symbol_ch_estimate(span<cbf16_t>(h.data() + (((size_t)p * data_syms.size() + k) * nl + l) * nsc, nsc),
                                       data_syms[k], l);
          }
        }
      }

      // Equalisation and demapping per data symbol, then descrambling.
      const unsigned                    g = data_syms.size() * nsc * nl * qm;
      std::vector<log_likelihood_ratio> llr(g);
      dynamic_re_buffer<cbf16_t>        y(np, nsc);
      dynamic_ch_est_list               hl(nsc, np, nl);
      std::vector<cf_t>                 eqs(nsc * nl);
      std::vector<float>                eqv(nsc * nl);
      for (unsigned k = 0; k < data_syms.size(); ++k) {
        for (unsigned p = 0; p < np; ++p) {
          span<const cbf16_t> row = reader.get_view(p, data_syms[k]);
          std::copy_n(row.begin() + 12 * u.rb_start, nsc, y.get_slice(p).begin());
          for (unsigned l = 0; l < nl; ++l) {
            std::copy_n(h.data() + (((size_t)p * data_syms.size() + k) * nl + l) * nsc, nsc,
                        hl.get_channel(p, l).begin());
          }
        }
        eq->equalize(eqs, eqv, y, hl, nvar, 1.0F);
        demap->demodulate_soft(span<log_likelihood_ratio>(llr).subspan((size_t)k * nsc * nl * qm, nsc * nl * qm), eqs, eqv,
                               to_mod(qm));
      }
      prg->init((static_cast<unsigned>(u.rnti) << 15) + u.n_id_data);
      prg->apply_xor(span<log_likelihood_ratio>(llr), span<const log_likelihood_ratio>(llr));

      // Segmentation, dematching and decoding of every codeblock; TB join.
      segmenter_config sc;
      sc.transport_block_size = units::bytes(u.tbs_bits / 8);
      sc.base_graph           = u.base_graph == 1 ? ldpc_base_graph_type::BG1 : ldpc_base_graph_type::BG2;
      sc.rv                   = u.rv;
      sc.mod                  = to_mod(qm);
      sc.Nref                 = u.nref;
      sc.nof_layers           = nl;
      sc.nof_ch_symbols       = g / qm;
      static_vector<described_rx_codeblock, MAX_NOF_SEGMENTS> cbs;
      if (llr_out != nullptr) {
        std::memcpy(llr_out + u.llr_offset, llr.data(), llr.size());
      }
      seg->segment(cbs, llr, sc);
      const unsigned  C      = cbs.size();
      if (nof_cbs != nullptr) {
        nof_cbs[i] = static_cast<int32_t>(C);
      }
      crc_calculator* cb_crc = C > 1 ? crc24b.get() : (u.tbs_bits <= 3824 ? crc16.get() : crc24a.get());
      std::vector<uint8_t> tb_bits;
      bool                 all_ok = true;
      unsigned             it_sum = 0;
      for (unsigned c = 0; c < C; ++c) {
        const codeblock_metadata& md = cbs[c].second;
        const unsigned            N  = md.cb_specific.full_length;
        const unsigned            z  = static_cast<unsigned>(md.tb_common.lifting_size);
        const unsigned            K  = (u.base_graph == 1 ? 22 : 10) * z;
        std::vector<log_likelihood_ratio> rm(N);
        dem->rate_dematch(rm, cbs[c].first, true, md);
        ldpc_decoder::configuration dc;
        dc.base_graph      = sc.base_graph;
        dc.lifting_size    = md.tb_common.lifting_size;
        dc.nof_filler_bits = md.cb_specific.nof_filler_bits;
        dc.nof_crc_bits    = md.cb_specific.nof_crc_bits;
        dc.max_iterations  = u.max_iterations;
        dynamic_bit_buffer           out(K);
        std::optional<unsigned>      r = dec->decode(out, rm, cb_crc, dc);
        all_ok                         = all_ok && r.has_value();
        if (cb_iters != nullptr) {
          cb_iters[cb_first[i] + c] = r.has_value() ? static_cast<int32_t>(*r) : 0;
        }
        it_sum += r.has_value() ? *r : u.max_iterations;
        const unsigned payload = K - md.cb_specific.nof_filler_bits - (C > 1 ? 24 : 0);
        for (unsigned b = 0; b < payload; ++b) {
          tb_bits.push_back(static_cast<uint8_t>(out.extract(b, 1)));
        }
      }
      bool tb_ok = false;
      if (C == 1) {
        tb_ok = all_ok;
      } else if (all_ok) {
        dynamic_bit_buffer tb(u.tbs_bits);
        ocuduvec::bit_pack(tb, span<const uint8_t>(tb_bits.data(), u.tbs_bits));
        unsigned checksum = 0;
        for (unsigned b = 0; b < 24; ++b) {
          checksum = (checksum << 1) | tb_bits[u.tbs_bits + b];
        }
        tb_ok = crc24a->calculate(tb) == checksum;
      }
      ok[i]         = tb_ok ? 1 : 0;
      mean_iters[i] = static_cast<float>(it_sum) / static_cast<float>(C);
      if (tb_ok) {
        for (unsigned b = 0; b < u.tbs_bits / 8; ++b) {
          uint8_t v = 0;
          for (unsigned j = 0; j < 8; ++j) {
            v = static_cast<uint8_t>((v << 1) | tb_bits[8 * b + j]);
          }
          tb_out[u.tb_out_offset + b] = v;
        }
      }
    }
  };
  const auto               t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (int t = 0; t < std::max(1, nof_threads); ++t) {
    pool.emplace_back(worker);
  }
  for (auto& th : pool) {
    th.join();
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double ref_pusch_decode_mt(const pg_pusch_ue* ues,
                           int                nof_ues,
                           const uint32_t*    grids,
                           uint8_t*           tb_out,
                           int32_t*           ok,
                           float*             mean_iters,
                           int                nof_threads)
{
  return pusch_decode_impl(ues, nof_ues, grids, tb_out, ok, mean_iters, nof_threads, nullptr, nullptr, nullptr,
                           nullptr);
}

/// ref_pusch_decode_mt with the stage taps a slot-level parity check needs: nof_cbs[u] = C of UE u,
/// cb_iters[cb_first[u] + c] = the ldpc_decoder result of codeblock c (iterations, 0 = the
/// reference's empty optional), and llr_out (may be NULL) = the descrambled codeword LLRs of every
/// UE at its llr_offset - the soft bits pusch_processor hands to pusch_decoder.
double ref_pusch_decode_detail(const pg_pusch_ue* ues,
                               int                nof_ues,
                               const uint32_t*    grids,
                               uint8_t*           tb_out,
                               int32_t*           ok,
                               float*             mean_iters,
                               const int32_t*     cb_first,
                               int32_t*           cb_iters,
                               int32_t*           nof_cbs,
                               int8_t*            llr_out,
                               int                nof_threads)
{
  return pusch_decode_impl(ues, nof_ues, grids, tb_out, ok, mean_iters, nof_threads, cb_first, cb_iters, nof_cbs,
                           llr_out);
}

} // extern "C"

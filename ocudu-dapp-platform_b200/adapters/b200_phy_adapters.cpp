// Implementation of the reference-interface adapters over the pusch_b200 C ABI.
#include "b200_phy_adapters.h"

#include "../../include/pusch_b200.h"
#include "ocudu/ocuduvec/bit.h"
#include "ocudu/ocuduvec/copy.h"
#include "ocudu/phy/support/resource_grid_reader.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_notifier.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_result.h"
#include "ocudu/phy/upper/rx_buffer.h"
#include "ocudu/ran/pusch/pusch_constants.h"
#include "ocudu/ran/sch/modulation_scheme.h"
#include "ocudu/support/error_handling.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ocudu {
namespace b200 {

context_handle::context_handle(const device_config& cfg)
{
  pg_config c{cfg.device, cfg.max_codeblocks, 0};
  const int rc = pg_create(&c, &ctx);
  report_fatal_error_if_not(rc == PG_OK, "pusch_b200: pg_create on device {} failed with status {}.", cfg.device, rc);
}

context_handle::~context_handle()
{
  if (ctx != nullptr) {
    pg_destroy(ctx);
  }
}

void context_handle::check(int rc, const char* what) const
{
  report_fatal_error_if_not(rc == PG_OK, "pusch_b200: {} failed: {}.", what, pg_last_error(ctx));
}

namespace {

uint32_t to_pg_poly(crc_generator_poly poly)
{
  switch (poly) {
    case crc_generator_poly::CRC16:
      return PG_CRC16;
    case crc_generator_poly::CRC24A:
      return PG_CRC24A;
    case crc_generator_poly::CRC24B:
      return PG_CRC24B;
    default:
      return PG_CRC_NONE;
  }
}

int to_pg_base_graph(ldpc_base_graph_type bg)
{
  return bg == ldpc_base_graph_type::BG1 ? 1 : 2;
}

const int8_t* raw(span<const log_likelihood_ratio> s)
{
  static_assert(sizeof(log_likelihood_ratio) == 1, "log_likelihood_ratio is one byte");
  return reinterpret_cast<const int8_t*>(s.data());
}

int8_t* raw(span<log_likelihood_ratio> s)
{
  return reinterpret_cast<int8_t*>(s.data());
}

} // namespace

// ---------------------------------------------------------------------------------------------
// ldpc_decoder

std::optional<unsigned> ldpc_decoder_b200::decode(bit_buffer&                      output,
                                                  span<const log_likelihood_ratio> input,
                                                  crc_calculator*                  crc,
                                                  const configuration&             cfg)
{
  const int      bg      = to_pg_base_graph(cfg.base_graph);
  const unsigned z       = static_cast<unsigned>(cfg.lifting_size);
  const unsigned msg_len = (bg == 1 ? 22U : 10U) * z;

  // The reference's contract on short inputs (ldpc_decoder_impl.cpp:66-80): with fewer significant
  // LLRs than message bits nothing is decoded; without an external CRC the output is all ones.
  const auto     last       = std::find_if(input.rbegin(), input.rend(), [](log_likelihood_ratio v) { return v != 0; });
  const unsigned input_size = static_cast<unsigned>(std::distance(input.begin(), last.base()));
  if (input_size < msg_len) {
    if (crc == nullptr) {
      output.one();
    }
    return std::nullopt;
  }

  pg_ldpc_cb d      = {};
  d.llr_offset      = 0;
  d.nof_llrs        = static_cast<uint32_t>(input.size());
  d.out_offset      = 0;
  d.lifting_size    = static_cast<uint16_t>(z);
  d.nof_filler_bits = static_cast<uint16_t>(cfg.nof_filler_bits);
  d.base_graph      = static_cast<uint8_t>(bg);
  d.crc_poly        = static_cast<uint8_t>(crc != nullptr ? to_pg_poly(crc->get_generator_poly()) : PG_CRC_NONE);
  d.max_iterations  = static_cast<uint8_t>(cfg.max_iterations);
  report_fatal_error_if_not(crc == nullptr || d.crc_poly != PG_CRC_NONE,
                            "pusch_b200: unsupported codeblock CRC polynomial.");

  bits.resize(static_cast<size_t>(pg_ldpc_output_bytes(bg, static_cast<int>(z))));
  int32_t iterations = 0;
  ctx.check(pg_ldpc_decode_batch_host(ctx.get(), &d, 1, raw(input), input.size(), bits.data(), bits.size(), &iterations),
            "pg_ldpc_decode_batch_host");
  report_fatal_error_if_not(iterations >= 0, "pusch_b200: invalid LDPC configuration.");

  span<uint8_t> out = output.get_buffer();
  std::memcpy(out.data(), bits.data(), std::min(out.size(), bits.size()));
  if (iterations == 0) {
    return std::nullopt;
  }
  return static_cast<unsigned>(iterations);
}

// ---------------------------------------------------------------------------------------------
// ldpc_rate_dematcher

void ldpc_rate_dematcher_b200::rate_dematch(span<log_likelihood_ratio>       output,
                                            span<const log_likelihood_ratio> input,
                                            bool                             new_data,
                                            const codeblock_metadata&        cfg)
{
  pg_rm_cb d         = {};
  d.in_offset        = 0;
  d.rm_length        = static_cast<uint32_t>(input.size());
  d.out_offset       = 0;
  d.nref             = cfg.tb_common.Nref;
  d.lifting_size     = static_cast<uint16_t>(cfg.tb_common.lifting_size);
  d.nof_filler_bits  = static_cast<uint16_t>(cfg.cb_specific.nof_filler_bits);
  d.base_graph       = static_cast<uint8_t>(to_pg_base_graph(cfg.tb_common.base_graph));
  d.rv               = static_cast<uint8_t>(cfg.tb_common.rv);
  d.modulation_order = static_cast<uint8_t>(get_bits_per_symbol(cfg.tb_common.mod));
  d.new_data         = new_data ? 1 : 0;
  ctx.check(pg_rate_dematch_batch_host(ctx.get(), &d, 1, raw(input), input.size(), raw(output), output.size()),
            "pg_rate_dematch_batch_host");
}

// ---------------------------------------------------------------------------------------------
// crc_calculator

crc_calculator_b200::crc_calculator_b200(const device_config& cfg, crc_generator_poly poly_) :
  ctx(cfg), poly(poly_), pg_poly(to_pg_poly(poly_))
{
  report_fatal_error_if_not(pg_poly != PG_CRC_NONE, "pusch_b200: CRC polynomial {:#x} is not supported.",
                            to_uint(poly_));
}

crc_calculator_checksum_t crc_calculator_b200::run(const uint8_t* packed, size_t nof_bits) const
{
  if (nof_bits == 0) {
    return 0;
  }
  pg_crc_item item = {0, static_cast<uint32_t>(nof_bits), pg_poly};
  uint32_t    crc  = 0;
  ctx.check(pg_crc_calculate_host(ctx.get(), &item, 1, packed, (nof_bits + 7) / 8, &crc), "pg_crc_calculate_host");
  return crc;
}

crc_calculator_checksum_t crc_calculator_b200::calculate_byte(span<const uint8_t> data) const
{
  return run(data.data(), data.size() * 8);
}

crc_calculator_checksum_t crc_calculator_b200::calculate_bit(span<const uint8_t> data) const
{
  dynamic_bit_buffer packed(data.size());
  ocuduvec::bit_pack(packed, data);
  return run(packed.get_buffer().data(), data.size());
}

crc_calculator_checksum_t crc_calculator_b200::calculate(const bit_buffer& data) const
{
  return run(data.get_buffer().data(), data.size());
}

// ---------------------------------------------------------------------------------------------
// demodulation_mapper

void demodulation_mapper_b200::demodulate_soft(span<log_likelihood_ratio> llrs,
                                               span<const cf_t>           symbols,
                                               span<const float>          noise_vars,
                                               modulation_scheme          mod)
{
  const unsigned qm = get_bits_per_symbol(mod);
  report_fatal_error_if_not(mod == modulation_scheme::QPSK || mod == modulation_scheme::QAM16 ||
                                mod == modulation_scheme::QAM64 || mod == modulation_scheme::QAM256,
                            "pusch_b200: modulation {} is not supported.", to_string(mod));
  report_fatal_error_if_not(llrs.size() == symbols.size() * qm && noise_vars.size() == symbols.size(),
                            "pusch_b200: inconsistent demapper buffer sizes.");
  ctx.check(pg_demodulate_soft_host(ctx.get(), static_cast<int>(qm), static_cast<int>(symbols.size()),
                                    reinterpret_cast<const float*>(symbols.data()), noise_vars.data(), raw(llrs)),
            "pg_demodulate_soft_host");
}

// ---------------------------------------------------------------------------------------------
// channel_equalizer

bool channel_equalizer_b200::is_supported(unsigned nof_ports, unsigned nof_layers)
{
  // Zero forcing is implemented for one layer (where it equals the reference's MRC reduction).
  if (type == channel_equalizer_algorithm_type::zf && nof_layers > 1) {
    return false;
  }
  switch (nof_layers) {
    case 1:
      return nof_ports == 1 || nof_ports == 2 || nof_ports == 4 || nof_ports == 8;
    case 2:
      return nof_ports == 2 || nof_ports == 4 || nof_ports == 8;
    case 4:
      return nof_ports == 4 || nof_ports == 8;
    default:
      return false;
  }
}

void channel_equalizer_b200::equalize(span<cf_t>                       eq_symbols,
                                      span<float>                      eq_noise_vars,
                                      const re_buffer_reader<cbf16_t>& ch_symbols,
                                      const ch_est_list&               ch_estimates,
                                      span<const float>                noise_var_estimates,
                                      float                            tx_scaling)
{
  static_assert(sizeof(cbf16_t) == sizeof(uint32_t), "cbf16_t is two bf16 values");
  const unsigned nof_re     = ch_estimates.get_nof_re();
  const unsigned nof_ports  = ch_estimates.get_nof_rx_ports();
  const unsigned nof_layers = ch_estimates.get_nof_tx_layers();
  report_fatal_error_if_not(is_supported(nof_ports, nof_layers), "pusch_b200: {} ports x {} layers not supported.",
                            nof_ports, nof_layers);
  // Gather into the contiguous [port][re] and [port][layer][re] layouts of the C ABI.
  symbols.resize(static_cast<size_t>(nof_ports) * nof_re);
  estimates.resize(static_cast<size_t>(nof_ports) * nof_layers * nof_re);
  for (unsigned p = 0; p != nof_ports; ++p) {
    std::memcpy(symbols.data() + static_cast<size_t>(p) * nof_re, ch_symbols.get_slice(p).data(), nof_re * 4);
    for (unsigned l = 0; l != nof_layers; ++l) {
      std::memcpy(estimates.data() + (static_cast<size_t>(p) * nof_layers + l) * nof_re,
                  ch_estimates.get_channel(p, l).data(),
                  nof_re * 4);
    }
  }
  const int algorithm = type == channel_equalizer_algorithm_type::zf ? PG_EQ_ZF : PG_EQ_MMSE;
  ctx.check(pg_equalize_host(ctx.get(), algorithm, static_cast<int>(nof_re), static_cast<int>(nof_ports),
                             static_cast<int>(nof_layers), symbols.data(), estimates.data(), noise_var_estimates.data(),
                             tx_scaling, reinterpret_cast<float*>(eq_symbols.data()), eq_noise_vars.data()),
            "pg_equalize_host");
}

// ---------------------------------------------------------------------------------------------
// port_channel_estimator

const port_channel_estimator_results& port_channel_estimator_b200::compute(const resource_grid_reader& grid,
                                                                           unsigned                    port,
                                                                           const dmrs_symbol_list&     pilots,
                                                                           const configuration&        cfg)
{
  static_assert(sizeof(cbf16_t) == sizeof(uint32_t), "cbf16_t is two bf16 values");
  report_fatal_error_if_not(!cfg.dmrs_pattern.empty() && cfg.dmrs_pattern.size() <= 2,
                            "pusch_b200: the estimator supports one or two layers.");
  report_fatal_error_if_not(cfg.cp == cyclic_prefix::NORMAL, "pusch_b200: only the normal cyclic prefix is supported.");
  const layer_dmrs_pattern& pattern = cfg.dmrs_pattern.front();
  report_fatal_error_if_not(!pattern.hopping_symbol_index.has_value(), "pusch_b200: frequency hopping not supported.");
  report_fatal_error_if_not(pattern.rb_mask.is_contiguous() && pattern.rb_mask.any(),
                            "pusch_b200: the allocation must be contiguous.");
  for (unsigned k = 0; k != NOF_SUBCARRIERS_PER_RB; ++k) {
    report_fatal_error_if_not(pattern.re_pattern.test(k) == (k % 2 == 0),
                              "pusch_b200: DM-RS type 1, CDM group 0 only.");
  }
  nof_layers             = static_cast<unsigned>(cfg.dmrs_pattern.size());
  const unsigned nd      = static_cast<unsigned>(pattern.symbols.count());
  const unsigned rb0     = static_cast<unsigned>(pattern.rb_mask.find_lowest());
  const unsigned nof_rb  = static_cast<unsigned>(pattern.rb_mask.count());
  const unsigned npil    = 6 * nof_rb;
  const unsigned rx_port = cfg.rx_ports.empty() ? port : cfg.rx_ports[port];
  report_fatal_error_if_not(nd >= 1 && nd <= 2, "pusch_b200: one or two DM-RS symbols.");
  report_fatal_error_if_not(pilots.size().nof_subc == npil && pilots.size().nof_symbols == nd &&
                                pilots.size().nof_slices == nof_layers,
                            "pusch_b200: pilot list does not match the configuration.");

  nof_subc = 12 * nof_rb;
  const unsigned grid_subc = grid.get_nof_subc();
  grid_rows.assign(static_cast<size_t>(MAX_NSYMB_PER_SLOT) * grid_subc, 0);
  uint16_t mask = 0;
  for (unsigned s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
    if (s < pattern.symbols.size() && pattern.symbols.test(s)) {
      mask |= static_cast<uint16_t>(1U << s);
      span<const cbf16_t> row = grid.get_view(rx_port, s);
      std::memcpy(grid_rows.data() + static_cast<size_t>(s) * grid_subc, row.data(), grid_subc * sizeof(cbf16_t));
    }
  }
  pilot_buf.resize(static_cast<size_t>(nd) * nof_layers * npil);
  for (unsigned d = 0; d != nd; ++d) {
    for (unsigned l = 0; l != nof_layers; ++l) {
      span<const cf_t> p = pilots.get_symbol(d, l);
      std::copy(p.begin(), p.end(), pilot_buf.begin() + (static_cast<size_t>(d) * nof_layers + l) * npil);
    }
  }

  pg_port_estimate_cfg pc = {};
  pc.grid_nof_subc        = grid_subc;
  pc.scaling              = cfg.scaling;
  pc.rb_start             = static_cast<uint16_t>(rb0);
  pc.nof_rb               = static_cast<uint16_t>(nof_rb);
  pc.dmrs_symbol_mask     = mask;
  pc.first_symbol         = static_cast<uint8_t>(cfg.first_symbol);
  pc.nof_symbols          = static_cast<uint8_t>(cfg.nof_symbols);
  pc.nof_layers           = static_cast<uint8_t>(nof_layers);
  pc.scs_khz              = static_cast<uint8_t>(scs_to_khz(cfg.scs));
  freq_response.resize(static_cast<size_t>(nd) * nof_layers * nof_subc);
  symbol_estimates.resize(static_cast<size_t>(MAX_NSYMB_PER_SLOT) * nof_layers * nof_subc);
  pg_port_estimate_result r = {};
  ctx.check(pg_port_channel_estimate_host(ctx.get(), &pc, grid_rows.data(), reinterpret_cast<const float*>(pilot_buf.data()),
                                          reinterpret_cast<float*>(freq_response.data()), symbol_estimates.data(), &r),
            "pg_port_channel_estimate_host");
  noise_var = r.noise_var;
  epre      = r.epre;
  snr       = r.snr;
  rsrp      = {r.rsrp[0], r.rsrp[1]};
  cfo_hz    = std::isnan(r.cfo_hz) ? std::nullopt : std::optional<float>(r.cfo_hz);
  // The reference keeps the estimate in a float (port_channel_estimator_average_impl.h:230).
  time_alignment_s = static_cast<float>(r.time_alignment_s);
  return *this;
}

void port_channel_estimator_b200::get_symbol_ch_estimate(span<cbf16_t> symbol, unsigned i_symbol, unsigned tx_layer) const
{
  report_fatal_error_if_not(symbol.size() == nof_subc && i_symbol < MAX_NSYMB_PER_SLOT && tx_layer < nof_layers,
                            "pusch_b200: invalid symbol estimate request.");
  std::memcpy(symbol.data(), symbol_estimates.data() + (static_cast<size_t>(i_symbol) * nof_layers + tx_layer) * nof_subc,
              nof_subc * sizeof(cbf16_t));
}

void port_channel_estimator_b200::get_symbol_ch_estimate(span<cbf16_t>                              symbol,
                                                         unsigned                                   i_symbol,
                                                         unsigned                                   tx_layer,
                                                         const bounded_bitset<MAX_NOF_SUBCARRIERS>& re_mask) const
{
  report_fatal_error_if_not(re_mask.size() == nof_subc && symbol.size() == re_mask.count() &&
                                i_symbol < MAX_NSYMB_PER_SLOT && tx_layer < nof_layers,
                            "pusch_b200: invalid symbol estimate request.");
  const uint32_t* src = symbol_estimates.data() + (static_cast<size_t>(i_symbol) * nof_layers + tx_layer) * nof_subc;
  unsigned        o   = 0;
  re_mask.for_each(0, re_mask.size(), [&](unsigned i_re) { std::memcpy(&symbol[o++], src + i_re, sizeof(cbf16_t)); });
}

// ---------------------------------------------------------------------------------------------
// pusch_decoder

pusch_decoder_b200::pusch_decoder_b200(const device_config& cfg, unsigned max_softbits) :
  ctx(cfg), softbits(max_softbits), cb_stats(MAX_NOF_SEGMENTS, 0)
{
}

pusch_decoder_buffer& pusch_decoder_b200::new_data(span<uint8_t>           transport_block_,
                                                   unique_rx_buffer        rm_buffer_,
                                                   pusch_decoder_notifier& notifier_,
                                                   const configuration&    cfg)
{
  transport_block = transport_block_;
  rm_buffer       = std::move(rm_buffer_);
  notifier        = &notifier_;
  current         = cfg;
  softbits_count  = 0;
  nof_ulsch_softbits.reset();
  if (current.new_data) {
    span<bool> crcs = rm_buffer->get_codeblocks_crc();
    std::fill(crcs.begin(), crcs.end(), false);
  }
  return *this;
}

void pusch_decoder_b200::set_nof_softbits(units::bits nof_softbits)
{
  nof_ulsch_softbits = static_cast<unsigned>(nof_softbits.value());
}

span<log_likelihood_ratio> pusch_decoder_b200::get_next_block_view(unsigned block_size)
{
  report_fatal_error_if_not(softbits_count + block_size <= softbits.size(), "pusch_b200: codeword too long.");
  return span<log_likelihood_ratio>(softbits).subspan(softbits_count, block_size);
}

void pusch_decoder_b200::on_new_softbits(span<const log_likelihood_ratio> in)
{
  span<log_likelihood_ratio> block = get_next_block_view(static_cast<unsigned>(in.size()));
  if (block.data() != in.data()) {
    std::copy(in.begin(), in.end(), block.begin());
  }
  softbits_count += static_cast<unsigned>(in.size());
}

void pusch_decoder_b200::on_end_softbits()
{
  const unsigned qm  = get_bits_per_symbol(current.mod);
  const unsigned G   = softbits_count;
  const unsigned tbs = static_cast<unsigned>(transport_block.size()) * 8;
  const int      bg  = to_pg_base_graph(current.base_graph);
  report_fatal_error_if_not(!nof_ulsch_softbits.has_value() || *nof_ulsch_softbits == G,
                            "pusch_b200: {} soft bits received, {} announced.", G, *nof_ulsch_softbits);
  report_fatal_error_if_not(qm > 0 && G % qm == 0, "pusch_b200: codeword length not a multiple of Qm.");

  pg_sch_segmentation seg = {};
  ctx.check(pg_sch_segment(tbs, bg, static_cast<int>(qm), static_cast<int>(current.nof_layers), G / qm, &seg),
            "pg_sch_segment");
  const unsigned C      = seg.nof_cbs;
  const unsigned Z      = seg.lifting_size;
  const unsigned N      = (bg == 1 ? 66U : 50U) * Z;
  const unsigned K      = (bg == 1 ? 22U : 10U) * Z;
  const unsigned F      = seg.nof_filler_bits;
  const unsigned L      = C > 1 ? 24U : seg.tb_crc_bits;
  const unsigned n_data = K - L - F;
  report_fatal_error_if_not(C == rm_buffer->get_nof_codeblocks(), "pusch_b200: rx buffer holds {} codeblocks, {} needed.",
                            rm_buffer->get_nof_codeblocks(), C);
  span<bool> cb_crcs = rm_buffer->get_codeblocks_crc();

  // Rate dematching of every codeblock into its soft buffer (also those whose CRC already passed:
  // their buffers keep combining, pusch_decoder_impl.cpp:409-423).
  std::vector<pg_rm_cb> rm(C);
  cb_buffers.resize(static_cast<size_t>(C) * N);
  for (unsigned c = 0, off = 0; c != C; ++c) {
    const unsigned e = c < seg.nof_short_cbs ? seg.e_short : seg.e_long;
    rm[c]            = {off, e, c * N, current.Nref, static_cast<uint16_t>(Z), static_cast<uint16_t>(F),
                        static_cast<uint8_t>(bg), static_cast<uint8_t>(current.rv), static_cast<uint8_t>(qm),
                        static_cast<uint8_t>(current.new_data ? 1 : 0)};
    off += e;
    span<log_likelihood_ratio> soft = rm_buffer->get_codeblock_soft_bits(c, N);
    std::memcpy(cb_buffers.data() + static_cast<size_t>(c) * N, soft.data(), N);
  }
  ctx.check(pg_rate_dematch_batch_host(ctx.get(), rm.data(), static_cast<int>(C), raw(span<const log_likelihood_ratio>(softbits).first(G)),
                                       G, cb_buffers.data(), cb_buffers.size()),
            "pg_rate_dematch_batch_host");
  for (unsigned c = 0; c != C; ++c) {
    span<log_likelihood_ratio> soft = rm_buffer->get_codeblock_soft_bits(c, N);
    std::memcpy(soft.data(), cb_buffers.data() + static_cast<size_t>(c) * N, N);
  }

  // LDPC decoding of the codeblocks without a passed CRC.
  const uint32_t poly = C > 1 ? PG_CRC24B : (tbs <= 3824 ? PG_CRC16 : PG_CRC24A);
  std::vector<pg_ldpc_cb> ldpc;
  std::vector<unsigned>   which;
  const unsigned          out_bytes = static_cast<unsigned>(pg_ldpc_output_bytes(bg, static_cast<int>(Z)));
  for (unsigned c = 0; c != C; ++c) {
    if (cb_crcs[c]) {
      continue;
    }
    pg_ldpc_cb d      = {};
    d.llr_offset      = c * N;
    d.nof_llrs        = N;
    d.out_offset      = static_cast<uint32_t>(which.size()) * out_bytes;
    d.lifting_size    = static_cast<uint16_t>(Z);
    d.nof_filler_bits = static_cast<uint16_t>(F);
    d.base_graph      = static_cast<uint8_t>(bg);
    d.crc_poly        = static_cast<uint8_t>(current.use_early_stop ? poly : PG_CRC_NONE);
    d.max_iterations  = static_cast<uint8_t>(current.nof_ldpc_iterations);
    ldpc.push_back(d);
    which.push_back(c);
  }
  if (!ldpc.empty()) {
    cb_bits.assign(static_cast<size_t>(ldpc.size()) * out_bytes, 0);
    std::vector<int32_t> iters(ldpc.size(), 0);
    ctx.check(pg_ldpc_decode_batch_host(ctx.get(), ldpc.data(), static_cast<int>(ldpc.size()), cb_buffers.data(),
                                        cb_buffers.size(), cb_bits.data(), cb_bits.size(), iters.data()),
              "pg_ldpc_decode_batch_host");
    for (size_t i = 0; i != which.size(); ++i) {
      const unsigned c    = which[i];
      const uint8_t* bits = cb_bits.data() + i * out_bytes;
      int            it   = iters[i];
      if (!current.use_early_stop && it > 0) {
        // Without early stop the CRC follows a passed syndrome check (pusch_codeblock_decoder.cpp:50-63).
        pg_crc_item item = {0, K - F, poly};
        uint32_t    crc  = 1;
        ctx.check(pg_crc_calculate_host(ctx.get(), &item, 1, bits, out_bytes, &crc), "pg_crc_calculate_host");
        it = crc == 0 ? static_cast<int>(current.nof_ldpc_iterations) : 0;
      }
      bit_buffer message = rm_buffer->get_codeblock_data_bits(c, K);
      std::memcpy(message.get_buffer().data(), bits, std::min<size_t>(message.get_buffer().size(), out_bytes));
      if (it > 0) {
        cb_crcs[c]  = true;
        cb_stats[c] = static_cast<unsigned>(it);
      } else {
        cb_stats[c] = current.nof_ldpc_iterations;
      }
    }
  }

  // Join (pusch_decoder_impl.cpp:612-781).
  pusch_decoder_result result;
  result.tb_crc_ok            = false;
  result.nof_codeblocks_total = C;
  result.ldpc_decoder_stats.reset();
  for (unsigned c = 0; c != C; ++c) {
    result.ldpc_decoder_stats.update(cb_stats[c]);
  }
  if (C == 1) {
    result.tb_crc_ok = cb_crcs[0];
    if (result.tb_crc_ok) {
      const bit_buffer data = rm_buffer->get_codeblock_data_bits(0, tbs);
      std::memcpy(transport_block.data(), data.get_buffer().data(), transport_block.size());
    }
  } else if (std::all_of(cb_crcs.begin(), cb_crcs.end(), [](bool b) { return b; })) {
    bit_buffer tb_data  = bit_buffer::from_bytes(transport_block);
    unsigned   offset   = 0;
    unsigned   checksum = 0;
    for (unsigned c = 0; c != C; ++c) {
      const unsigned   n_new = std::min(tbs - offset, n_data);
      const bit_buffer data  = rm_buffer->get_codeblock_data_bits(c, n_data);
      ocuduvec::copy_offset(tb_data, offset, data, 0, n_new);
      if (c == C - 1) {
        for (unsigned b = 0; b != 3; ++b) {
          checksum = (checksum << 8U) | data.extract(n_new + b * 8, 8);
        }
      }
      offset += n_new;
    }
    pg_crc_item item = {0, tbs, PG_CRC24A};
    uint32_t    crc  = 0;
    ctx.check(pg_crc_calculate_host(ctx.get(), &item, 1, transport_block.data(), transport_block.size(), &crc),
              "pg_crc_calculate_host");
    if (crc == checksum) {
      result.tb_crc_ok = true;
    } else {
      rm_buffer->reset_codeblocks_crc();
    }
  }
  if (result.tb_crc_ok) {
    rm_buffer.release();
  } else {
    rm_buffer.unlock();
  }
  pusch_decoder_notifier* n = std::exchange(notifier, nullptr);
  n->on_sch_data(result);
}

// ---------------------------------------------------------------------------------------------
// pusch_resident_codeblock_decoder

std::vector<pusch_resident_codeblock_decoder::codeblock_result>
pusch_resident_codeblock_decoder_b200::decode_batch(span<const described_rx_codeblock> codeblock_llrs,
                                                    span<bit_buffer>                   cb_data_buffers,
                                                    span<span<log_likelihood_ratio>>   rm_buffers,
                                                    bool                               new_data,
                                                    crc_generator_poly                 crc_poly,
                                                    bool                               use_early_stop,
                                                    unsigned                           nof_ldpc_iterations)
{
  const size_t n = codeblock_llrs.size();
  report_fatal_error_if_not(cb_data_buffers.size() == n && rm_buffers.size() == n,
                            "pusch_b200: inconsistent batch sizes.");
  std::vector<codeblock_result> out(n);
  if (n == 0) {
    return out;
  }
  // Rate dematching of the batch into the caller's soft buffers (pusch_codeblock_decoder::rate_match).
  std::vector<pg_rm_cb>   rm(n);
  std::vector<int8_t>     in;
  std::vector<uint32_t>   buf_off(n);
  size_t                  total = 0;
  for (size_t i = 0; i != n; ++i) {
    const codeblock_metadata& md = codeblock_llrs[i].second;
    span<const log_likelihood_ratio> e = codeblock_llrs[i].first;
    rm[i]            = {static_cast<uint32_t>(in.size()), static_cast<uint32_t>(e.size()), static_cast<uint32_t>(total),
                        md.tb_common.Nref, static_cast<uint16_t>(md.tb_common.lifting_size),
                        static_cast<uint16_t>(md.cb_specific.nof_filler_bits),
                        static_cast<uint8_t>(to_pg_base_graph(md.tb_common.base_graph)),
                        static_cast<uint8_t>(md.tb_common.rv), static_cast<uint8_t>(get_bits_per_symbol(md.tb_common.mod)),
                        static_cast<uint8_t>(new_data ? 1 : 0)};
    const int8_t* p = raw(e);
    in.insert(in.end(), p, p + e.size());
    buf_off[i] = static_cast<uint32_t>(total);
    total += (rm_buffers[i].size() + 15) & ~static_cast<size_t>(15);
  }
  buffers.assign(total, 0);
  for (size_t i = 0; i != n; ++i) {
    std::memcpy(buffers.data() + buf_off[i], rm_buffers[i].data(), rm_buffers[i].size());
  }
  if (in.empty()) {
    in.push_back(0);
  }
  ctx.check(pg_rate_dematch_batch_host(ctx.get(), rm.data(), static_cast<int>(n), in.data(), in.size(), buffers.data(),
                                       buffers.size()),
            "pg_rate_dematch_batch_host");
  for (size_t i = 0; i != n; ++i) {
    std::memcpy(rm_buffers[i].data(), buffers.data() + buf_off[i], rm_buffers[i].size());
  }
  // LDPC decoding with CRC early stop, or syndrome check then CRC (pusch_codeblock_decoder::decode).
  const uint32_t          poly = to_pg_poly(crc_poly);
  std::vector<pg_ldpc_cb> ldpc(n);
  std::vector<uint32_t>   out_off(n);
  size_t                  bytes = 0;
  for (size_t i = 0; i != n; ++i) {
    const codeblock_metadata& md = codeblock_llrs[i].second;
    const int                 bg = to_pg_base_graph(md.tb_common.base_graph);
    const unsigned            z  = static_cast<unsigned>(md.tb_common.lifting_size);
    ldpc[i]                      = {buf_off[i], static_cast<uint32_t>(rm_buffers[i].size()), static_cast<uint32_t>(bytes),
                                    static_cast<uint16_t>(z), static_cast<uint16_t>(md.cb_specific.nof_filler_bits),
                                    static_cast<uint8_t>(bg), static_cast<uint8_t>(use_early_stop ? poly : PG_CRC_NONE),
                                    static_cast<uint8_t>(nof_ldpc_iterations), 0};
    out_off[i] = static_cast<uint32_t>(bytes);
    bytes += static_cast<size_t>(pg_ldpc_output_bytes(bg, static_cast<int>(z)));
  }
  bits.assign(bytes, 0);
  std::vector<int32_t> iters(n, 0);
  ctx.check(pg_ldpc_decode_batch_host(ctx.get(), ldpc.data(), static_cast<int>(n), buffers.data(), buffers.size(),
                                      bits.data(), bits.size(), iters.data()),
            "pg_ldpc_decode_batch_host");
  for (size_t i = 0; i != n; ++i) {
    const codeblock_metadata& md = codeblock_llrs[i].second;
    const unsigned            k  = (to_pg_base_graph(md.tb_common.base_graph) == 1 ? 22U : 10U) *
                       static_cast<unsigned>(md.tb_common.lifting_size);
    const unsigned obytes = static_cast<unsigned>(
        pg_ldpc_output_bytes(to_pg_base_graph(md.tb_common.base_graph), static_cast<int>(md.tb_common.lifting_size)));
    int it = iters[i];
    if (!use_early_stop && it > 0) {
      pg_crc_item item = {0, k - md.cb_specific.nof_filler_bits, poly};
      uint32_t    crc  = 1;
      ctx.check(pg_crc_calculate_host(ctx.get(), &item, 1, bits.data() + out_off[i], obytes, &crc),
                "pg_crc_calculate_host");
      it = crc == 0 ? static_cast<int>(nof_ldpc_iterations) : 0;
    }
    span<uint8_t> dst = cb_data_buffers[i].get_buffer();
    std::memcpy(dst.data(), bits.data() + out_off[i], std::min<size_t>(dst.size(), obytes));
    out[i].crc_ok         = it > 0;
    out[i].nof_iterations = it > 0 ? static_cast<unsigned>(it) : nof_ldpc_iterations;
  }
  timing.nof_cbs = static_cast<unsigned>(n);
  return out;
}

void pusch_resident_codeblock_decoder_b200::rate_dematch_only(span<const log_likelihood_ratio> cb_llrs,
                                                              span<log_likelihood_ratio>       rm_buffer,
                                                              bool                             new_data,
                                                              const codeblock_metadata&        md)
{
  pg_rm_cb d = {0, static_cast<uint32_t>(cb_llrs.size()), 0, md.tb_common.Nref,
                static_cast<uint16_t>(md.tb_common.lifting_size), static_cast<uint16_t>(md.cb_specific.nof_filler_bits),
                static_cast<uint8_t>(to_pg_base_graph(md.tb_common.base_graph)), static_cast<uint8_t>(md.tb_common.rv),
                static_cast<uint8_t>(get_bits_per_symbol(md.tb_common.mod)), static_cast<uint8_t>(new_data ? 1 : 0)};
  ctx.check(pg_rate_dematch_batch_host(ctx.get(), &d, 1, raw(cb_llrs), cb_llrs.size(), raw(rm_buffer), rm_buffer.size()),
            "pg_rate_dematch_batch_host");
}

pusch_resident_codeblock_decoder::tb_decode_result pusch_resident_codeblock_decoder_b200::decode_resident_softbits(
    void*                                                resident_llrs,
    size_t                                               nof_softbits,
    const scrambling_config*                             scrambling_cfg,
    const codeblock_metadata::tb_common_metadata&        tb_common,
    span<const codeblock_metadata::cb_specific_metadata> cb_specific,
    span<uint8_t>                                        tb_output,
    crc_generator_poly                                   cb_crc_poly,
    unsigned                                             nof_ldpc_iterations,
    void*                                                execution_context,
    int                                                  buffer_index)
{
  (void)cb_crc_poly; // implied by the transport block size and the codeblock count
  (void)execution_context;
  (void)buffer_index;
  const unsigned qm = get_bits_per_symbol(tb_common.mod);
  report_fatal_error_if_not(qm > 0 && nof_softbits % qm == 0 && !cb_specific.empty(),
                            "pusch_b200: invalid resident codeword.");
  // The layer count is not part of the metadata: take the one whose TS 38.212 split reproduces the
  // codeblocks' rate-matching lengths.
  const unsigned tbs = static_cast<unsigned>(tb_output.size()) * 8;
  const int      bg  = to_pg_base_graph(tb_common.base_graph);
  unsigned       nl  = 0;
  for (unsigned l = 1; l <= 4 && nl == 0; ++l) {
    pg_sch_segmentation sg = {};
    if ((nof_softbits / qm) % l != 0 ||
        pg_sch_segment(tbs, bg, static_cast<int>(qm), static_cast<int>(l), static_cast<uint32_t>(nof_softbits / qm), &sg) !=
            PG_OK ||
        sg.nof_cbs != cb_specific.size()) {
      continue;
    }
    bool match = true;
    for (unsigned c = 0; c != sg.nof_cbs; ++c) {
      match = match && cb_specific[c].rm_length == (c < sg.nof_short_cbs ? sg.e_short : sg.e_long);
    }
    nl = match ? l : 0;
  }
  report_fatal_error_if_not(nl != 0, "pusch_b200: codeblock lengths match no layer count.");
  pg_sch_tb tb      = {};
  tb.llr_offset     = 0;
  tb.nof_ch_symbols = static_cast<uint32_t>(nof_softbits / qm);
  tb.tbs_bits       = tbs;
  tb.tb_out_offset  = 0;
  tb.nref           = tb_common.Nref;
  tb.base_graph     = static_cast<uint8_t>(bg);
  tb.modulation_order = static_cast<uint8_t>(qm);
  tb.nof_layers       = static_cast<uint8_t>(nl);
  tb.rv               = static_cast<uint8_t>(tb_common.rv);
  tb.max_iterations   = static_cast<uint8_t>(nof_ldpc_iterations);
  uint32_t c_init = 0, offset = 0;
  if (scrambling_cfg != nullptr) {
    // TS 38.211 Section 6.3.1.1 (PUSCH): c_init = n_RNTI 2^15 + n_ID.
    c_init = (static_cast<uint32_t>(scrambling_cfg->n_rnti) << 15) + (static_cast<uint32_t>(scrambling_cfg->q) << 14) +
             scrambling_cfg->n_id;
    offset = scrambling_cfg->bit_offset;
  }
  pg_sch_result r = {};
  ctx.check(pg_sch_decode_batch_resident(ctx.get(), &tb, 1, static_cast<const int8_t*>(resident_llrs), nof_softbits,
                                         scrambling_cfg != nullptr ? &c_init : nullptr,
                                         scrambling_cfg != nullptr ? &offset : nullptr, tb_output.data(),
                                         tb_output.size(), &r),
            "pg_sch_decode_batch_resident");
  timing.nof_cbs = r.nof_cbs;
  return {r.tb_crc_ok != 0, r.nof_cbs_crc_ok == r.nof_cbs, static_cast<unsigned>(std::lround(r.mean_iterations))};
}

void pusch_resident_codeblock_decoder_b200::set_ldpc_decoder_algorithm(const std::string& algorithm)
{
  report_fatal_error_if_not(algorithm.empty() || algorithm == "layered_min_sum",
                            "pusch_b200: LDPC algorithm '{}' is not supported.", algorithm);
}

// ---------------------------------------------------------------------------------------------
// Factories

namespace {

class ldpc_decoder_factory_b200 : public ldpc_decoder_factory
{
public:
  explicit ldpc_decoder_factory_b200(const device_config& dev_) : dev(dev_) {}
  std::unique_ptr<ldpc_decoder> create() override { return std::make_unique<ldpc_decoder_b200>(dev); }

private:
  device_config dev;
};

class ldpc_rate_dematcher_factory_b200 : public ldpc_rate_dematcher_factory
{
public:
  explicit ldpc_rate_dematcher_factory_b200(const device_config& dev_) : dev(dev_) {}
  std::unique_ptr<ldpc_rate_dematcher> create() override { return std::make_unique<ldpc_rate_dematcher_b200>(dev); }

private:
  device_config dev;
};

class crc_calculator_factory_b200 : public crc_calculator_factory
{
public:
  explicit crc_calculator_factory_b200(const device_config& dev_) : dev(dev_) {}
  std::unique_ptr<crc_calculator> create(crc_generator_poly poly) override
  {
    return std::make_unique<crc_calculator_b200>(dev, poly);
  }

private:
  device_config dev;
};

class demodulation_mapper_factory_b200 : public demodulation_mapper_factory
{
public:
  explicit demodulation_mapper_factory_b200(const device_config& dev_) : dev(dev_) {}
  std::unique_ptr<demodulation_mapper> create() override { return std::make_unique<demodulation_mapper_b200>(dev); }

private:
  device_config dev;
};

class channel_equalizer_factory_b200 : public channel_equalizer_factory
{
public:
  channel_equalizer_factory_b200(const device_config& dev_, channel_equalizer_algorithm_type type_) :
    dev(dev_), type(type_)
  {
  }
  std::unique_ptr<channel_equalizer> create() override { return std::make_unique<channel_equalizer_b200>(dev, type); }

private:
  device_config                    dev;
  channel_equalizer_algorithm_type type;
};

class port_channel_estimator_factory_b200 : public port_channel_estimator_factory
{
public:
  explicit port_channel_estimator_factory_b200(const device_config& dev_) : dev(dev_) {}
  std::unique_ptr<port_channel_estimator> create(port_channel_estimator_fd_smoothing_strategy     fd,
                                                 port_channel_estimator_td_interpolation_strategy td,
                                                 bool                                             compensate_cfo) override
  {
    if (fd != port_channel_estimator_fd_smoothing_strategy::filter ||
        td != port_channel_estimator_td_interpolation_strategy::interpolate || compensate_cfo) {
      return nullptr;
    }
    return std::make_unique<port_channel_estimator_b200>(dev);
  }

private:
  device_config dev;
};

class pusch_decoder_factory_b200 : public pusch_decoder_factory
{
public:
  pusch_decoder_factory_b200(const device_config& dev_, unsigned max_softbits_) : dev(dev_), max_softbits(max_softbits_)
  {
  }
  std::unique_ptr<pusch_decoder> create() override { return std::make_unique<pusch_decoder_b200>(dev, max_softbits); }

private:
  device_config dev;
  unsigned      max_softbits;
};

} // namespace

std::shared_ptr<port_channel_estimator_factory> create_port_channel_estimator_factory_b200(const device_config& dev)
{
  return std::make_shared<port_channel_estimator_factory_b200>(dev);
}

std::shared_ptr<pusch_decoder_factory>
create_pusch_decoder_factory_b200(const device_config& dev, unsigned max_nof_prb, unsigned max_nof_layers)
{
  return std::make_shared<pusch_decoder_factory_b200>(
      dev, static_cast<unsigned>(pusch_constants::get_max_codeword_size(max_nof_prb, max_nof_layers).value()));
}

std::shared_ptr<ldpc_decoder_factory>
create_ldpc_decoder_factory_b200(const device_config&                                            dev,
                                 const ldpc_decoder_factory::ldpc_decoder_factory_configuration& cfg)
{
  // The GPU decoder implements the reference's default decision rules: CRC early stop, or a
  // syndrome check after the last iteration; inputs shorter than the message are not decoded.
  if (cfg.force_decoding || cfg.early_stop_syndrome) {
    return nullptr;
  }
  return std::make_shared<ldpc_decoder_factory_b200>(dev);
}

std::shared_ptr<ldpc_rate_dematcher_factory> create_ldpc_rate_dematcher_factory_b200(const device_config& dev)
{
  return std::make_shared<ldpc_rate_dematcher_factory_b200>(dev);
}

std::shared_ptr<crc_calculator_factory> create_crc_calculator_factory_b200(const device_config& dev)
{
  return std::make_shared<crc_calculator_factory_b200>(dev);
}

std::shared_ptr<demodulation_mapper_factory> create_demodulation_mapper_factory_b200(const device_config& dev)
{
  return std::make_shared<demodulation_mapper_factory_b200>(dev);
}

std::shared_ptr<channel_equalizer_factory> create_channel_equalizer_factory_b200(const device_config&             dev,
                                                                               channel_equalizer_algorithm_type type)
{
  return std::make_shared<channel_equalizer_factory_b200>(dev, type);
}

} // namespace b200
} // namespace ocudu

// Implementation of the reference-interface adapters over the pusch_b200 C ABI.
#include "b200_phy_adapters.h"

#include "../../include/pusch_b200.h"
#include "ocudu/ocuduvec/bit.h"
#include "ocudu/ran/sch/modulation_scheme.h"
#include "ocudu/support/error_handling.h"

#include <algorithm>
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

} // namespace

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

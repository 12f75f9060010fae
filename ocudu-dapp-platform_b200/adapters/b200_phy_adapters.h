// C++17 adapters that implement the reference's PHY interfaces on top of the pusch_b200 C ABI
// (include/pusch_b200.h). They are the binding a maintainer adds to the reference tree: each
// class derives from the reference's abstract interface, translates its arguments into the flat
// C structures and calls the library; the factories slot into the reference's factory wiring
// (lib/phy/upper/upper_phy_factories.cpp:807-953) in place of the *_sw factories.
//
// Every adapter instance owns one pg_context (a CUDA stream and its device buffers on one
// device): like the reference's objects, an instance is used by one thread at a time, and the
// factories hand one instance to each worker. Failures of the library (no device, a CUDA error,
// an unsupported configuration) end the process through report_fatal_error: there is no CPU
// fallback behind these classes.
#pragma once

#include "ocudu/phy/upper/channel_coding/channel_coding_factories.h"
#include "ocudu/phy/upper/channel_coding/crc_calculator.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h"
#include "ocudu/phy/upper/channel_modulation/channel_modulation_factories.h"
#include "ocudu/phy/upper/channel_modulation/demodulation_mapper.h"
#include "ocudu/phy/upper/equalization/channel_equalizer.h"
#include "ocudu/phy/upper/equalization/equalization_factories.h"

#include <memory>
#include <vector>

struct pg_context;

namespace ocudu {
namespace b200 {

/// Device and capacity of the contexts the factories create.
struct device_config {
  /// CUDA device ordinal.
  int device = 0;
  /// Largest LDPC batch per call (one codeblock per call through ldpc_decoder::decode).
  int max_codeblocks = 64;
};

/// One pg_context; closes it on destruction.
class context_handle
{
public:
  explicit context_handle(const device_config& cfg);
  ~context_handle();
  context_handle(const context_handle&)            = delete;
  context_handle& operator=(const context_handle&) = delete;

  pg_context* get() const { return ctx; }
  /// Ends the process with the library's error text when rc is not PG_OK.
  void check(int rc, const char* what) const;

private:
  pg_context* ctx = nullptr;
};

/// ldpc_decoder (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_decoder.h:19-58) on the GPU
/// decoder: same bits and the same optional iteration count as the AVX-512/AVX2 decoders.
class ldpc_decoder_b200 : public ldpc_decoder
{
public:
  explicit ldpc_decoder_b200(const device_config& cfg) : ctx(cfg) {}

  std::optional<unsigned>
  decode(bit_buffer& output, span<const log_likelihood_ratio> input, crc_calculator* crc, const configuration& cfg)
      override;

private:
  context_handle       ctx;
  std::vector<uint8_t> bits;
};

/// ldpc_rate_dematcher (include/ocudu/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher.h:17-40).
class ldpc_rate_dematcher_b200 : public ldpc_rate_dematcher
{
public:
  explicit ldpc_rate_dematcher_b200(const device_config& cfg) : ctx(cfg) {}

  void rate_dematch(span<log_likelihood_ratio>       output,
                    span<const log_likelihood_ratio> input,
                    bool                             new_data,
                    const codeblock_metadata&        cfg) override;

private:
  context_handle ctx;
};

/// crc_calculator (include/ocudu/phy/upper/channel_coding/crc_calculator.h:59-81) for the three
/// polynomials of the shared channel: CRC16, CRC24A and CRC24B.
class crc_calculator_b200 : public crc_calculator
{
public:
  crc_calculator_b200(const device_config& cfg, crc_generator_poly poly);

  crc_calculator_checksum_t calculate_byte(span<const uint8_t> data) const override;
  crc_calculator_checksum_t calculate_bit(span<const uint8_t> data) const override;
  crc_calculator_checksum_t calculate(const bit_buffer& data) const override;
  crc_generator_poly        get_generator_poly() const override { return poly; }

private:
  crc_calculator_checksum_t run(const uint8_t* packed, size_t nof_bits) const;

  context_handle     ctx;
  crc_generator_poly poly;
  uint32_t           pg_poly;
};

/// demodulation_mapper (include/ocudu/phy/upper/channel_modulation/demodulation_mapper.h:28-52)
/// for QPSK, 16QAM, 64QAM and 256QAM.
class demodulation_mapper_b200 : public demodulation_mapper
{
public:
  explicit demodulation_mapper_b200(const device_config& cfg) : ctx(cfg) {}

  void demodulate_soft(span<log_likelihood_ratio> llrs,
                       span<const cf_t>           symbols,
                       span<const float>          noise_vars,
                       modulation_scheme          mod) override;

private:
  context_handle ctx;
};

/// channel_equalizer (include/ocudu/phy/upper/equalization/channel_equalizer.h:20-77): one layer
/// with 1, 2, 4 or 8 receive ports, two layers with 2, 4 or 8, four layers with 4 or 8 (MMSE).
class channel_equalizer_b200 : public channel_equalizer
{
public:
  channel_equalizer_b200(const device_config& cfg, channel_equalizer_algorithm_type type_) : ctx(cfg), type(type_) {}

  bool is_supported(unsigned nof_ports, unsigned nof_layers) override;

  void equalize(span<cf_t>                       eq_symbols,
                span<float>                      eq_noise_vars,
                const re_buffer_reader<cbf16_t>& ch_symbols,
                const ch_est_list&               ch_estimates,
                span<const float>                noise_var_estimates,
                float                            tx_scaling) override;

private:
  context_handle                   ctx;
  channel_equalizer_algorithm_type type;
  std::vector<uint32_t>            symbols, estimates;
};

/// Factories in the shape of the reference's *_sw factories.
std::shared_ptr<ldpc_decoder_factory>
create_ldpc_decoder_factory_b200(const device_config&                                            dev,
                                 const ldpc_decoder_factory::ldpc_decoder_factory_configuration& cfg);
std::shared_ptr<ldpc_rate_dematcher_factory> create_ldpc_rate_dematcher_factory_b200(const device_config& dev);
std::shared_ptr<crc_calculator_factory>      create_crc_calculator_factory_b200(const device_config& dev);
std::shared_ptr<demodulation_mapper_factory> create_demodulation_mapper_factory_b200(const device_config& dev);
std::shared_ptr<channel_equalizer_factory>
create_channel_equalizer_factory_b200(const device_config& dev, channel_equalizer_algorithm_type type);

} // namespace b200
} // namespace ocudu

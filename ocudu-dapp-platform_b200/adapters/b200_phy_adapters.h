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
#include "ocudu/phy/upper/channel_processors/pusch/factories.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_buffer.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_resident_codeblock_decoder.h"
#include "ocudu/phy/upper/signal_processors/channel_estimator/factories.h"
#include "ocudu/phy/upper/signal_processors/channel_estimator/port_channel_estimator.h"
#include "ocudu/phy/upper/unique_rx_buffer.h"

#include <array>
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

/// port_channel_estimator (include/ocudu/phy/upper/signal_processors/channel_estimator/
/// port_channel_estimator.h:63-139) with frequency smoothing "filter", time interpolation
/// "interpolate" and no CFO compensation: one port per compute() call, on the GPU entry
/// pg_port_channel_estimate_host, with the pilots the caller gives (dmrs_pusch_estimator's). It is
/// also its own results object, valid until the next compute(). Supported: DM-RS type 1, CDM group
/// 0 (one or two layers), one or two DM-RS symbols, contiguous resource blocks, no frequency hopping,
/// normal cyclic prefix; anything else ends the process.
class port_channel_estimator_b200 : public port_channel_estimator, private port_channel_estimator_results
{
public:
  explicit port_channel_estimator_b200(const device_config& cfg) : ctx(cfg) {}

  const port_channel_estimator_results&
  compute(const resource_grid_reader& grid, unsigned port, const dmrs_symbol_list& pilots, const configuration& cfg)
      override;

private:
  void  get_symbol_ch_estimate(span<cbf16_t> symbol, unsigned i_symbol, unsigned tx_layer) const override;
  void  get_symbol_ch_estimate(span<cbf16_t>                              symbol,
                               unsigned                                   i_symbol,
                               unsigned                                   tx_layer,
                               const bounded_bitset<MAX_NOF_SUBCARRIERS>& re_mask) const override;
  float get_epre() const override { return epre; }
  float get_noise_variance() const override { return noise_var; }
  float get_snr() const override { return snr; }
  float get_rsrp(unsigned tx_layer) const override { return rsrp[tx_layer]; }
  std::optional<float> get_cfo_Hz() const override { return cfo_hz; }
  phy_time_unit        get_time_alignment() const override { return phy_time_unit::from_seconds(time_alignment_s); }

  context_handle        ctx;
  std::vector<uint32_t> grid_rows, symbol_estimates;
  std::vector<cf_t>     pilot_buf, freq_response;
  unsigned              nof_layers = 1, nof_subc = 0;
  float                 noise_var = 0, epre = 0, snr = 0;
  std::array<float, 2>  rsrp     = {};
  std::optional<float>  cfo_hz;
  float                 time_alignment_s = 0;
};

/// pusch_decoder (include/ocudu/phy/upper/channel_processors/pusch/pusch_decoder.h:38-145): the soft
/// bits arrive through the pusch_decoder_buffer interface and, at on_end_softbits(), every codeblock
/// of the transport block is rate dematched into its rx_buffer soft buffer (saturating combination
/// for retransmissions) and the ones without a passed CRC are LDPC decoded, in one GPU batch each;
/// then the TB is joined, its CRC checked on the GPU and the notifier called, with the reference's
/// rules for the codeblock CRC flags, the decoded-bit storage and the iteration statistics
/// (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:80-145, :390-477, :612-781).
/// Decoding completes inside on_end_softbits() (the reference's synchronous mode, no executor).
class pusch_decoder_b200 : public pusch_decoder, private pusch_decoder_buffer
{
public:
  /// max_softbits: the largest codeword (G) of one transport block.
  pusch_decoder_b200(const device_config& cfg, unsigned max_softbits);

  pusch_decoder_buffer& new_data(span<uint8_t>           transport_block,
                                 unique_rx_buffer        rm_buffer,
                                 pusch_decoder_notifier& notifier,
                                 const configuration&    cfg) override;
  void                  set_nof_softbits(units::bits nof_softbits) override;

private:
  span<log_likelihood_ratio> get_next_block_view(unsigned block_size) override;
  void                       on_new_softbits(span<const log_likelihood_ratio> softbits) override;
  void                       on_end_softbits() override;

  context_handle                    ctx;
  std::vector<log_likelihood_ratio> softbits;
  unsigned                          softbits_count = 0;
  std::optional<unsigned>           nof_ulsch_softbits;
  span<uint8_t>                     transport_block;
  unique_rx_buffer                  rm_buffer;
  pusch_decoder_notifier*           notifier = nullptr;
  configuration                     current;
  /// Iterations of each codeblock index, kept across transport blocks as the reference keeps them.
  std::vector<unsigned> cb_stats;
  std::vector<int8_t>   cb_buffers;
  std::vector<uint8_t>  cb_bits;
};

/// pusch_resident_codeblock_decoder (include/ocudu/phy/upper/channel_processors/pusch/
/// pusch_resident_codeblock_decoder.h:61-150), the batch hook of pusch_decoder_impl
/// (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:492-600): decode_batch dematches
/// every codeblock into its host soft buffer and decodes them in one GPU batch each;
/// decode_resident_softbits decodes a transport block whose soft bits are already in device memory
/// (int8 LLRs, descrambled on the device when a scrambling configuration is given) through
/// pg_sch_decode_batch_resident. The dematched soft bits of a resident decode stay in the library's
/// scratch, so export_resident_softbits reports that none can be exported (the interface's contract
/// for that case: the caller resets the HARQ buffers).
class pusch_resident_codeblock_decoder_b200 : public pusch_resident_codeblock_decoder
{
public:
  explicit pusch_resident_codeblock_decoder_b200(const device_config& cfg) : ctx(cfg) {}

  std::vector<codeblock_result> decode_batch(span<const described_rx_codeblock> codeblock_llrs,
                                             span<bit_buffer>                   cb_data_buffers,
                                             span<span<log_likelihood_ratio>>   rm_buffers,
                                             bool                               new_data,
                                             crc_generator_poly                 crc_poly,
                                             bool                               use_early_stop,
                                             unsigned                           nof_ldpc_iterations) override;
  void rate_dematch_only(span<const log_likelihood_ratio> cb_llrs,
                         span<log_likelihood_ratio>       rm_buffer,
                         bool                             new_data,
                         const codeblock_metadata&        metadata) override;
  bool export_resident_softbits(span<span<log_likelihood_ratio>> rm_buffers) override { return false; }
  tb_decode_result decode_resident_softbits(void*                                                resident_llrs,
                                            size_t                                               nof_softbits,
                                            const scrambling_config*                             scrambling_cfg,
                                            const codeblock_metadata::tb_common_metadata&        tb_common,
                                            span<const codeblock_metadata::cb_specific_metadata> cb_specific,
                                            span<uint8_t>                                        tb_output,
                                            crc_generator_poly                                   cb_crc_poly,
                                            unsigned                                             nof_ldpc_iterations,
                                            void*                                                execution_context,
                                            int                                                  buffer_index) override;
  const pusch_resident_codeblock_decoder_timing_stats& get_last_timing_stats() const override { return timing; }
  void set_demod_timing(float grid_staging_us, float demod_sync_us) override
  {
    timing.grid_staging_us = grid_staging_us;
    timing.demod_sync_us   = demod_sync_us;
  }
  void set_timing_enabled(bool enable) override { timing.timing_enabled = enable; }
  /// "" or "layered_min_sum" (the only algorithm: the reference's layered normalised min-sum).
  void set_ldpc_decoder_algorithm(const std::string& algorithm) override;

private:
  context_handle                                 ctx;
  pusch_resident_codeblock_decoder_timing_stats  timing;
  std::vector<int8_t>                            buffers;
  std::vector<uint8_t>                           bits;
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
/// Estimators with FD "filter", TD "interpolate" and no CFO compensation; other strategies give nullptr.
std::shared_ptr<port_channel_estimator_factory> create_port_channel_estimator_factory_b200(const device_config& dev);
/// Decoders for codewords of up to the largest PUSCH codeword of max_nof_prb PRBs and max_nof_layers layers.
std::shared_ptr<pusch_decoder_factory>
create_pusch_decoder_factory_b200(const device_config& dev, unsigned max_nof_prb, unsigned max_nof_layers);

} // namespace b200
} // namespace ocudu

// Test infrastructure only (checker, never shipped): the two factories the reference's offline
// replay tool (apps/tools/pusch_replay/ocudu_pusch_replay.cpp) takes from
// lib/phy/upper/channel_processors/pusch/processor_factories.cpp, built here without that file
// (which pulls in the whole PUSCH processor and the hardware decoders): the software PUSCH decoder
// over the caller's CRC / LDPC / dematcher / segmenter factories with one codeblock decoder, and
// the software UL-SCH demultiplexer. This lets oracle/Makefile compile the tool's own source, as it
// lies in the reference checkout, into oracle/_ref/ocudu_pusch_replay.
#include "lib/phy/upper/channel_processors/pusch/pusch_codeblock_decoder.h"
#include "lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.h"
#include "lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.h"
#include "ocudu/phy/upper/channel_processors/pusch/factories.h"
#include <memory>
#include <vector>

using namespace ocudu;

namespace {

class replay_decoder_factory : public pusch_decoder_factory
{
public:
  explicit replay_decoder_factory(pusch_decoder_factory_sw_configuration c) : cfg(std::move(c))
  {
    std::vector<std::unique_ptr<pusch_codeblock_decoder>> decoders(1);
    pusch_codeblock_decoder::sch_crc                      crcs{cfg.crc_factory->create(crc_generator_poly::CRC16),
                                          cfg.crc_factory->create(crc_generator_poly::CRC24A),
                                          cfg.crc_factory->create(crc_generator_poly::CRC24B)};
    decoders[0] = std::make_unique<pusch_codeblock_decoder>(cfg.dematcher_factory->create(),
                                                            cfg.decoder_factory->create(), crcs);
    pool        = std::make_shared<pusch_decoder_impl::codeblock_decoder_pool>(decoders);
  }
  std::unique_ptr<pusch_decoder> create() override
  {
    return std::make_unique<pusch_decoder_impl>(
        cfg.segmenter_factory->create(), pool,
        pusch_decoder_impl::sch_crc{cfg.crc_factory->create(crc_generator_poly::CRC16),
                                    cfg.crc_factory->create(crc_generator_poly::CRC24A),
                                    cfg.crc_factory->create(crc_generator_poly::CRC24B)},
        cfg.executor, cfg.nof_prb, cfg.nof_layers);
  }

private:
  pusch_decoder_factory_sw_configuration                     cfg;
  std::shared_ptr<pusch_decoder_impl::codeblock_decoder_pool> pool;
};

class replay_demux_factory : public ulsch_demultiplex_factory
{
public:
  std::unique_ptr<ulsch_demultiplex> create() override { return std::make_unique<ulsch_demultiplex_impl>(); }
};

} // namespace

std::shared_ptr<pusch_decoder_factory> ocudu::create_pusch_decoder_factory_sw(pusch_decoder_factory_sw_configuration config)
{
  return std::make_shared<replay_decoder_factory>(std::move(config));
}

std::shared_ptr<ulsch_demultiplex_factory> ocudu::create_ulsch_demultiplex_factory_sw()
{
  return std::make_shared<replay_demux_factory>();
}

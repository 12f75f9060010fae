// Test infrastructure only (checker, never shipped): a flat C ABI over the reference's own CPU
// implementation of UCI on PUSCH, so tests can call it through ctypes:
//   ulsch_demultiplex::demultiplex     include/ocudu/phy/upper/channel_processors/pusch/ulsch_demultiplex.h:31-90
//                                      (lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.cpp)
//   short_block_detector::detect       include/ocudu/phy/upper/channel_coding/short/short_block_detector.h
//   short_block_encoder::encode        include/ocudu/phy/upper/channel_coding/short/short_block_encoder.h
// The scrambling sequence handed to the demultiplexer is the reference's own pseudo-random
// generator output for c_init, as pusch_demodulator_impl produces it.

#include "lib/phy/upper/channel_coding/short/short_block_detector_impl.h"
#include "lib/phy/upper/channel_coding/short/short_block_encoder_impl.h"
#include "lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.h"
#include "ocudu/adt/bit_buffer.h"
#include "ocudu/ocuduvec/bit.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_buffer.h"
#include "ocudu/phy/upper/sequence_generators/sequence_generator_factories.h"
#include "ocudu/ran/pusch/ulsch_info.h"
#include "ocudu/ran/uci/uci_info.h"
#include <cstring>
#include <memory>
#include <vector>

using namespace ocudu;

namespace {

// Collects every soft bit notified to a decoder buffer.
class collect_buffer : public pusch_decoder_buffer
{
public:
  std::vector<log_likelihood_ratio> data;
  std::vector<log_likelihood_ratio> view;
  bool                              ended = false;

  span<log_likelihood_ratio> get_next_block_view(unsigned block_size) override
  {
    view.resize(block_size);
    return view;
  }
  void on_new_softbits(span<const log_likelihood_ratio> softbits) override
  {
    data.insert(data.end(), softbits.begin(), softbits.end());
  }
  void on_end_softbits() override { ended = true; }
};

modulation_scheme mod_from_qm(int qm)
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

int copy_out(const collect_buffer& b, int8_t* out, int cap)
{
  const int n = (int)b.data.size();
  for (int i = 0; i < n && i < cap; ++i) {
    out[i] = (int8_t)b.data[i].to_int();
  }
  return n;
}

} // namespace

extern "C" {

// Demultiplexes one codeword of descrambled soft bits (G of them) through the reference, fed in
// blocks of block_size soft bits. Writes the SCH, HARQ-ACK and CSI Part 1 streams (caps in soft
// bits) and their lengths to lens[0..2]; lens[3] = 1 if both UCI buffers were closed.
int ref_ulsch_demultiplex(int qm, int nof_layers, int nof_prb, int start_symbol, int nof_symbols, int dmrs_mask,
                          int dmrs_type, int nof_cdm_groups_without_data, int nof_harq_ack_rvd, int nof_harq_ack_bits,
                          int nof_enc_harq_ack_bits, int nof_csi_part1_bits, int nof_enc_csi_part1_bits,
                          uint32_t c_init, const int8_t* llrs, int G, int block_size, int8_t* sch, int sch_cap,
                          int8_t* ack, int ack_cap, int8_t* csi1, int csi1_cap, int* lens)
{
  ulsch_demultiplex::configuration cfg;
  cfg.modulation         = mod_from_qm(qm);
  cfg.nof_layers         = nof_layers;
  cfg.nof_prb            = nof_prb;
  cfg.start_symbol_index = start_symbol;
  cfg.nof_symbols        = nof_symbols;
  cfg.nof_harq_ack_rvd   = nof_harq_ack_rvd;
  cfg.dmrs               = dmrs_type == 2 ? dmrs_config_type::type2 : dmrs_config_type::type1;
  cfg.dmrs_symbol_mask   = symbol_slot_mask(14);
  for (int s = 0; s < 14; ++s) {
    if ((dmrs_mask >> s) & 1) {
      cfg.dmrs_symbol_mask.set(s);
    }
  }
  cfg.nof_cdm_groups_without_data = nof_cdm_groups_without_data;
  cfg.nof_harq_ack_bits           = nof_harq_ack_bits;
  cfg.nof_enc_harq_ack_bits       = nof_enc_harq_ack_bits;
  cfg.nof_csi_part1_bits          = nof_csi_part1_bits;
  cfg.nof_enc_csi_part1_bits      = nof_enc_csi_part1_bits;

  // Scrambling sequence of the codeword (c_init), packed.
  auto                      prg_factory = create_pseudo_random_generator_sw_factory();
  auto                      prg         = prg_factory->create();
  dynamic_bit_buffer        seq(G);
  prg->init(c_init);
  prg->generate(seq);

  collect_buffer b_sch, b_ack, b_csi1;
  // Value-initialised, as the reference's factory creates it (std::make_unique): the soft-bit
  // count of the current symbol starts at zero.
  auto                   demux = std::make_unique<ulsch_demultiplex_impl>();
  pusch_codeword_buffer& cw    = demux->demultiplex(b_sch, b_ack, b_csi1, cfg);
  std::vector<log_likelihood_ratio> in(G);
  for (int i = 0; i < G; ++i) {
    in[i] = llrs[i];
  }
  std::vector<uint8_t> seq_bits(G);
  ocuduvec::bit_unpack(seq_bits, seq);
  int pos = 0;
  while (pos < G) {
    const unsigned             want = (unsigned)std::min(block_size, G - pos);
    span<log_likelihood_ratio> view = cw.get_next_block_view(want);
    const unsigned             n    = (unsigned)view.size();
    if (n == 0) {
      break; // the demultiplexer takes no more soft bits (an allocation that starts with a symbol without data)
    }
    std::memcpy(view.data(), in.data() + pos, n);
    dynamic_bit_buffer blk(n);
    ocuduvec::bit_pack(blk, span<const uint8_t>(seq_bits.data() + pos, n));
    cw.on_new_block(view, blk);
    pos += (int)n;
  }
  if (pos == G) {
    cw.on_end_codeword();
  }
  lens[0] = copy_out(b_sch, sch, sch_cap);
  lens[1] = copy_out(b_ack, ack, ack_cap);
  lens[2] = copy_out(b_csi1, csi1, csi1_cap);
  lens[3] = pos == G && (nof_harq_ack_bits == 0 || b_ack.ended) && (nof_csi_part1_bits == 0 || b_csi1.ended) ? 1 : 0;
  return 0;
}

// Encodes a K-bit UCI message (1..11 bits) into E bits for modulation order qm (placeholders of
// 1- and 2-bit messages as the reference's values).
int ref_short_block_encode(int K, const uint8_t* msg, int E, int qm, uint8_t* out)
{
  short_block_encoder_impl enc;
  enc.encode(span<uint8_t>(out, E), span<const uint8_t>(msg, K), mod_from_qm(qm));
  return 0;
}

// Detects a K-bit message from E soft bits; returns 1 if the reference declares it valid.
int ref_short_block_detect(int K, const int8_t* llrs, int E, int qm, uint8_t* out)
{
  short_block_detector_impl         det;
  std::vector<log_likelihood_ratio> in(E);
  for (int i = 0; i < E; ++i) {
    in[i] = llrs[i];
  }
  return det.detect(span<uint8_t>(out, K), in, mod_from_qm(qm)) ? 1 : 0;
}

// The reference's minimum number of rate-matched bits for a K-bit short block.
int ref_uci_min_encoded_bits(int K)
{
  return (int)calculate_uci_min_encoded_bits((unsigned)K);
}

} // extern "C"

/// get_ulsch_information (lib/ran/pusch/ulsch_info.cpp) for DM-RS type 1: out[0..8] = UL-SCH,
/// HARQ-ACK, reserved HARQ-ACK, CSI-1 and CSI-2 soft bits, HARQ-ACK, CSI-1 and CSI-2 REs, DC overlap
/// bits. rate_x1024 is the MCS's target code rate times 1024.
extern "C" int ref_ulsch_information(unsigned tbs_bits, float rate_x1024, int qm, int nof_layers, unsigned harq_ack,
                                     unsigned csi1, unsigned csi2, float alpha, float beta_ack, float beta_csi1,
                                     float beta_csi2, unsigned nof_rb, unsigned start, unsigned nof_symbols,
                                     unsigned dmrs_mask, unsigned nof_cdm, int contains_dc, uint32_t* out)
{
  ulsch_configuration c;
  c.tbs                          = units::bits(tbs_bits);
  c.mcs_descr.modulation         = static_cast<modulation_scheme>(qm);
  c.mcs_descr.target_code_rate   = rate_x1024;
  c.nof_harq_ack_bits            = units::bits(harq_ack);
  c.nof_csi_part1_bits           = units::bits(csi1);
  c.nof_csi_part2_bits           = units::bits(csi2);
  c.alpha_scaling                = alpha;
  c.beta_offset_harq_ack         = beta_ack;
  c.beta_offset_csi_part1        = beta_csi1;
  c.beta_offset_csi_part2        = beta_csi2;
  c.nof_rb                       = nof_rb;
  c.start_symbol_index           = start;
  c.nof_symbols                  = nof_symbols;
  c.dmrs_type                    = dmrs_config_type::type1;
  c.dmrs_symbol_mask             = bounded_bitset<MAX_NSYMB_PER_SLOT>(MAX_NSYMB_PER_SLOT);
  for (unsigned s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
    if ((dmrs_mask >> s) & 1U) {
      c.dmrs_symbol_mask.set(s);
    }
  }
  c.nof_cdm_groups_without_data = nof_cdm;
  c.nof_layers                  = static_cast<unsigned>(nof_layers);
  c.contains_dc                 = contains_dc != 0;
  const ulsch_information i     = get_ulsch_information(c);
  const uint32_t v[9] = {i.nof_ul_sch_bits.value(), i.nof_harq_ack_bits.value(), i.nof_harq_ack_rvd.value(),
                         i.nof_csi_part1_bits.value(), i.nof_csi_part2_bits.value(), i.nof_harq_ack_re,
                         i.nof_csi_part1_re, i.nof_csi_part2_re, i.nof_dc_overlap_bits.value()};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

// Test infrastructure only (checker, never shipped): a flat C ABI over the reference's own CPU
// implementation of UCI on PUSCH, so tests can call it through ctypes:
//   ulsch_demultiplex::demultiplex     include/ocudu/phy/upper/channel_processors/pusch/ulsch_demultiplex.h:31-90
//                                      (lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.cpp)
//   short_block_detector::detect       include/ocudu/phy/upper/channel_coding/short/short_block_detector.h
//   short_block_encoder::encode        include/ocudu/phy/upper/channel_coding/short/short_block_encoder.h
//   uci_decoder::decode (polar)        lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:25-111
//   polar_code::set                    lib/phy/upper/channel_coding/polar/polar_code_impl.cpp:432-480
//   a polar UCI test-vector encoder    polar_allocator, polar_encoder, polar_rate_matcher
// The scrambling sequence handed to the demultiplexer is the reference's own pseudo-random
// generator output for c_init, as pusch_demodulator_impl produces it.

#include "lib/phy/upper/channel_coding/polar/polar_allocator_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_code_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_deallocator_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_decoder_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_encoder_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_rate_dematcher_impl.h"
#include "lib/phy/upper/channel_coding/polar/polar_rate_matcher_impl.h"
#include "lib/phy/upper/channel_coding/short/short_block_detector_impl.h"
#include "lib/phy/upper/channel_processors/uci/uci_decoder_impl.h"
#include "ocudu/phy/upper/channel_coding/channel_coding_factories.h"
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

// polar_code_impl::set for (K, E) on the uplink (nMax 10, channel interleaver present): info[0..3] =
// n, N, nPC, valid (0 when the reference's range checks fail); kset[0..N) = 1 for K_set
// sub-channels; pc[0..4) = PC_set; subblock[0..N) = the sub-block interleaver.
int ref_polar_code(unsigned K, unsigned E, int* info, uint8_t* kset, uint16_t* pc, uint16_t* subblock)
{
  if (E > polar_code::EMAX || K < 18 || (K > 25 && K < 31) || K > 1023 || !(K + (K <= 25 ? 3 : 0) < E)) {
    info[3] = 0;
    return 0;
  }
  polar_code_impl code;
  code.set(K, E, 10, polar_code_ibil::present);
  info[0] = (int)code.get_n();
  info[1] = (int)code.get_N();
  info[2] = (int)code.get_nPC();
  info[3] = 1;
  for (unsigned i = 0; i != code.get_N(); ++i) {
    kset[i] = code.get_K_set().test(i) ? 1 : 0;
  }
  span<const uint16_t> pcs = code.get_PC_set();
  for (unsigned i = 0; i != 4; ++i) {
    pc[i] = i < pcs.size() ? pcs[i] : polar_code::NMAX;
  }
  span<const uint16_t> blk = code.get_blk_interleaver();
  for (unsigned i = 0; i != code.get_N(); ++i) {
    subblock[i] = blk[i];
  }
  return 1;
}

// Test-vector encoder for polar-coded UCI (TS 38.212 6.3.1.2-6.3.1.4 with the reference's pieces):
// A message bits into E bits. Segmentation and CRC size of uci_info.h, a leading zero filler bit
// when A is odd and split in two, the CRC of each codeblock by the reference's CRC calculator,
// polar_allocator + polar_encoder + polar_rate_matcher with the channel interleaver.
int ref_uci_polar_encode(unsigned A, const uint8_t* msg, unsigned E, uint8_t* out)
{
  const unsigned C  = get_nof_uci_codeblocks(A, E);
  const unsigned L  = get_uci_crc_size(A);
  auto           cf = create_crc_calculator_factory_sw("auto");
  auto           crc = cf->create(L == 11 ? crc_generator_poly::CRC11 : crc_generator_poly::CRC6);
  const unsigned A0 = A / C, E0 = E / C, F = A % C;
  unsigned       msg_pos = 0;
  for (unsigned c = 0; c != C; ++c) {
    const unsigned       Ac = c == 0 ? A0 : (A + C - 1) / C;
    const unsigned       Ec = c == 0 ? E0 : E - E0;
    const unsigned       Fc = c == 0 ? F : 0;
    const unsigned       K  = Fc + Ac + L;
    std::vector<uint8_t> blk(K, 0);
    std::memcpy(blk.data() + Fc, msg + msg_pos, Ac);
    msg_pos += Ac;
    const unsigned ck = crc->calculate_bit(span<const uint8_t>(blk.data(), Fc + Ac));
    for (unsigned i = 0; i != L; ++i) {
      blk[Fc + Ac + i] = (ck >> (L - 1 - i)) & 1U;
    }
    polar_code_impl code;
    code.set(K, Ec, 10, polar_code_ibil::present);
    std::vector<uint8_t> u(code.get_N()), x(code.get_N());
    polar_allocator_impl().allocate(u, blk, code);
    polar_encoder_impl().encode(x, u, code.get_n());
    polar_rate_matcher_impl().rate_match(span<uint8_t>(out + (c == 0 ? 0 : E0), Ec), x, code);
  }
  return (int)C;
}

// uci_decoder_impl::decode of an A-bit message (12..1706 bits) from E soft bits into out (A
// bytes); returns 1 when the reference declares it valid.
int ref_uci_polar_decode(unsigned A, const int8_t* llrs, unsigned E, uint8_t* out)
{
  auto             cf = create_crc_calculator_factory_sw("auto");
  uci_decoder_impl dec(std::make_unique<short_block_detector_impl>(), std::make_unique<polar_code_impl>(),
                       std::make_unique<polar_rate_dematcher_impl>(),
                       std::make_unique<polar_decoder_impl>(std::make_unique<polar_encoder_impl>(), 10),
                       std::make_unique<polar_deallocator_impl>(), cf->create(crc_generator_poly::CRC6),
                       cf->create(crc_generator_poly::CRC11));
  std::vector<log_likelihood_ratio> in(E);
  for (unsigned i = 0; i != E; ++i) {
    in[i] = llrs[i];
  }
  uci_decoder::configuration cfg = {};
  cfg.modulation                 = modulation_scheme::QPSK;
  return dec.decode(span<uint8_t>(out, A), in, cfg) == uci_status::valid ? 1 : 0;
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

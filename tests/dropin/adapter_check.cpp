// Drop-in check of the reference-interface adapters: each of the reference's PHY interfaces is
// served twice, by the reference's own implementation (its *_sw factories, AVX-512/AVX2 code) and
// by the pusch_b200 adapter over the GPU library, and both are fed the same seeded inputs through
// the interface's own virtual methods. One line per interface; the exit status is non-zero when
// any result differs beyond the interface's tolerance:
//   ldpc_decoder         bit-exact output bits and equal optional iteration counts
//   ldpc_rate_dematcher  bit-exact (finite LLRs), new transmission and soft combining
//   crc_calculator       equal checksums from calculate / calculate_byte / calculate_bit
//   demodulation_mapper  |difference| <= 1 LSB, at least 99.9 % equal
//   channel_equalizer    relative error <= 2.5e-4 (the reference's 14-bit reciprocal estimate)
// Test infrastructure: it links the reference's compiled code (oracle/_ref).
#include "../../ocudu-dapp-platform_b200/adapters/b200_phy_adapters.h"

#include "ocudu/adt/bit_buffer.h"
#include "ocudu/ocuduvec/bit.h"
#include "ocudu/phy/support/re_buffer.h"
#include "ocudu/phy/upper/channel_coding/channel_coding_factories.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_encoder.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_encoder_buffer.h"
#include "ocudu/phy/upper/channel_modulation/channel_modulation_factories.h"
#include "ocudu/phy/upper/equalization/dynamic_ch_est_list.h"
#include "ocudu/phy/upper/equalization/equalization_factories.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

using namespace ocudu;

namespace {

std::mt19937 rng(20260923);

int uniform(int lo, int hi)
{
  return std::uniform_int_distribution<int>(lo, hi)(rng);
}

float gauss()
{
  return std::normal_distribution<float>(0.f, 1.f)(rng);
}

const unsigned kLiftingSizes[] = {2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 18, 20, 22, 24, 26, 28, 30,
                                  32, 36, 40, 44, 48, 52, 56, 60, 64, 72, 80, 88, 96, 104, 112, 120, 128, 144, 160, 176,
                                  192, 208, 224, 240, 256, 288, 320, 352, 384};

int failures = 0;

void report(const char* name, bool ok, const char* detail)
{
  std::printf("%-20s %s  %s\n", name, ok ? "OK  " : "FAIL", detail);
  if (!ok) {
    ++failures;
  }
}

// ---------------------------------------------------------------------------------------------
void check_ldpc(const b200::device_config& dev)
{
  ldpc_decoder_factory::ldpc_decoder_factory_configuration fcfg = {false, false};
  auto ref_dec  = create_ldpc_decoder_factory_sw("auto", fcfg)->create();
  auto b200_dec = b200::create_ldpc_decoder_factory_b200(dev, fcfg)->create();
  auto encoder  = create_ldpc_encoder_factory_sw("generic")->create();
  auto crc_fac  = create_crc_calculator_factory_sw("auto");
  std::unique_ptr<crc_calculator> crcs[3] = {crc_fac->create(crc_generator_poly::CRC16),
                                             crc_fac->create(crc_generator_poly::CRC24A),
                                             crc_fac->create(crc_generator_poly::CRC24B)};
  int cases = 0, decoded = 0, mismatches = 0;
  for (int t = 0; t < 240; ++t) {
    const int      bg    = uniform(1, 2);
    const unsigned z     = kLiftingSizes[uniform(6, 50)];
    const unsigned K     = (bg == 1 ? 22 : 10) * z;
    const unsigned N     = (bg == 1 ? 66 : 50) * z;
    const int      which = uniform(0, 3); // 0..2: CRC16/24A/24B, 3: no CRC (syndrome)
    const unsigned L     = which == 0 ? 16 : 24;
    if (K < 2 * z + L + 8) {
      continue;
    }
    const unsigned F = static_cast<unsigned>(uniform(0, static_cast<int>(std::min(K / 4, K - 2 * z - L - 1))));

    // Message: random bits, CRC over them, then F zero filler bits.
    std::vector<uint8_t> msg(K, 0);
    for (unsigned i = 0; i < K - F - L; ++i) {
      msg[i] = static_cast<uint8_t>(uniform(0, 1));
    }
    const unsigned crc_idx = which == 3 ? 2 : static_cast<unsigned>(which);
    {
      dynamic_bit_buffer payload(K - F - L);
      ocuduvec::bit_pack(payload, span<const uint8_t>(msg.data(), K - F - L));
      const unsigned c = crcs[crc_idx]->calculate(payload);
      for (unsigned i = 0; i < L; ++i) {
        msg[K - F - L + i] = static_cast<uint8_t>((c >> (L - 1 - i)) & 1U);
      }
    }
    dynamic_bit_buffer packed(K);
    ocuduvec::bit_pack(packed, span<const uint8_t>(msg));
    ldpc_encoder::configuration ecfg;
    ecfg.base_graph   = bg == 1 ? ldpc_base_graph_type::BG1 : ldpc_base_graph_type::BG2;
    ecfg.lifting_size = static_cast<ldpc::lifting_size_t>(z);
    ecfg.Nref         = 0;
    const ldpc_encoder_buffer& eb = encoder->encode(packed, ecfg);
    std::vector<uint8_t>       cw(eb.get_codeblock_length());
    eb.write_codeblock(span<uint8_t>(cw), 0);

    // BPSK over AWGN at an SNR drawn per codeblock; E significant LLRs, zeros after them.
    const unsigned E     = static_cast<unsigned>(uniform(static_cast<int>(t % 7 == 0 ? K / 2 : K + 2 * z),
                                                     static_cast<int>(std::min<size_t>(N, cw.size()))));
    const float    snr   = std::pow(10.f, std::uniform_real_distribution<float>(-1.f, 5.f)(rng) / 10.f);
    const float    sigma = std::sqrt(1.f / (2.f * snr * static_cast<float>(K) / static_cast<float>(E)));
    std::vector<log_likelihood_ratio> llrs(N, 0);
    for (unsigned i = 0; i < E && i < cw.size(); ++i) {
      const float y = (1.f - 2.f * cw[i]) + sigma * gauss();
      llrs[i]       = static_cast<int8_t>(std::max(-120.f, std::min(120.f, std::rint(y * 2.f / (sigma * sigma) * 3.f))));
    }
    for (unsigned i = K - F - 2 * z; i < K - 2 * z && i < E; ++i) {
      llrs[i] = LLR_INFINITY;
    }

    ldpc_decoder::configuration dcfg;
    dcfg.base_graph      = ecfg.base_graph;
    dcfg.lifting_size    = ecfg.lifting_size;
    dcfg.nof_filler_bits = F;
    dcfg.nof_crc_bits    = L;
    dcfg.max_iterations  = static_cast<unsigned>(uniform(1, 10));
    crc_calculator* crc  = which == 3 ? nullptr : crcs[which].get();

    std::vector<uint8_t> out_ref((K + 7) / 8, 0x5a), out_b200((K + 7) / 8, 0x5a);
    bit_buffer           bref  = bit_buffer::from_bytes(span<uint8_t>(out_ref)).first(K);
    bit_buffer           bb200 = bit_buffer::from_bytes(span<uint8_t>(out_b200)).first(K);
    const auto           r_ref = ref_dec->decode(bref, llrs, crc, dcfg);
    const auto           r_b   = b200_dec->decode(bb200, llrs, crc, dcfg);
    bool                 same  = r_ref.has_value() == r_b.has_value() && (!r_ref.has_value() || *r_ref == *r_b);
    for (unsigned i = 0; i < K && same; ++i) {
      same = bref.extract(i, 1) == bb200.extract(i, 1);
    }
    ++cases;
    decoded += r_ref.has_value() ? 1 : 0;
    mismatches += same ? 0 : 1;
  }
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%d codeblocks (%d decoded), %d mismatches", cases, decoded, mismatches);
  report("ldpc_decoder", mismatches == 0 && decoded > 0 && decoded < cases, buf);
}

// ---------------------------------------------------------------------------------------------
void check_rate_dematcher(const b200::device_config& dev)
{
  auto ref  = create_ldpc_rate_dematcher_factory_sw("auto")->create();
  auto b200 = b200::create_ldpc_rate_dematcher_factory_b200(dev)->create();
  int  cases = 0, mismatches = 0;
  for (int t = 0; t < 120; ++t) {
    const int      bg = uniform(1, 2);
    const unsigned z  = kLiftingSizes[uniform(10, 50)];
    const unsigned K  = (bg == 1 ? 22 : 10) * z;
    const unsigned N  = (bg == 1 ? 66 : 50) * z;
    const unsigned qm = std::array<unsigned, 5>{1, 2, 4, 6, 8}[uniform(0, 4)];
    codeblock_metadata md          = {};
    md.tb_common.base_graph        = bg == 1 ? ldpc_base_graph_type::BG1 : ldpc_base_graph_type::BG2;
    md.tb_common.lifting_size      = static_cast<ldpc::lifting_size_t>(z);
    md.tb_common.rv                = static_cast<unsigned>(uniform(0, 3));
    md.tb_common.mod               = qm == 1 ? modulation_scheme::BPSK
                                     : qm == 2 ? modulation_scheme::QPSK
                                     : qm == 4 ? modulation_scheme::QAM16
                                     : qm == 6 ? modulation_scheme::QAM64
                                               : modulation_scheme::QAM256;
    md.tb_common.Nref              = uniform(0, 3) == 0 ? (N * 2 / 3) : 0;
    md.cb_specific.full_length     = N;
    md.cb_specific.nof_filler_bits = static_cast<unsigned>(uniform(0, static_cast<int>(K / 8)));
    const unsigned E               = qm * static_cast<unsigned>(uniform(static_cast<int>(K / qm / 2), static_cast<int>(2 * N / qm)));
    md.cb_specific.rm_length       = E;
    std::vector<log_likelihood_ratio> in(E), out_ref(N), out_b(N);
    for (int pass = 0; pass < 2; ++pass) {
      for (auto& v : in) {
        v = static_cast<int8_t>(uniform(-120, 120));
      }
      ref->rate_dematch(out_ref, in, pass == 0, md);
      b200->rate_dematch(out_b, in, pass == 0, md);
      ++cases;
      mismatches += std::memcmp(out_ref.data(), out_b.data(), N) == 0 ? 0 : 1;
    }
  }
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%d calls (new data + combining), %d mismatches", cases, mismatches);
  report("ldpc_rate_dematcher", mismatches == 0, buf);
}

// ---------------------------------------------------------------------------------------------
void check_crc(const b200::device_config& dev)
{
  auto ref_fac  = create_crc_calculator_factory_sw("auto");
  auto b200_fac = b200::create_crc_calculator_factory_b200(dev);
  int  cases = 0, mismatches = 0;
  for (crc_generator_poly poly : {crc_generator_poly::CRC16, crc_generator_poly::CRC24A, crc_generator_poly::CRC24B}) {
    auto ref  = ref_fac->create(poly);
    auto b200 = b200_fac->create(poly);
    for (int t = 0; t < 40; ++t) {
      const unsigned       nbits = static_cast<unsigned>(uniform(1, 8448));
      std::vector<uint8_t> bits(nbits);
      for (auto& b : bits) {
        b = static_cast<uint8_t>(uniform(0, 1));
      }
      dynamic_bit_buffer packed(nbits);
      ocuduvec::bit_pack(packed, span<const uint8_t>(bits));
      std::vector<uint8_t> bytes(nbits / 8 + 1);
      for (auto& b : bytes) {
        b = static_cast<uint8_t>(uniform(0, 255));
      }
      const bool same = ref->calculate(packed) == b200->calculate(packed) &&
                        ref->calculate_bit(bits) == b200->calculate_bit(bits) &&
                        ref->calculate_byte(bytes) == b200->calculate_byte(bytes);
      ++cases;
      mismatches += same ? 0 : 1;
    }
  }
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%d strings x 3 methods, %d mismatches", cases, mismatches);
  report("crc_calculator", mismatches == 0, buf);
}

// ---------------------------------------------------------------------------------------------
void check_demapper(const b200::device_config& dev)
{
  auto ref  = create_demodulation_mapper_factory()->create();
  auto b200 = b200::create_demodulation_mapper_factory_b200(dev)->create();
  long total = 0, equal = 0;
  int  worst = 0;
  for (modulation_scheme mod :
       {modulation_scheme::QPSK, modulation_scheme::QAM16, modulation_scheme::QAM64, modulation_scheme::QAM256}) {
    const unsigned     qm = get_bits_per_symbol(mod);
    const unsigned     n  = 4096 + static_cast<unsigned>(uniform(0, 31));
    std::vector<cf_t>  sym(n);
    std::vector<float> nv(n);
    for (unsigned i = 0; i < n; ++i) {
      sym[i] = cf_t(1.3f * gauss(), 1.3f * gauss());
      nv[i]  = std::pow(10.f, std::uniform_real_distribution<float>(-3.f, 0.5f)(rng));
    }
    nv[0] = 0.f;
    nv[1] = -1.f;
    std::vector<log_likelihood_ratio> a(n * qm), b(n * qm);
    ref->demodulate_soft(a, sym, nv, mod);
    b200->demodulate_soft(b, sym, nv, mod);
    for (unsigned i = 0; i < n * qm; ++i) {
      const int d = std::abs(static_cast<int>(a[i].to_value_type()) - static_cast<int>(b[i].to_value_type()));
      worst       = std::max(worst, d);
      equal += d == 0 ? 1 : 0;
      ++total;
    }
  }
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%ld LLRs, %.5f equal, max |diff| %d", total, double(equal) / double(total), worst);
  report("demodulation_mapper", worst <= 1 && equal >= total - total / 1000, buf);
}

// ---------------------------------------------------------------------------------------------
void check_equalizer(const b200::device_config& dev)
{
  struct shape {
    unsigned                         ports, layers;
    channel_equalizer_algorithm_type type;
  };
  const shape shapes[] = {{1, 1, channel_equalizer_algorithm_type::zf},
                          {2, 1, channel_equalizer_algorithm_type::zf},
                          {4, 1, channel_equalizer_algorithm_type::mmse},
                          {2, 2, channel_equalizer_algorithm_type::mmse},
                          {4, 2, channel_equalizer_algorithm_type::mmse},
                          {4, 4, channel_equalizer_algorithm_type::mmse}};
  double worst = 0.0;
  int    calls = 0;
  for (const shape& s : shapes) {
    auto           ref    = create_channel_equalizer_generic_factory(s.type)->create();
    auto           b200   = b200::create_channel_equalizer_factory_b200(dev, s.type)->create();
    const unsigned nof_re = 3276;
    dynamic_re_buffer<cbf16_t> y(s.ports, nof_re);
    dynamic_ch_est_list        h(nof_re, s.ports, s.layers);
    std::vector<float>         nv(s.ports);
    for (unsigned p = 0; p < s.ports; ++p) {
      nv[p] = 0.01f * (1.f + static_cast<float>(p));
      for (unsigned i = 0; i < nof_re; ++i) {
        y.get_slice(p)[i] = cbf16_t(gauss(), gauss());
      }
      for (unsigned l = 0; l < s.layers; ++l) {
        for (unsigned i = 0; i < nof_re; ++i) {
          h.get_channel(p, l)[i] = cbf16_t(0.7f * gauss(), 0.7f * gauss());
        }
      }
    }
    std::vector<cf_t>  eq_a(nof_re * s.layers), eq_b(nof_re * s.layers);
    std::vector<float> v_a(nof_re * s.layers), v_b(nof_re * s.layers);
    ref->equalize(eq_a, v_a, y, h, nv, 1.0f);
    b200->equalize(eq_b, v_b, y, h, nv, 1.0f);
    float max_eq = 0.f, max_v = 0.f;
    for (unsigned i = 0; i < eq_a.size(); ++i) {
      max_eq = std::max(max_eq, std::abs(eq_a[i]));
      if (std::isfinite(v_a[i])) {
        max_v = std::max(max_v, v_a[i]);
      }
    }
    for (unsigned i = 0; i < eq_a.size(); ++i) {
      worst = std::max(worst, double(std::abs(eq_a[i] - eq_b[i]) / std::max(std::abs(eq_a[i]), 1e-3f * max_eq)));
      if (std::isfinite(v_a[i]) || std::isfinite(v_b[i])) {
        worst = std::max(worst, double(std::abs(v_a[i] - v_b[i]) / std::max(std::abs(v_a[i]), 1e-3f * max_v)));
      }
    }
    ++calls;
  }
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%d shapes x 3276 RE, worst relative error %.2e", calls, worst);
  report("channel_equalizer", worst <= 2.5e-4, buf);
}

} // namespace

int main()
{
  b200::device_config dev;
  dev.device         = 0;
  dev.max_codeblocks = 4;
  check_ldpc(dev);
  check_rate_dematcher(dev);
  check_crc(dev);
  check_demapper(dev);
  check_equalizer(dev);
  std::printf("%s\n", failures == 0 ? "ALL OK" : "FAILED");
  return failures == 0 ? 0 : 1;
}

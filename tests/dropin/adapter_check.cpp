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
//   port_channel_estimator  noise, EPRE, SNR, RSRP within 1e-4; per-symbol bf16 estimates equal or
//                        one unit apart (over 99 % equal); CFO within 1e-3 Hz (or 1e-3 relative);
//                        time alignment within one T_c
//   pusch_decoder        (with a codeword file, argv[1]) bit-exact TBs, CRC flags, codeblock counts,
//                        iteration statistics and rx-buffer soft bits over two transmissions (HARQ)
//   resident_decoder     (same file) pusch_resident_codeblock_decoder::decode_batch bit-exact with the
//                        reference's codeblock decoder: CRC verdicts, iterations, bits, soft buffers
// Test infrastructure: it links the reference's compiled code (oracle/_ref).
#include "../../ocudu-dapp-platform_b200/adapters/b200_phy_adapters.h"

#include "lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.h"
#include "lib/phy/upper/signal_processors/dmrs_helper.h"
#include "ocudu/phy/generic_functions/generic_functions_factories.h"
#include "ocudu/phy/support/resource_grid_reader.h"
#include "ocudu/phy/support/time_alignment_estimator/time_alignment_estimator_factories.h"
#include "ocudu/phy/upper/channel_coding/ldpc/ldpc_segmenter_rx.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_notifier.h"
#include "ocudu/phy/upper/channel_processors/pusch/pusch_decoder_result.h"
#include "ocudu/phy/upper/rx_buffer_pool.h"
#include "ocudu/phy/upper/sequence_generators/sequence_generator_factories.h"
#include "ocudu/phy/upper/signal_processors/channel_estimator/factories.h"

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

// ---------------------------------------------------------------------------------------------
// A resource_grid_reader over a cbf16 array [port][symbol][subcarrier].
class vector_grid_reader : public resource_grid_reader
{
public:
  vector_grid_reader(const std::vector<cbf16_t>& data, unsigned nports, unsigned nsubc) :
    data_(data), nports_(nports), nsubc_(nsubc)
  {
  }
  unsigned     get_nof_ports() const override { return nports_; }
  unsigned     get_nof_subc() const override { return nsubc_; }
  unsigned     get_nof_symbols() const override { return MAX_NSYMB_PER_SLOT; }
  bool         is_empty(unsigned) const override { return false; }
  bool         is_empty() const override { return false; }
  crb_interval get_allocation_range(unsigned, unsigned) const override { return {0, nsubc_ / 12}; }
  span<cf_t>   get(span<cf_t> symbols, unsigned port, unsigned l, unsigned k_init,
                   const bounded_bitset<MAX_NOF_SUBCARRIERS>& mask) const override
  {
    mask.for_each(0, mask.size(), [&](unsigned k) {
      symbols.front() = to_cf(view(port, l)[k_init + k]);
      symbols         = symbols.last(symbols.size() - 1);
    });
    return symbols;
  }
  span<cbf16_t> get(span<cbf16_t> symbols, unsigned port, unsigned l, unsigned k_init,
                    const bounded_bitset<MAX_NOF_SUBCARRIERS>& mask) const override
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
    return span<const cbf16_t>(data_.data() + (static_cast<size_t>(port) * MAX_NSYMB_PER_SLOT + l) * nsubc_, nsubc_);
  }
  const std::vector<cbf16_t>& data_;
  unsigned                    nports_, nsubc_;
};

// port_channel_estimator: seeded slots (random PRB allocation, one or two layers, one or two DM-RS
// symbols, a multipath channel with a delay and a frequency offset, noise), both estimators on every
// receive port with the same pilots.
void check_port_estimator(const b200::device_config& dev)
{
  auto ta_factory = create_time_alignment_estimator_dft_factory(create_dft_processor_factory_generic());
  auto ref_est    = create_port_channel_estimator_factory_sw(ta_factory)
                     ->create(port_channel_estimator_fd_smoothing_strategy::filter,
                              port_channel_estimator_td_interpolation_strategy::interpolate, false);
  auto b200_est = b200::create_port_channel_estimator_factory_b200(dev)->create(
      port_channel_estimator_fd_smoothing_strategy::filter, port_channel_estimator_td_interpolation_strategy::interpolate,
      false);
  auto   prg     = create_pseudo_random_generator_sw_factory()->create();
  int    ports   = 0, bad = 0;
  double worst_s = 0, worst_ta = 0, worst_cfo = 0;
  for (int t = 0; t < 24; ++t) {
    const unsigned nof_prb_grid = 273, nsubc = 12 * nof_prb_grid, nports = 4;
    const unsigned nof_rb   = static_cast<unsigned>(uniform(1, 273));
    const unsigned rb_start = static_cast<unsigned>(uniform(0, static_cast<int>(nof_prb_grid - nof_rb)));
    const unsigned nl       = static_cast<unsigned>(uniform(1, 2));
    const bool     two      = uniform(0, 3) != 0;
    const unsigned n_id = static_cast<unsigned>(uniform(0, 1007)), slot = static_cast<unsigned>(uniform(0, 19));
    bounded_bitset<MAX_NSYMB_PER_SLOT> symbols(MAX_NSYMB_PER_SLOT);
    symbols.set(2);
    if (two) {
      symbols.set(11);
    }
    crb_bitmap rb_mask(rb_start + nof_rb);
    rb_mask.fill(rb_start, rb_start + nof_rb);
    const unsigned   nd = two ? 2 : 1, npil = 6 * nof_rb;
    dmrs_symbol_list pilots({npil, nd, nl});
    for (unsigned d = 0, s = 0; s < MAX_NSYMB_PER_SLOT; ++s) {
      if (!symbols.test(s)) {
        continue;
      }
      prg->init(((14 * slot + s + 1) * (2 * n_id + 1) * (1U << 17) + 2 * n_id) % (1U << 31));
      dmrs_sequence_generate(pilots.get_symbol(d, 0), *prg, M_SQRT1_2, 0, 6, rb_mask);
      if (nl > 1) {
        dmrs_pxsch_parameters p1 = get_pxsch_dmrs_params(dmrs_config_type::type1, 1);
        span<cf_t>            dst = pilots.get_symbol(d, 1);
        span<const cf_t>      src = pilots.get_symbol(d, 0);
        std::copy(src.begin(), src.end(), dst.begin());
        for (unsigned k = 1; k < dst.size(); k += 2) {
          dst[k] *= p1.w_f[1];
        }
      }
      ++d;
    }
    port_channel_estimator::configuration cfg;
    cfg.scs          = subcarrier_spacing::kHz30;
    cfg.cp           = cyclic_prefix::NORMAL;
    cfg.first_symbol = 0;
    cfg.nof_symbols  = MAX_NSYMB_PER_SLOT;
    cfg.scaling      = 1.41254f;
    for (unsigned p = 0; p != nports; ++p) {
      cfg.rx_ports.push_back(static_cast<uint8_t>(p));
    }
    for (unsigned l = 0; l != nl; ++l) {
      cfg.dmrs_pattern.push_back(
          {symbols, rb_mask, {}, std::nullopt, get_pxsch_dmrs_params(dmrs_config_type::type1, l).re_pattern});
    }
    // Grid: per port and layer a two-tap channel with a delay, a slow CFO rotation, pilots on the
    // DM-RS comb, noise everywhere.
    std::vector<cbf16_t> grid(static_cast<size_t>(nports) * MAX_NSYMB_PER_SLOT * nsubc);
    const float          snr = std::pow(10.f, static_cast<float>(uniform(0, 30)) / 10.f);
    const float          sig = std::sqrt(0.5f / snr);
    const float          cfo = static_cast<float>(uniform(-300, 300)); // Hz
    for (unsigned p = 0; p != nports; ++p) {
      cf_t  a[2][2];
      float tau[2];
      for (unsigned l = 0; l != 2; ++l) {
        a[l][0] = {gauss() * 0.6f, gauss() * 0.6f};
        a[l][1] = {gauss() * 0.4f, gauss() * 0.4f};
        tau[l]  = static_cast<float>(uniform(0, 400)) * 1e-9f;
      }
      for (unsigned s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
        const cf_t rot = std::polar(1.f, 6.2831853f * cfo * static_cast<float>(s) * 35.7e-6f);
        for (unsigned k = 0; k != nsubc; ++k) {
          cf_t y = {sig * gauss(), sig * gauss()};
          if (k >= 12 * rb_start && k < 12 * (rb_start + nof_rb)) {
            const unsigned j = k - 12 * rb_start;
            if (symbols.test(s) && (j % 2) == 0) {
              const unsigned d = (s == 2) ? 0 : 1;
              for (unsigned l = 0; l != nl; ++l) {
                const float f = 30e3f * static_cast<float>(j);
                const cf_t  h = a[l][0] + a[l][1] * std::polar(1.f, -6.2831853f * f * tau[l]);
                y += h * pilots.get_symbol(d, l)[j / 2] * cfg.scaling * rot;
              }
            } else if (!symbols.test(s)) {
              y += cf_t{(uniform(0, 1) ? 0.7071f : -0.7071f), (uniform(0, 1) ? 0.7071f : -0.7071f)};
            }
          }
          grid[(static_cast<size_t>(p) * MAX_NSYMB_PER_SLOT + s) * nsubc + k] = to_cbf16(y);
        }
      }
    }
    vector_grid_reader reader(grid, nports, nsubc);
    std::vector<cbf16_t> a_sym(12 * nof_rb), b_sym(12 * nof_rb);
    for (unsigned p = 0; p != nports; ++p, ++ports) {
      const port_channel_estimator_results& r = ref_est->compute(reader, p, pilots, cfg);
      const port_channel_estimator_results& g = b200_est->compute(reader, p, pilots, cfg);
      auto rel = [](float x, float y) { return std::abs(x - y) / std::max(std::abs(y), 1e-30f); };
      double e = std::max({rel(g.get_noise_variance(), r.get_noise_variance()), rel(g.get_epre(), r.get_epre()),
                           rel(g.get_snr(), r.get_snr()), rel(g.get_rsrp(0), r.get_rsrp(0))});
      if (nl > 1) {
        e = std::max<double>(e, rel(g.get_rsrp(1), r.get_rsrp(1)));
      }
      worst_s = std::max(worst_s, e);
      const double ta = std::abs(static_cast<double>(g.get_time_alignment().to_Tc() - r.get_time_alignment().to_Tc()));
      worst_ta        = std::max(worst_ta, ta);
      bool ok         = e <= 1e-4 && ta <= 1;
      if (r.get_cfo_Hz().has_value() != g.get_cfo_Hz().has_value()) {
        ok = false;
      } else if (r.get_cfo_Hz().has_value()) {
        const double d = std::abs(*g.get_cfo_Hz() - *r.get_cfo_Hz());
        worst_cfo      = std::max(worst_cfo, d);
        ok             = ok && d <= std::max(1e-3, 1e-3 * std::abs(*r.get_cfo_Hz()));
      }
      // Per-symbol bf16 estimates: 99 % of the components bit-equal, every component within one bf16
      // unit of its own magnitude plus 1e-4 of the coefficient's magnitude (a component much smaller
      // than its coefficient carries the FP32 difference of the whole coefficient in many of its own
      // units).
      unsigned diff1 = 0, equal = 0, total = 0;
      for (unsigned s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
        for (unsigned l = 0; l != nl; ++l) {
          r.get_symbol_ch_estimate(a_sym, s, l);
          g.get_symbol_ch_estimate(b_sym, s, l);
          for (unsigned k = 0; k != a_sym.size(); ++k) {
            uint32_t x, y;
            std::memcpy(&x, &a_sym[k], 4);
            std::memcpy(&y, &b_sym[k], 4);
            auto  val = [](uint32_t w, int part) {
              const uint32_t b = part == 0 ? (w << 16) : (w & 0xffff0000u);
              float          f;
              std::memcpy(&f, &b, 4);
              return static_cast<double>(f);
            };
            const double mag = std::hypot(val(x, 0), val(x, 16));
            for (int part = 0; part < 32; part += 16) {
              const double a   = val(x, part), b = val(y, part);
              const double top = std::max(std::abs(a), std::abs(b));
              const double ulp = top > 0 ? std::ldexp(1.0, std::ilogb(top) - 7) : 0.0;
              diff1 += std::abs(a - b) > ulp + 1e-4 * mag;
              equal += a == b;
              ++total;
            }
          }
        }
      }
      ok = ok && diff1 == 0 && equal > 0.99 * total;
      bad += ok ? 0 : 1;
    }
  }
  char detail[200];
  std::snprintf(detail, sizeof(detail), "%d ports, worst scalar rel %.2e, TA %.0f Tc, CFO %.2e Hz, %d off", ports,
                worst_s, worst_ta, worst_cfo, bad);
  report("port_channel_estimator", bad == 0, detail);
}

// pusch_decoder: codewords from a file (written by tests/test_dropin.py with the project's
// transmit-side codec): per transport block its parameters and two transmissions of soft bits.
// Both decoders get rx buffers of their own pool with the same identifiers.
struct sch_notifier : public pusch_decoder_notifier {
  pusch_decoder_result result;
  bool                 called = false;
  void                 on_sch_data(const pusch_decoder_result& r) override
  {
    result = r;
    called = true;
  }
};

void check_pusch_decoder(const b200::device_config& dev, const char* path)
{
  FILE* f = std::fopen(path, "rb");
  if (f == nullptr) {
    report("pusch_decoder", false, "cannot open the codeword file");
    return;
  }
  auto crcf = create_crc_calculator_factory_sw("auto");
  pusch_codeblock_decoder::sch_crc cb_crcs{crcf->create(crc_generator_poly::CRC16),
                                           crcf->create(crc_generator_poly::CRC24A),
                                           crcf->create(crc_generator_poly::CRC24B)};
  ldpc_decoder_factory::ldpc_decoder_factory_configuration fcfg = {false, false};
  std::vector<std::unique_ptr<pusch_codeblock_decoder>>   cbd;
  cbd.push_back(std::make_unique<pusch_codeblock_decoder>(create_ldpc_rate_dematcher_factory_sw("auto")->create(),
                                                          create_ldpc_decoder_factory_sw("auto", fcfg)->create(),
                                                          cb_crcs));
  auto pool = std::make_shared<pusch_decoder_impl::codeblock_decoder_pool>(span<std::unique_ptr<pusch_codeblock_decoder>>(cbd));
  pusch_decoder_impl ref_dec(create_ldpc_segmenter_rx_factory_sw()->create(), pool,
                             {crcf->create(crc_generator_poly::CRC16), crcf->create(crc_generator_poly::CRC24A),
                              crcf->create(crc_generator_poly::CRC24B)},
                             nullptr, 273, 2);
  auto b200_dec = b200::create_pusch_decoder_factory_b200(dev, 273, 2)->create();

  rx_buffer_pool_config pcfg = {};
  pcfg.max_codeblock_size    = 66 * 384;
  pcfg.nof_buffers           = 8;
  pcfg.nof_codeblocks        = 400;
  pcfg.expire_timeout_slots  = 100;
  pcfg.external_soft_bits    = false;
  auto ref_pool  = create_rx_buffer_pool(pcfg);
  auto b200_pool = create_rx_buffer_pool(pcfg);

  int32_t ntb = 0;
  bool    ok  = std::fread(&ntb, 4, 1, f) == 1;
  int     tbs_ok = 0, tx = 0, mismatches = 0;
  for (int i = 0; ok && i < ntb; ++i) {
    int32_t h[8]; // tbs bytes, bg, qm, layers, nref, G, C, transmissions
    ok = std::fread(h, 4, 8, f) == 8;
    if (!ok) {
      break;
    }
    std::vector<uint8_t> tb_a(h[0]), tb_b(h[0]);
    for (int x = 0; ok && x < h[7]; ++x, ++tx) {
      int32_t rv_nd[2];
      ok = std::fread(rv_nd, 4, 2, f) == 2;
      std::vector<log_likelihood_ratio> llrs(h[5]);
      ok = ok && std::fread(llrs.data(), 1, h[5], f) == static_cast<size_t>(h[5]);
      if (!ok) {
        break;
      }
      pusch_decoder::configuration dc;
      dc.base_graph          = h[1] == 1 ? ldpc_base_graph_type::BG1 : ldpc_base_graph_type::BG2;
      dc.rv                  = static_cast<unsigned>(rv_nd[0]);
      dc.mod                 = h[2] == 2 ? modulation_scheme::QPSK
                                         : (h[2] == 4 ? modulation_scheme::QAM16
                                                      : (h[2] == 6 ? modulation_scheme::QAM64 : modulation_scheme::QAM256));
      dc.Nref                = static_cast<unsigned>(h[4]);
      dc.nof_layers          = static_cast<unsigned>(h[3]);
      dc.nof_ldpc_iterations = 6;
      dc.use_early_stop      = true;
      dc.new_data            = rv_nd[1] != 0;
      const slot_point sl(1, static_cast<uint32_t>(2 * i + x));
      unique_rx_buffer ra = ref_pool->get_pool().reserve(sl, trx_buffer_identifier(to_rnti(0x4601 + i), 0), h[6], dc.new_data);
      unique_rx_buffer rb = b200_pool->get_pool().reserve(sl, trx_buffer_identifier(to_rnti(0x4601 + i), 0), h[6], dc.new_data);
      if (!ra.is_valid() || !rb.is_valid()) {
        ok = false;
        break;
      }
      rx_buffer&   buf_a = *ra;
      rx_buffer&   buf_b = *rb;
      sch_notifier na, nb;
      pusch_decoder_buffer& ia = ref_dec.new_data(tb_a, std::move(ra), na, dc);
      pusch_decoder_buffer& ib = b200_dec->new_data(tb_b, std::move(rb), nb, dc);
      ref_dec.set_nof_softbits(units::bits(h[5]));
      b200_dec->set_nof_softbits(units::bits(h[5]));
      for (unsigned off = 0; off < static_cast<unsigned>(h[5]); off += 4096) {
        const unsigned                   n   = std::min(4096U, static_cast<unsigned>(h[5]) - off);
        span<const log_likelihood_ratio> blk = span<const log_likelihood_ratio>(llrs).subspan(off, n);
        span<log_likelihood_ratio>       va  = ia.get_next_block_view(n);
        std::copy(blk.begin(), blk.end(), va.begin());
        ia.on_new_softbits(va);
        ib.on_new_softbits(blk);
      }
      ia.on_end_softbits();
      ib.on_end_softbits();
      bool same = na.called && nb.called && na.result.tb_crc_ok == nb.result.tb_crc_ok &&
                  na.result.nof_codeblocks_total == nb.result.nof_codeblocks_total &&
                  na.result.ldpc_decoder_stats.get_nof_observations() ==
                      nb.result.ldpc_decoder_stats.get_nof_observations() &&
                  na.result.ldpc_decoder_stats.get_min() == nb.result.ldpc_decoder_stats.get_min() &&
                  na.result.ldpc_decoder_stats.get_max() == nb.result.ldpc_decoder_stats.get_max() &&
                  na.result.ldpc_decoder_stats.get_mean() == nb.result.ldpc_decoder_stats.get_mean();
      if (same && na.result.tb_crc_ok) {
        same = tb_a == tb_b;
        ++tbs_ok;
      }
      // The buffers: CRC flags and soft bits (unlocked buffers keep them for the retransmission).
      if (same && !na.result.tb_crc_ok) {
        span<bool> ca = buf_a.get_codeblocks_crc(), cb = buf_b.get_codeblocks_crc();
        same = std::equal(ca.begin(), ca.end(), cb.begin());
        const unsigned z = 384, n_cb = (h[1] == 1 ? 66U : 50U);
        (void)z;
        for (unsigned c = 0; same && c < static_cast<unsigned>(h[6]); ++c) {
          const unsigned n = buf_a.get_codeblock_soft_bits(c, 0).size();
          (void)n_cb;
          span<log_likelihood_ratio> sa = buf_a.get_codeblock_soft_bits(c, n), sb = buf_b.get_codeblock_soft_bits(c, n);
          same = std::equal(sa.begin(), sa.end(), sb.begin());
        }
      }
      mismatches += same ? 0 : 1;
    }
  }
  std::fclose(f);
  char detail[200];
  std::snprintf(detail, sizeof(detail), "%d transport blocks, %d transmissions, %d decoded, %d mismatches%s", ntb, tx,
                tbs_ok, mismatches, ok ? "" : " (input error)");
  report("pusch_decoder", ok && mismatches == 0 && tx > 0, detail);
}

// pusch_resident_codeblock_decoder::decode_batch against the reference's pusch_codeblock_decoder on
// the codeblocks of the same codewords (segmented by the reference's ldpc_segmenter_rx): CRC
// verdicts, iteration counts, decoded bits and the soft buffers, over both transmissions.
void check_resident_decoder(const b200::device_config& dev, const char* path)
{
  FILE* f = std::fopen(path, "rb");
  if (f == nullptr) {
    report("resident_decoder", false, "cannot open the codeword file");
    return;
  }
  auto                             crcf = create_crc_calculator_factory_sw("auto");
  pusch_codeblock_decoder::sch_crc cb_crcs{crcf->create(crc_generator_poly::CRC16),
                                           crcf->create(crc_generator_poly::CRC24A),
                                           crcf->create(crc_generator_poly::CRC24B)};
  ldpc_decoder_factory::ldpc_decoder_factory_configuration fcfg = {false, false};
  pusch_codeblock_decoder ref_cb(create_ldpc_rate_dematcher_factory_sw("auto")->create(),
                                 create_ldpc_decoder_factory_sw("auto", fcfg)->create(), cb_crcs);
  b200::pusch_resident_codeblock_decoder_b200 res(dev);
  auto                                        seg = create_ldpc_segmenter_rx_factory_sw()->create();
  int32_t                                     ntb = 0;
  bool                                        ok  = std::fread(&ntb, 4, 1, f) == 1;
  int                                         cbs = 0, decoded = 0, mismatches = 0;
  for (int i = 0; ok && i < ntb; ++i) {
    int32_t h[8];
    ok = std::fread(h, 4, 8, f) == 8;
    if (!ok) {
      break;
    }
    const unsigned                                 N = 0;
    std::vector<std::vector<log_likelihood_ratio>> ref_bufs, b200_bufs;
    for (int x = 0; ok && x < h[7]; ++x) {
      int32_t rv_nd[2];
      ok = std::fread(rv_nd, 4, 2, f) == 2;
      std::vector<log_likelihood_ratio> llrs(h[5]);
      ok = ok && std::fread(llrs.data(), 1, h[5], f) == static_cast<size_t>(h[5]);
      if (!ok) {
        break;
      }
      segmenter_config sc;
      sc.transport_block_size = units::bytes(h[0]);
      sc.base_graph           = h[1] == 1 ? ldpc_base_graph_type::BG1 : ldpc_base_graph_type::BG2;
      sc.rv                   = static_cast<unsigned>(rv_nd[0]);
      sc.mod                  = h[2] == 2 ? modulation_scheme::QPSK
                                          : (h[2] == 4 ? modulation_scheme::QAM16
                                                       : (h[2] == 6 ? modulation_scheme::QAM64 : modulation_scheme::QAM256));
      sc.Nref                 = static_cast<unsigned>(h[4]);
      sc.nof_layers           = static_cast<unsigned>(h[3]);
      sc.nof_ch_symbols       = static_cast<unsigned>(h[5]) / static_cast<unsigned>(h[2]);
      static_vector<described_rx_codeblock, MAX_NOF_SEGMENTS> cbl;
      seg->segment(cbl, llrs, sc);
      const unsigned C       = static_cast<unsigned>(cbl.size());
      const bool     newdata = rv_nd[1] != 0;
      const unsigned n_full  = cbl[0].second.cb_specific.full_length;
      if (newdata) {
        ref_bufs.assign(C, std::vector<log_likelihood_ratio>(n_full));
        b200_bufs.assign(C, std::vector<log_likelihood_ratio>(n_full));
      }
      const crc_generator_poly poly =
          C > 1 ? crc_generator_poly::CRC24B : (8 * h[0] <= 3824 ? crc_generator_poly::CRC16 : crc_generator_poly::CRC24A);
      const unsigned                      k = n_full / (h[1] == 1 ? 3 : 5);
      std::vector<dynamic_bit_buffer>     ref_bits, b200_bits;
      std::vector<bit_buffer>             b200_views;
      std::vector<span<log_likelihood_ratio>> b200_rm;
      for (unsigned c = 0; c != C; ++c) {
        ref_bits.emplace_back(k);
        b200_bits.emplace_back(k);
      }
      for (unsigned c = 0; c != C; ++c) {
        b200_views.push_back(b200_bits[c]);
        b200_rm.push_back(b200_bufs[c]);
      }
      std::vector<pusch_resident_codeblock_decoder::codeblock_result> got =
          res.decode_batch(span<const described_rx_codeblock>(cbl.data(), C), b200_views, b200_rm, newdata, poly, true, 6);
      for (unsigned c = 0; c != C; ++c, ++cbs) {
        std::optional<unsigned> want = ref_cb.decode(ref_bits[c], ref_bufs[c], cbl[c].first, newdata, poly, true, 6,
                                                     cbl[c].second);
        bool same = got[c].crc_ok == want.has_value() && got[c].nof_iterations == (want.has_value() ? *want : 6U) &&
                    ref_bufs[c] == b200_bufs[c];
        if (same && want.has_value()) {
          same = std::equal(ref_bits[c].get_buffer().begin(), ref_bits[c].get_buffer().end(),
                            b200_bits[c].get_buffer().begin());
          ++decoded;
        }
        mismatches += same ? 0 : 1;
      }
      (void)N;
    }
  }
  std::fclose(f);
  char detail[200];
  std::snprintf(detail, sizeof(detail), "%d codeblocks, %d decoded, %d mismatches%s", cbs, decoded, mismatches,
                ok ? "" : " (input error)");
  report("resident_decoder", ok && mismatches == 0 && cbs > 0, detail);
}

int main(int argc, char** argv)
{
  b200::device_config dev;
  dev.device         = 0;
  dev.max_codeblocks = 4;
  check_ldpc(dev);
  check_rate_dematcher(dev);
  check_crc(dev);
  check_demapper(dev);
  check_equalizer(dev);
  check_port_estimator(dev);
  if (argc > 1) {
    b200::device_config dec_dev = dev;
    dec_dev.max_codeblocks      = 160;
    check_pusch_decoder(dec_dev, argv[1]);
    check_resident_decoder(dec_dev, argv[1]);
  }
  std::printf("%s\n", failures == 0 ? "ALL OK" : "FAILED");
  return failures == 0 ? 0 : 1;
}

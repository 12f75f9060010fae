// Check of the dApp plug-in module (ocudu-dapp-platform_b200/adapters/dapp_module_b200.cpp): the
// module is loaded the way the reference's dApp runtime loads native modules (dlopen, then
// ocudu_dapp_query_v1), its descriptor is validated by the reference's own ABI validator
// (lib/dapp/runtime/abi_validation.cpp, compiled from the reference's sources), and its two Class-A
// interfaces are invoked with the tensors the reference's host hooks build
// (lib/phy/upper/dapp/pusch_dapp_channel_estimator.cpp:183-302 and
// lib/phy/upper/dapp/pusch_dapp_demodulator.cpp:430-600) on seeded allocations. Their outputs are
// compared with the reference's native chain on the same grid and pilots:
//   dapp_channel_estimator  per-symbol estimates equal to port_channel_estimator's bf16 values or one
//                           bf16 unit apart (over 99 % equal), noise variances within 1e-4
//   dapp_receiver           LLRs (before descrambling) against the reference's channel_equalizer (MMSE,
//                           tx scaling 1) + demodulation_mapper on the module's own estimates: |diff|
//                           <= 1, at least 99.9 % equal, post-equalisation noise within 5e-4 (the
//                           reference's equaliser divides by 14-bit reciprocal estimates); and
//                           against the whole reference chain (its port_channel_estimator too): at
//                           least 99.5 % equal
//   dapp_bypass             DM-RS type 2 and device-resident tensors are declined (BYPASS),
//                           malformed tensors are refused (INVALID_INPUT)
// Usage: dapp_check <module.so> [--describe]   (--describe: descriptor checks only, no GPU)
// Test infrastructure: it links the reference's compiled code (oracle/_ref).
#include "lib/phy/upper/signal_processors/dmrs_helper.h"
#include "ocudu/dapp/abi/v1/module.h"
#include "ocudu/dapp/runtime/abi_validation.h"
#include "ocudu/dapp/use_cases/v1/channel_estimator.h"
#include "ocudu/dapp/use_cases/v1/receiver.h"
#include "ocudu/phy/generic_functions/generic_functions_factories.h"
#include "ocudu/phy/support/re_buffer.h"
#include "ocudu/phy/support/resource_grid_reader.h"
#include "ocudu/phy/support/time_alignment_estimator/time_alignment_estimator_factories.h"
#include "ocudu/phy/upper/channel_modulation/channel_modulation_factories.h"
#include "ocudu/phy/upper/equalization/dynamic_ch_est_list.h"
#include "ocudu/phy/upper/equalization/equalization_factories.h"
#include "ocudu/phy/upper/sequence_generators/sequence_generator_factories.h"
#include "ocudu/phy/upper/signal_processors/channel_estimator/factories.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <memory>
#include <random>
#include <vector>

using namespace ocudu;

namespace {

std::mt19937 rng(20261204);

int uniform(int lo, int hi)
{
  return std::uniform_int_distribution<int>(lo, hi)(rng);
}

float gauss()
{
  return std::normal_distribution<float>(0.f, 1.f)(rng);
}

int failures = 0;

void report(const char* name, bool ok, const char* detail)
{
  std::printf("%-22s %s  %s\n", name, ok ? "OK  " : "FAIL", detail);
  if (!ok) {
    ++failures;
  }
}

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

template <typename T>
ocudu_dapp_tensor_view_v1 host_tensor(T* data, uint32_t element, uint32_t access, std::initializer_list<uint64_t> dims)
{
  ocudu_dapp_tensor_view_v1 t{};
  t.struct_size           = sizeof(t);
  t.abi_major             = OCUDU_DAPP_ABI_MAJOR_V1;
  t.abi_minor             = OCUDU_DAPP_ABI_MINOR_V1;
  t.domain                = OCUDU_DAPP_MEM_HOST_V1;
  t.backend_id            = OCUDU_DAPP_BACKEND_HOST_V1;
  t.element_type          = element;
  t.rank                  = static_cast<uint32_t>(dims.size());
  t.access                = access | OCUDU_DAPP_ACCESS_HOST_VISIBLE_V1;
  t.allocation_id         = 1;
  t.allocation_generation = 1;
  t.native_handle         = reinterpret_cast<uintptr_t>(data);
  uint64_t n = 1, k = 0;
  for (uint64_t d : dims) {
    t.dimensions[k++] = d;
    n *= d;
  }
  uint64_t stride = sizeof(T);
  for (unsigned d = t.rank; d != 0; --d) {
    t.byte_strides[d - 1] = stride;
    stride *= t.dimensions[d - 1];
  }
  t.byte_length = n * sizeof(T);
  return t;
}

template <typename M>
ocudu_dapp_typed_metadata_v1 metadata(uint32_t schema, const M& value)
{
  ocudu_dapp_typed_metadata_v1 m{};
  m.struct_size             = sizeof(m);
  m.abi_major               = OCUDU_DAPP_ABI_MAJOR_V1;
  m.abi_minor               = OCUDU_DAPP_ABI_MINOR_V1;
  m.metadata_schema_id      = schema;
  m.metadata_schema_version = 1;
  m.metadata                = {&value, static_cast<uint32_t>(sizeof(value)), 0};
  return m;
}

double bf16_value(cbf16_t v, int part)
{
  uint32_t w;
  std::memcpy(&w, &v, 4);
  const uint32_t b = part == 0 ? (w << 16) : (w & 0xffff0000u);
  float          f;
  std::memcpy(&f, &b, 4);
  return f;
}

// One seeded allocation: a 273-PRB carrier, a contiguous PRB range, DM-RS type 1 at symbols 2 (and
// 11), a two-tap channel per (port, layer), QAM data on the data REs, noise everywhere.
struct allocation {
  unsigned                             nports = 4, nlayers = 1, rb_start = 0, nof_rb = 0, first_symbol = 0, nof_symbols = 14;
  unsigned                             nd = 2, qm = 2;
  float                                scaling = 1.41254f;
  bounded_bitset<MAX_NSYMB_PER_SLOT>   dmrs = bounded_bitset<MAX_NSYMB_PER_SLOT>(MAX_NSYMB_PER_SLOT); // 14 symbols
  std::vector<cbf16_t>                 grid; // [port][14][3276]
  std::unique_ptr<dmrs_symbol_list>    pilots;
  port_channel_estimator::configuration cfg;
};

constexpr unsigned kGridPrb = 273, kGridSubc = 12 * kGridPrb;

allocation make_allocation(pseudo_random_generator& prg, unsigned nlayers, unsigned qm)
{
  allocation a;
  a.nlayers  = nlayers;
  a.qm       = qm;
  a.nof_rb   = static_cast<unsigned>(uniform(1, 273));
  a.rb_start = static_cast<unsigned>(uniform(0, static_cast<int>(kGridPrb - a.nof_rb)));
  a.nd       = uniform(0, 3) != 0 ? 2 : 1;
  a.dmrs.set(2);
  if (a.nd == 2) {
    a.dmrs.set(11);
  }
  const unsigned n_id = static_cast<unsigned>(uniform(0, 1007)), slot = static_cast<unsigned>(uniform(0, 19));
  crb_bitmap     rb_mask(a.rb_start + a.nof_rb);
  rb_mask.fill(a.rb_start, a.rb_start + a.nof_rb);
  const unsigned npil = 6 * a.nof_rb;
  a.pilots            = std::make_unique<dmrs_symbol_list>(re_measurement_dimensions{npil, a.nd, nlayers});
  for (unsigned d = 0, s = 0; s < MAX_NSYMB_PER_SLOT; ++s) {
    if (!a.dmrs.test(s)) {
      continue;
    }
    prg.init(((14 * slot + s + 1) * (2 * n_id + 1) * (1U << 17) + 2 * n_id) % (1U << 31));
    dmrs_sequence_generate(a.pilots->get_symbol(d, 0), prg, M_SQRT1_2, 0, 6, rb_mask);
    if (nlayers > 1) {
      dmrs_pxsch_parameters p1  = get_pxsch_dmrs_params(dmrs_config_type::type1, 1);
      span<cf_t>            dst = a.pilots->get_symbol(d, 1);
      span<const cf_t>      src = a.pilots->get_symbol(d, 0);
      std::copy(src.begin(), src.end(), dst.begin());
      for (unsigned k = 1; k < dst.size(); k += 2) {
        dst[k] *= p1.w_f[1];
      }
    }
    ++d;
  }
  a.cfg.scs          = subcarrier_spacing::kHz30;
  a.cfg.cp           = cyclic_prefix::NORMAL;
  a.cfg.first_symbol = 0;
  a.cfg.nof_symbols  = MAX_NSYMB_PER_SLOT;
  a.cfg.scaling      = a.scaling;
  for (unsigned p = 0; p != a.nports; ++p) {
    a.cfg.rx_ports.push_back(static_cast<uint8_t>(p));
  }
  for (unsigned l = 0; l != nlayers; ++l) {
    a.cfg.dmrs_pattern.push_back(
        {a.dmrs, rb_mask, {}, std::nullopt, get_pxsch_dmrs_params(dmrs_config_type::type1, l).re_pattern});
  }
  a.grid.assign(static_cast<size_t>(a.nports) * MAX_NSYMB_PER_SLOT * kGridSubc, cbf16_t{});
  const float snr  = std::pow(10.f, static_cast<float>(uniform(5, 30)) / 10.f);
  const float sig  = std::sqrt(0.5f / snr);
  const float lvl  = qm == 2 ? 0.7071f : (qm == 4 ? 0.3162f : (qm == 6 ? 0.1543f : 0.0767f));
  const int   nlev = 1 << (qm / 2);
  for (unsigned p = 0; p != a.nports; ++p) {
    cf_t  h0[2], h1[2];
    float tau[2];
    for (unsigned l = 0; l != 2; ++l) {
      h0[l]  = {gauss() * 0.6f, gauss() * 0.6f};
      h1[l]  = {gauss() * 0.4f, gauss() * 0.4f};
      tau[l] = static_cast<float>(uniform(0, 400)) * 1e-9f;
    }
    for (unsigned s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
      for (unsigned k = 0; k != kGridSubc; ++k) {
        cf_t y = {sig * gauss(), sig * gauss()};
        if (k >= 12 * a.rb_start && k < 12 * (a.rb_start + a.nof_rb)) {
          const unsigned j = k - 12 * a.rb_start;
          for (unsigned l = 0; l != nlayers; ++l) {
            const float f = 30e3f * static_cast<float>(j);
            const cf_t  h = h0[l] + h1[l] * std::polar(1.f, -6.2831853f * f * tau[l]);
            if (a.dmrs.test(s)) {
              if ((j % 2) == 0) {
                y += h * a.pilots->get_symbol(s == 2 ? 0 : 1, l)[j / 2] * a.scaling;
              }
            } else {
              const float re = lvl * static_cast<float>(2 * uniform(0, nlev - 1) - (nlev - 1));
              const float im = lvl * static_cast<float>(2 * uniform(0, nlev - 1) - (nlev - 1));
              y += h * cf_t{re, im};
            }
          }
        }
        a.grid[(static_cast<size_t>(p) * MAX_NSYMB_PER_SLOT + s) * kGridSubc + k] = to_cbf16(y);
      }
    }
  }
  return a;
}

// The host hooks' inputs for an allocation: the allocation-local CF32 grid, the pilots times the
// DM-RS scaling with their coordinates, the PUSCH metadata.
struct hook_inputs {
  std::vector<cf_t>            grid;
  std::vector<cf_t>            refs;
  std::vector<uint16_t>        coords;
  std::vector<uint32_t>        data_re;
  ocudu_dapp_pusch_metadata_v1 pusch{};
  ocudu_dapp_dmrs_metadata_v1  dmrs{};
  ocudu_dapp_invocation_v1     invocation{};
};

void make_hook_inputs(const allocation& a, uint32_t worker_id, hook_inputs& in)
{
  const unsigned N = 12 * a.nof_rb, S = a.nof_symbols, P = a.nports, L = a.nlayers;
  in.grid.resize(static_cast<size_t>(P) * S * N);
  for (unsigned p = 0; p != P; ++p) {
    for (unsigned s = 0; s != S; ++s) {
      for (unsigned k = 0; k != N; ++k) {
        in.grid[(static_cast<size_t>(p) * S + s) * N + k] =
            to_cf(a.grid[(static_cast<size_t>(p) * MAX_NSYMB_PER_SLOT + a.first_symbol + s) * kGridSubc + 12 * a.rb_start + k]);
      }
    }
  }
  const unsigned npil = 6 * a.nof_rb, np = a.nd * npil;
  in.refs.assign(static_cast<size_t>(L) * np, cf_t{});
  in.coords.resize(2 * static_cast<size_t>(np));
  for (unsigned d = 0, s = 0; s != MAX_NSYMB_PER_SLOT; ++s) {
    if (!a.dmrs.test(s)) {
      continue;
    }
    for (unsigned k = 0; k != npil; ++k) {
      const unsigned i = d * npil + k;
      for (unsigned l = 0; l != L; ++l) {
        in.refs[static_cast<size_t>(l) * np + i] = a.pilots->get_symbol(d, l)[k] * a.scaling;
      }
      in.coords[2 * i]     = static_cast<uint16_t>(s - a.first_symbol);
      in.coords[2 * i + 1] = static_cast<uint16_t>(2 * k);
    }
    ++d;
  }
  in.data_re.clear();
  for (unsigned s = 0; s != S; ++s) {
    if (a.dmrs.test(a.first_symbol + s)) {
      continue;
    }
    for (unsigned k = 0; k != N; ++k) {
      in.data_re.push_back(s * N + k);
    }
  }
  in.pusch                  = {};
  in.pusch.struct_size      = sizeof(in.pusch);
  in.pusch.abi_major        = OCUDU_DAPP_ABI_MAJOR_V1;
  in.pusch.abi_minor        = OCUDU_DAPP_ABI_MINOR_V1;
  in.pusch.nof_rx_ports     = P;
  in.pusch.nof_layers       = L;
  in.pusch.modulation       = static_cast<ocudu_dapp_modulation_v1>(a.qm);
  in.pusch.start_symbol     = a.first_symbol;
  in.pusch.nof_symbols      = S;
  in.pusch.start_subcarrier = 12 * a.rb_start;
  in.pusch.nof_subcarriers  = N;
  in.pusch.flags            = OCUDU_DAPP_PUSCH_DATA_RE_SELECTION_COMPLETE_V1;
  in.pusch.data_re_indices  = host_tensor(in.data_re.data(), OCUDU_DAPP_ELEMENT_U32_V1, OCUDU_DAPP_ACCESS_READ_V1,
                                          {static_cast<uint64_t>(in.data_re.size())});
  in.pusch.nof_data_re      = static_cast<uint32_t>(in.data_re.size());
  in.pusch.reserved[OCUDU_DAPP_PUSCH_RESERVED_SUBCARRIER_SPACING_HZ_V1] = 30000;
  in.pusch.reserved[OCUDU_DAPP_PUSCH_RESERVED_GRID_NOF_SUBCARRIERS_V1] = kGridSubc;
  in.dmrs                   = {};
  in.dmrs.struct_size       = sizeof(in.dmrs);
  in.dmrs.abi_major         = OCUDU_DAPP_ABI_MAJOR_V1;
  in.dmrs.abi_minor         = OCUDU_DAPP_ABI_MINOR_V1;
  in.dmrs.nof_pilots        = np;
  in.dmrs.flags = OCUDU_DAPP_DMRS_REFERENCE_SYMBOLS_LAYER_COMPLETE_V1 | OCUDU_DAPP_DMRS_COORDINATES_SHARED_ACROSS_LAYERS_V1;
  in.dmrs.dmrs_type         = 1;
  in.dmrs.reference_symbols = host_tensor(in.refs.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_READ_V1, {L, np});
  in.dmrs.coordinates       = host_tensor(in.coords.data(), OCUDU_DAPP_ELEMENT_U16_V1, OCUDU_DAPP_ACCESS_READ_V1, {np, 2});
  in.invocation             = {};
  in.invocation.struct_size = sizeof(in.invocation);
  in.invocation.abi_major   = OCUDU_DAPP_ABI_MAJOR_V1;
  in.invocation.abi_minor   = OCUDU_DAPP_ABI_MINOR_V1;
  in.invocation.invocation_id        = 1;
  in.invocation.worker_id            = worker_id;
  in.invocation.radio_time.numerology = 1;
}

struct module_handle {
  ocudu_dapp_module_v1 m{};
  void*                instance = nullptr;
  const ocudu_dapp_channel_estimator_interface_v1* est = nullptr;
  const ocudu_dapp_receiver_interface_v1*          rx  = nullptr;
};

void check_estimator(module_handle& mh, void* worker, uint32_t worker_id)
{
  auto ta  = create_time_alignment_estimator_dft_factory(create_dft_processor_factory_generic());
  auto ref = create_port_channel_estimator_factory_sw(ta)->create(
      port_channel_estimator_fd_smoothing_strategy::filter, port_channel_estimator_td_interpolation_strategy::interpolate,
      false);
  auto     prg   = create_pseudo_random_generator_sw_factory()->create();
  unsigned calls = 0, bad = 0;
  long     equal = 0, total = 0;
  double   worst_noise = 0;
  for (int t = 0; t < 16; ++t) {
    allocation a = make_allocation(*prg, static_cast<unsigned>(uniform(1, 2)), 2);
    hook_inputs in;
    make_hook_inputs(a, worker_id, in);
    const unsigned P = a.nports, L = a.nlayers, S = a.nof_symbols, N = 12 * a.nof_rb;
    std::vector<cf_t>  est(static_cast<size_t>(P) * L * S * N);
    std::vector<float> noise(static_cast<size_t>(P) * L);
    ocudu_dapp_channel_estimator_input_v1 input{};
    input.invocation = in.invocation;
    input.rx_grid    = host_tensor(in.grid.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_READ_V1, {P, S, N});
    input.pusch      = metadata(OCUDU_DAPP_METADATA_PUSCH_V1, in.pusch);
    input.dmrs       = metadata(OCUDU_DAPP_METADATA_DMRS_V1, in.dmrs);
    ocudu_dapp_channel_estimator_output_v1 output{};
    output.channel_estimates =
        host_tensor(est.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L, S, N});
    output.noise_variances = host_tensor(noise.data(), OCUDU_DAPP_ELEMENT_F32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L});
    const ocudu_dapp_status_v1 st = mh.est->invoke(worker, &input, &output);
    ++calls;
    if (st != OCUDU_DAPP_OK_V1) {
      std::printf("  estimator invoke returned %d\n", static_cast<int>(st));
      ++bad;
      continue;
    }
    vector_grid_reader   reader(a.grid, a.nports, kGridSubc);
    std::vector<cbf16_t> sym(N);
    bool                 ok = true;
    for (unsigned p = 0; p != P; ++p) {
      const port_channel_estimator_results& r = ref->compute(reader, p, *a.pilots, a.cfg);
      for (unsigned l = 0; l != L; ++l) {
        const double e = std::abs(noise[p * L + l] - r.get_noise_variance()) / r.get_noise_variance();
        worst_noise    = std::max(worst_noise, e);
        ok             = ok && e <= 1e-4;
        for (unsigned s = 0; s != S; ++s) {
          r.get_symbol_ch_estimate(sym, a.first_symbol + s, l);
          for (unsigned k = 0; k != N; ++k) {
            const cf_t   g   = est[((static_cast<size_t>(p) * L + l) * S + s) * N + k];
            const double mag = std::hypot(bf16_value(sym[k], 0), bf16_value(sym[k], 1));
            for (int part = 0; part < 2; ++part) {
              const double want = bf16_value(sym[k], part), got = part == 0 ? g.real() : g.imag();
              const double top  = std::max(std::abs(want), std::abs(got));
              const double ulp  = top > 0 ? std::ldexp(1.0, std::ilogb(top) - 7) : 0.0;
              ok                = ok && std::abs(want - got) <= ulp + 1e-4 * mag;
              equal += want == got;
              ++total;
            }
          }
        }
      }
    }
    bad += ok ? 0 : 1;
  }
  char detail[200];
  std::snprintf(detail, sizeof(detail), "%u allocations, %.4f of the estimate components equal, noise rel %.2e, %u off",
                calls, double(equal) / double(std::max(total, 1L)), worst_noise, bad);
  report("dapp_channel_estimator", bad == 0 && equal > 0.99 * total, detail);
}

// The reference's equaliser and demapper over the data REs of an allocation, one OFDM symbol at a
// time as pusch_demodulator_impl.cpp:330-420 runs them (they take one symbol's REs): est_sym rows
// [port][layer][symbol] of cbf16 estimates, nv the port noise variances.
void reference_llrs(const allocation& a, const hook_inputs& in, const std::vector<std::vector<cbf16_t>>& est_sym,
                    const std::vector<float>& nv, channel_equalizer& eq_ref, demodulation_mapper& demap,
                    std::vector<log_likelihood_ratio>& want, std::vector<float>& var)
{
  const unsigned P = a.nports, L = a.nlayers, S = a.nof_symbols, N = 12 * a.nof_rb, qm = a.qm;
  const unsigned nre = static_cast<unsigned>(in.data_re.size());
  std::vector<cf_t> eq(static_cast<size_t>(nre) * L);
  var.assign(static_cast<size_t>(nre) * L, 0.f);
  want.assign(static_cast<size_t>(nre) * L * qm, log_likelihood_ratio(0));
  for (unsigned i0 = 0; i0 != nre;) {
    const unsigned s  = in.data_re[i0] / N;
    unsigned       i1 = i0;
    while (i1 != nre && in.data_re[i1] / N == s) {
      ++i1;
    }
    const unsigned             n = i1 - i0;
    dynamic_re_buffer<cbf16_t> y(P, n);
    dynamic_ch_est_list        h(n, P, L);
    for (unsigned p = 0; p != P; ++p) {
      for (unsigned i = 0; i != n; ++i) {
        const unsigned k  = in.data_re[i0 + i] % N;
        y.get_slice(p)[i] = a.grid[(static_cast<size_t>(p) * MAX_NSYMB_PER_SLOT + a.first_symbol + s) * kGridSubc +
                                   12 * a.rb_start + k];
        for (unsigned l = 0; l != L; ++l) {
          h.get_channel(p, l)[i] = est_sym[(static_cast<size_t>(p) * L + l) * S + s][k];
        }
      }
    }
    span<cf_t>  eq_s  = span<cf_t>(eq).subspan(static_cast<size_t>(i0) * L, static_cast<size_t>(n) * L);
    span<float> var_s = span<float>(var).subspan(static_cast<size_t>(i0) * L, static_cast<size_t>(n) * L);
    eq_ref.equalize(eq_s, var_s, y, h, nv, 1.0f);
    demap.demodulate_soft(span<log_likelihood_ratio>(want).subspan(static_cast<size_t>(i0) * L * qm,
                                                                    static_cast<size_t>(n) * L * qm),
                          eq_s, var_s, static_cast<modulation_scheme>(qm));
    i0 = i1;
  }
}

// Two references for the module's receiver: (a) the reference's equaliser and demapper on the
// module's own channel estimates and noise (its channel estimator interface, checked above) - the
// receiver stage proper, held to +-1 LSB and the equaliser's 2.5e-4; (b) the reference's whole
// chain from its own estimator, where the one-bf16-unit estimate differences propagate (reported,
// held to 99.5 % equal LLRs).
void check_receiver(module_handle& mh, void* w_rx, uint32_t rx_id, void* w_est, uint32_t est_id)
{
  auto ta  = create_time_alignment_estimator_dft_factory(create_dft_processor_factory_generic());
  auto ref = create_port_channel_estimator_factory_sw(ta)->create(
      port_channel_estimator_fd_smoothing_strategy::filter, port_channel_estimator_td_interpolation_strategy::interpolate,
      false);
  auto     eq_ref = create_channel_equalizer_generic_factory(channel_equalizer_algorithm_type::mmse)->create();
  auto     demap  = create_demodulation_mapper_factory()->create();
  auto     prg    = create_pseudo_random_generator_sw_factory()->create();
  unsigned calls = 0, bad = 0;
  long     equal = 0, total = 0, equal_full = 0;
  int      worst = 0, worst_full = 0;
  double   worst_var = 0;
  for (int t = 0; t < 16; ++t) {
    const unsigned qm = 2u * static_cast<unsigned>(1 + t % 4);
    allocation     a  = make_allocation(*prg, static_cast<unsigned>(uniform(1, 2)), qm);
    hook_inputs    in;
    make_hook_inputs(a, rx_id, in);
    const unsigned P = a.nports, L = a.nlayers, S = a.nof_symbols, N = 12 * a.nof_rb;
    const unsigned nre = static_cast<unsigned>(in.data_re.size());
    std::vector<int8_t> llrs(static_cast<size_t>(nre) * L * qm);
    std::vector<float>  post_noise(static_cast<size_t>(nre) * L);
    std::vector<cf_t>   eq_symbols(static_cast<size_t>(nre) * L);
    ocudu_dapp_receiver_input_v1 input{};
    input.invocation = in.invocation;
    input.rx_grid    = host_tensor(in.grid.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_READ_V1, {P, S, N});
    input.pusch      = metadata(OCUDU_DAPP_METADATA_PUSCH_V1, in.pusch);
    input.dmrs       = metadata(OCUDU_DAPP_METADATA_DMRS_V1, in.dmrs);
    ocudu_dapp_receiver_metrics_v1 metrics{};
    metrics.struct_size             = sizeof(metrics);
    metrics.abi_major               = OCUDU_DAPP_ABI_MAJOR_V1;
    metrics.abi_minor               = OCUDU_DAPP_ABI_MINOR_V1;
    metrics.post_equalization_noise = host_tensor(post_noise.data(), OCUDU_DAPP_ELEMENT_F32_V1, OCUDU_DAPP_ACCESS_WRITE_V1,
                                                  {nre, L});
    metrics.equalized_symbols = host_tensor(eq_symbols.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_WRITE_V1,
                                            {nre, L});
    ocudu_dapp_receiver_output_v1 output{};
    output.llrs    = host_tensor(llrs.data(), OCUDU_DAPP_ELEMENT_I8_V1, OCUDU_DAPP_ACCESS_WRITE_V1,
                                 {static_cast<uint64_t>(nre) * L * qm});
    output.metrics = metadata(OCUDU_DAPP_METADATA_RECEIVER_METRICS_V1, metrics);
    const ocudu_dapp_status_v1 st = mh.rx->invoke(w_rx, &input, &output);
    ++calls;
    const uint32_t want_flags = OCUDU_DAPP_RECEIVER_METRICS_VALID_V1 | OCUDU_DAPP_RECEIVER_EQUALIZED_SYMBOLS_VALID_V1;
    // The module's channel estimates of the same allocation (estimator interface).
    std::vector<cf_t>  mest(static_cast<size_t>(P) * L * S * N);
    std::vector<float> mnoise(static_cast<size_t>(P) * L);
    ocudu_dapp_channel_estimator_input_v1 ein{};
    ein.invocation           = in.invocation;
    ein.invocation.worker_id = est_id;
    ein.rx_grid              = input.rx_grid;
    ein.pusch                = input.pusch;
    ein.dmrs                 = input.dmrs;
    ocudu_dapp_channel_estimator_output_v1 eout{};
    eout.channel_estimates = host_tensor(mest.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L, S, N});
    eout.noise_variances   = host_tensor(mnoise.data(), OCUDU_DAPP_ELEMENT_F32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L});
    const ocudu_dapp_status_v1 se = mh.est->invoke(w_est, &ein, &eout);
    if (st != OCUDU_DAPP_OK_V1 || output.reserved0 != want_flags || se != OCUDU_DAPP_OK_V1) {
      std::printf("  receiver invoke returned %d, flags %u, estimator %d\n", static_cast<int>(st), output.reserved0,
                  static_cast<int>(se));
      ++bad;
      continue;
    }
    // (a) on the module's estimates (CF32 values that are bf16 values: the conversion is exact).
    std::vector<std::vector<cbf16_t>> est_m(static_cast<size_t>(P) * L * S, std::vector<cbf16_t>(N));
    std::vector<float>                nv_m(P);
    for (unsigned p = 0; p != P; ++p) {
      nv_m[p] = mnoise[static_cast<size_t>(p) * L];
      for (unsigned l = 0; l != L; ++l) {
        for (unsigned s = 0; s != S; ++s) {
          for (unsigned k = 0; k != N; ++k) {
            est_m[(static_cast<size_t>(p) * L + l) * S + s][k] =
                to_cbf16(mest[((static_cast<size_t>(p) * L + l) * S + s) * N + k]);
          }
        }
      }
    }
    std::vector<log_likelihood_ratio> want;
    std::vector<float>                var;
    reference_llrs(a, in, est_m, nv_m, *eq_ref, *demap, want, var);
    bool ok = true;
    for (size_t i = 0; i != want.size(); ++i) {
      const int d = std::abs(static_cast<int>(want[i].to_value_type()) - static_cast<int>(llrs[i]));
      worst       = std::max(worst, d);
      equal += d == 0;
      ++total;
      ok = ok && d <= 1;
    }
    float max_v = 0.f;
    for (float v : var) {
      if (std::isfinite(v)) {
        max_v = std::max(max_v, v);
      }
    }
    for (size_t i = 0; i != var.size(); ++i) {
      if (std::isfinite(var[i]) || std::isfinite(post_noise[i])) {
        const double e = std::abs(var[i] - post_noise[i]) / std::max(std::abs(var[i]), 1e-3f * max_v);
        worst_var      = std::max(worst_var, e);
        ok             = ok && e <= 5e-4; // the reference's equaliser: 14-bit reciprocal estimates
      }
    }
    // (b) the reference's whole chain from its own estimator.
    vector_grid_reader                reader(a.grid, a.nports, kGridSubc);
    std::vector<std::vector<cbf16_t>> est_r(static_cast<size_t>(P) * L * S, std::vector<cbf16_t>(N));
    std::vector<float>                nv_r(P);
    for (unsigned p = 0; p != P; ++p) {
      const port_channel_estimator_results& r = ref->compute(reader, p, *a.pilots, a.cfg);
      nv_r[p]                                 = r.get_noise_variance();
      for (unsigned l = 0; l != L; ++l) {
        for (unsigned s = 0; s != S; ++s) {
          r.get_symbol_ch_estimate(est_r[(static_cast<size_t>(p) * L + l) * S + s], a.first_symbol + s, l);
        }
      }
    }
    reference_llrs(a, in, est_r, nv_r, *eq_ref, *demap, want, var);
    for (size_t i = 0; i != want.size(); ++i) {
      const int d = std::abs(static_cast<int>(want[i].to_value_type()) - static_cast<int>(llrs[i]));
      worst_full  = std::max(worst_full, d);
      equal_full += d == 0;
    }
    bad += ok ? 0 : 1;
  }
  char detail[260];
  std::snprintf(detail, sizeof(detail),
                "%u allocations, %ld LLRs: on its own estimates %.5f equal, max |diff| %d, noise rel %.2e, %u off; "
                "whole reference chain %.5f equal, max |diff| %d",
                calls, total, double(equal) / double(std::max(total, 1L)), worst, worst_var, bad,
                double(equal_full) / double(std::max(total, 1L)), worst_full);
  report("dapp_receiver",
         bad == 0 && equal >= total - total / 1000 && equal_full >= total - total / 200, detail);
}

void check_bypass(module_handle& mh, void* worker, uint32_t worker_id)
{
  auto        prg = create_pseudo_random_generator_sw_factory()->create();
  allocation  a   = make_allocation(*prg, 1, 2);
  hook_inputs in;
  make_hook_inputs(a, worker_id, in);
  const unsigned P = a.nports, L = 1, S = a.nof_symbols, N = 12 * a.nof_rb;
  std::vector<cf_t>  est(static_cast<size_t>(P) * L * S * N);
  std::vector<float> noise(P);
  auto run = [&](ocudu_dapp_dmrs_metadata_v1 dmrs, ocudu_dapp_tensor_view_v1 grid) {
    ocudu_dapp_channel_estimator_input_v1 input{};
    input.invocation = in.invocation;
    input.rx_grid    = grid;
    input.pusch      = metadata(OCUDU_DAPP_METADATA_PUSCH_V1, in.pusch);
    input.dmrs       = metadata(OCUDU_DAPP_METADATA_DMRS_V1, dmrs);
    ocudu_dapp_channel_estimator_output_v1 output{};
    output.channel_estimates = host_tensor(est.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L, S, N});
    output.noise_variances   = host_tensor(noise.data(), OCUDU_DAPP_ELEMENT_F32_V1, OCUDU_DAPP_ACCESS_WRITE_V1, {P, L});
    return mh.est->invoke(worker, &input, &output);
  };
  const auto grid = host_tensor(in.grid.data(), OCUDU_DAPP_ELEMENT_CF32_V1, OCUDU_DAPP_ACCESS_READ_V1, {P, S, N});
  ocudu_dapp_dmrs_metadata_v1 type2 = in.dmrs;
  type2.dmrs_type                   = 2;
  ocudu_dapp_tensor_view_v1 device  = grid;
  device.domain                     = OCUDU_DAPP_MEM_ACCELERATOR_DEVICE_V1;
  device.backend_id                 = OCUDU_DAPP_BACKEND_CUDA_V1;
  ocudu_dapp_tensor_view_v1 wrong   = grid;
  wrong.dimensions[2]               = N + 1;
  const auto s_type2 = run(type2, grid), s_device = run(in.dmrs, device), s_wrong = run(in.dmrs, wrong);
  const auto s_ok    = run(in.dmrs, grid);
  char       detail[200];
  std::snprintf(detail, sizeof(detail), "type 2 -> %d, device grid -> %d, bad extent -> %d, valid -> %d",
                static_cast<int>(s_type2), static_cast<int>(s_device), static_cast<int>(s_wrong), static_cast<int>(s_ok));
  report("dapp_bypass",
         s_type2 == OCUDU_DAPP_BYPASS_V1 && s_device == OCUDU_DAPP_BYPASS_V1 && s_wrong == OCUDU_DAPP_INVALID_INPUT_V1 &&
             s_ok == OCUDU_DAPP_OK_V1,
         detail);
}

} // namespace

int main(int argc, char** argv)
{
  if (argc < 2) {
    std::fprintf(stderr, "usage: dapp_check <module.so> [--describe]\n");
    return 2;
  }
  std::setvbuf(stdout, nullptr, _IONBF, 0); // every line reaches the log, also if a check aborts
  const bool describe = argc > 2 && std::strcmp(argv[2], "--describe") == 0;
  void*      so       = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
  if (so == nullptr) {
    std::fprintf(stderr, "dlopen: %s\n", dlerror());
    return 2;
  }
  auto query = reinterpret_cast<ocudu_dapp_query_v1_fn>(dlsym(so, "ocudu_dapp_query_v1"));
  if (query == nullptr) {
    std::fprintf(stderr, "no ocudu_dapp_query_v1\n");
    return 2;
  }
  ocudu_dapp_host_info_v1 host{};
  host.struct_size  = sizeof(host);
  host.abi_major    = OCUDU_DAPP_ABI_MAJOR_V1;
  host.abi_minor    = OCUDU_DAPP_ABI_MINOR_V1;
  host.backend_mask = 1u << OCUDU_DAPP_BACKEND_CUDA_V1;
  module_handle mh;
  const auto    qs = query(&host, &mh.m);
  const auto    ve = ocudu::dapp::validate_module_descriptor(&mh.m);
  bool          ifaces_ok = mh.m.nof_interfaces == 2;
  for (uint32_t i = 0; i < mh.m.nof_interfaces && ifaces_ok; ++i) {
    const auto& d = mh.m.interfaces[i];
    ifaces_ok     = ifaces_ok && ocudu::dapp::is_class_a_interface(d.interface_id) &&
                d.dapp_class == OCUDU_DAPP_CLASS_A_INLINE_V1;
    if (d.interface_id == OCUDU_DAPP_INTERFACE_CHANNEL_ESTIMATOR_V1) {
      mh.est = static_cast<const ocudu_dapp_channel_estimator_interface_v1*>(d.interface_vtable);
    } else if (d.interface_id == OCUDU_DAPP_INTERFACE_RECEIVER_V1) {
      mh.rx = static_cast<const ocudu_dapp_receiver_interface_v1*>(d.interface_vtable);
    }
  }
  ifaces_ok = ifaces_ok && mh.est != nullptr && mh.rx != nullptr;
  char detail[200];
  std::snprintf(detail, sizeof(detail), "query %d, reference validator: %s, %u Class-A interfaces (%s)",
                static_cast<int>(qs), ocudu::dapp::to_string(ve), mh.m.nof_interfaces,
                ifaces_ok ? "channel estimator v1, receiver v1" : "unexpected");
  report("dapp_module", qs == OCUDU_DAPP_OK_V1 && ve == ocudu::dapp::validation_error::none && ifaces_ok, detail);
  if (!describe && failures == 0) {
    if (mh.m.create(nullptr, nullptr, &mh.instance) != OCUDU_DAPP_OK_V1 ||
        mh.m.configure(mh.instance, nullptr) != OCUDU_DAPP_OK_V1 || mh.m.prepare(mh.instance, nullptr) != OCUDU_DAPP_OK_V1 ||
        mh.m.warmup(mh.instance, nullptr) != OCUDU_DAPP_OK_V1 || mh.m.start(mh.instance) != OCUDU_DAPP_OK_V1) {
      report("dapp_lifecycle", false, "create / configure / prepare / warmup / start failed");
    } else {
      void* w_est = nullptr;
      void* w_rx  = nullptr;
      const auto se = mh.est->worker.create_worker_context(mh.instance, 3, &w_est);
      const auto sr = mh.rx->worker.create_worker_context(mh.instance, 5, &w_rx);
      if (se != OCUDU_DAPP_OK_V1 || sr != OCUDU_DAPP_OK_V1) {
        std::snprintf(detail, sizeof(detail), "worker contexts: %d %d", static_cast<int>(se), static_cast<int>(sr));
        report("dapp_lifecycle", false, detail);
      } else {
        check_estimator(mh, w_est, 3);
        check_receiver(mh, w_rx, 5, w_est, 3);
        check_bypass(mh, w_est, 3);
        mh.est->worker.destroy_worker_context(mh.instance, w_est);
        mh.rx->worker.destroy_worker_context(mh.instance, w_rx);
      }
      const bool stopped = mh.m.quiesce(mh.instance, 0) == OCUDU_DAPP_OK_V1 && mh.m.stop(mh.instance) == OCUDU_DAPP_OK_V1;
      mh.m.destroy(mh.instance);
      report("dapp_lifecycle", stopped, "create, configure, prepare, warmup, start, two workers, quiesce, stop, destroy");
    }
  }
  std::printf("%s\n", failures == 0 ? "ALL OK" : "FAILED");
  return failures == 0 ? 0 : 1;
}

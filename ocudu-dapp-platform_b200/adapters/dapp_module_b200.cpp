// dApp plug-in module over the pusch_b200 GPU library: the reference's Class-A PUSCH interfaces
//   channel estimator v1 (include/ocudu/dapp/use_cases/v1/channel_estimator.h:22-43) and
//   receiver v1          (include/ocudu/dapp/use_cases/v1/receiver.h:62-88),
// exported through the module ABI's entry point ocudu_dapp_query_v1
// (include/ocudu/dapp/abi/v1/module.h), so that the reference's dApp runtime
// (lib/dapp/runtime/module_loader.cpp) loads it like any other native module. The host side that
// calls these interfaces is lib/phy/upper/dapp/pusch_dapp_channel_estimator.cpp (estimator hook,
// decorating dmrs_pusch_estimator) and lib/phy/upper/dapp/pusch_dapp_demodulator.cpp (receiver
// hook); this module serves their host-memory (HOST / HOST_PINNED / MANAGED) invocations.
//
// Channel estimator: rx_grid CF32 [rx_port, symbol, subcarrier] of one contiguous allocation, the
// DM-RS pilots as explicit reference symbols CF32 [layer, pilot] at coordinates U16 [pilot, 2]
// -> channel_estimates CF32 [rx_port, layer, symbol, subcarrier] and noise_variances F32
// [rx_port, layer]. Per receive port this is pg_port_channel_estimate_host: the estimator that
// replaces port_channel_estimator (LS, RC-FIR smoothing, linear time interpolation), whose
// per-symbol estimates are bf16 values; they are returned as CF32 (exact), which the host rounds to
// cbf16 again without change.
//
// Receiver: the same inputs plus the data REs (data_re_indices U32 or data_re_mask U8) and the
// modulation -> llrs I8 [data_re * layers * modulation_order] before descrambling, in data-RE order
// (then layer, then bit), as the host's demodulator would produce them (estimation, equalisation
// with tx scaling 1 as pusch_demodulator_impl.cpp:348-349, soft demapping): pg_equalize_host and
// pg_demodulate_soft_host. The optional metrics request (post-equalisation noise F32
// [data_re, layer], equalised symbols CF32 [data_re, layer]) is filled and flagged.
//
// Inputs the GPU path does not cover return OCUDU_DAPP_BYPASS_V1 (the host then runs its own
// implementation): device-resident tensors, DM-RS type 2 or other than CDM group 0, more than two
// DM-RS symbols or layers, pilots that are not QPSK, an allocation that overlaps DC, transform
// precoding. Malformed inputs return OCUDU_DAPP_INVALID_INPUT_V1, GPU failures
// OCUDU_DAPP_DEVICE_ERROR_V1.
#include "ocudu/dapp/abi/v1/module.h"
#include "ocudu/dapp/use_cases/v1/channel_estimator.h"
#include "ocudu/dapp/use_cases/v1/receiver.h"

#include "../../include/pusch_b200.h"

#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace {

constexpr unsigned kMaxPorts   = 4;
constexpr unsigned kMaxLayers  = 2;
constexpr unsigned kMaxPrb     = 275;
constexpr unsigned kSymbols    = 14;
constexpr float    kPilotValue = 0.70710678118654752440F; // DM-RS QPSK component magnitude

struct instance_state {
  int device = 0;
};

// One GPU context per worker: the interfaces run PER_WORKER, so a worker's calls never overlap.
struct worker_state {
  instance_state* inst      = nullptr;
  uint32_t        worker_id = 0;
  pg_context*     ctx       = nullptr;
  // Estimation of the current invocation.
  unsigned              nof_ports = 0, nof_layers = 0, nof_symbols = 0, nof_subc = 0, first_symbol = 0;
  std::vector<uint32_t> grid;     // cbf16 [port][14][nof_subc]
  std::vector<uint32_t> sym_est;  // cbf16 [port][14][layer][nof_subc]
  std::vector<float>    freq;     // per port call
  std::vector<float>    pilots;   // per port call: [dmrs symbol][layer][6 nof_rb] complex
  float                 noise[kMaxPorts] = {};
  // Receiver scratch.
  std::vector<uint32_t> y, h;
  std::vector<float>    eq, eq_var;
  std::vector<uint32_t> idx;
};

uint32_t to_cbf16(float re, float im)
{
  // Round to nearest even (the resource grid's cbf16 conversion); a CF32 grid that came from a
  // cbf16 grid converts back exactly.
  auto bf = [](float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) {
      return (uint32_t)((u >> 16) | 0x40u);
    }
    return (uint32_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
  };
  return bf(re) | (bf(im) << 16);
}

float bf16_part(uint32_t w, int hi)
{
  const uint32_t b = hi ? (w & 0xffff0000u) : (w << 16);
  float          f;
  std::memcpy(&f, &b, 4);
  return f;
}

bool host_domain(uint32_t d)
{
  return d == OCUDU_DAPP_MEM_HOST_V1 || d == OCUDU_DAPP_MEM_HOST_PINNED_V1 || d == OCUDU_DAPP_MEM_MANAGED_COHERENT_V1;
}

// A dense row-major host tensor of the given element type and extents with the given access.
// Returns 1 when it is, 0 when it lives in memory this module does not address (bypass), -1 when it
// is malformed.
int check_tensor(const ocudu_dapp_tensor_view_v1& t, uint32_t element, size_t element_bytes,
                 std::initializer_list<uint64_t> dims, uint32_t access)
{
  if (t.struct_size < sizeof(ocudu_dapp_tensor_view_v1) || t.abi_major != OCUDU_DAPP_ABI_MAJOR_V1) {
    return -1;
  }
  if (!host_domain(t.domain)) {
    return 0;
  }
  if (t.element_type != element || t.rank != dims.size() || t.native_handle == 0 || (t.access & access) != access) {
    return -1;
  }
  uint64_t stride = element_bytes;
  for (size_t k = dims.size(); k-- > 0;) {
    const uint64_t d = *(dims.begin() + k);
    if (t.dimensions[k] != d || t.byte_strides[k] != stride) {
      return -1;
    }
    stride *= d;
  }
  return t.byte_length >= stride ? 1 : -1;
}

template <typename T>
T* tensor_data(const ocudu_dapp_tensor_view_v1& t)
{
  return reinterpret_cast<T*>(static_cast<uintptr_t>(t.native_handle + t.byte_offset));
}

template <typename M>
const M* typed_metadata(const ocudu_dapp_typed_metadata_v1& m, uint32_t schema)
{
  if (m.metadata_schema_id != schema || m.metadata.data == nullptr || m.metadata.size < sizeof(M)) {
    return nullptr;
  }
  const M* v = static_cast<const M*>(m.metadata.data);
  return v->struct_size >= sizeof(M) && v->abi_major == OCUDU_DAPP_ABI_MAJOR_V1 ? v : nullptr;
}

// Channel estimation of one allocation into the worker's sym_est / noise. Returns a dApp status.
ocudu_dapp_status_v1 estimate(worker_state& w, const ocudu_dapp_tensor_view_v1& rx_grid,
                              const ocudu_dapp_pusch_metadata_v1& pusch, const ocudu_dapp_dmrs_metadata_v1& dmrs,
                              float scs_khz)
{
  const unsigned P = pusch.nof_rx_ports, L = pusch.nof_layers, S = pusch.nof_symbols, N = pusch.nof_subcarriers;
  if (P == 0 || P > kMaxPorts || (P != 1 && P != 2 && P != 4) || L == 0 || L > kMaxLayers || L > P || S == 0 ||
      pusch.start_symbol + S > kSymbols || N == 0 || N % 12 != 0 || N / 12 > kMaxPrb) {
    return OCUDU_DAPP_BYPASS_V1;
  }
  if ((pusch.flags & (OCUDU_DAPP_PUSCH_TRANSFORM_PRECODING_V1 | OCUDU_DAPP_PUSCH_DC_OVERLAP_V1)) != 0) {
    return OCUDU_DAPP_BYPASS_V1;
  }
  if (dmrs.dmrs_type != 1 || (dmrs.flags & OCUDU_DAPP_DMRS_COORDINATES_SHARED_ACROSS_LAYERS_V1) == 0) {
    return OCUDU_DAPP_BYPASS_V1;
  }
  const int g = check_tensor(rx_grid, OCUDU_DAPP_ELEMENT_CF32_V1, 8, {P, S, N}, OCUDU_DAPP_ACCESS_READ_V1);
  if (g <= 0) {
    return g == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
  }
  const unsigned npil_sym = N / 2;
  const unsigned np       = dmrs.nof_pilots;
  if (np == 0 || np % npil_sym != 0 || np / npil_sym > 2) {
    return OCUDU_DAPP_BYPASS_V1;
  }
  const unsigned nd     = np / npil_sym;
  const int      coords = check_tensor(dmrs.coordinates, OCUDU_DAPP_ELEMENT_U16_V1, 2, {np, 2}, OCUDU_DAPP_ACCESS_READ_V1);
  const unsigned rplanes = (dmrs.flags & OCUDU_DAPP_DMRS_REFERENCE_SYMBOLS_LAYER_COMPLETE_V1) != 0 ? L : 1;
  const int      refs = check_tensor(dmrs.reference_symbols, OCUDU_DAPP_ELEMENT_CF32_V1, 8, {rplanes, np},
                                     OCUDU_DAPP_ACCESS_READ_V1);
  if (coords <= 0 || refs <= 0) {
    return coords == 0 || refs == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
  }
  // Type 1, CDM group 0: every DM-RS symbol carries pilots on subcarriers 0, 2, 4, ... in order.
  const uint16_t* c   = tensor_data<const uint16_t>(dmrs.coordinates);
  const float*    r   = tensor_data<const float>(dmrs.reference_symbols);
  uint16_t        dsym[2] = {0, 0};
  for (unsigned d = 0; d != nd; ++d) {
    dsym[d] = c[2 * (d * npil_sym)];
    if (dsym[d] >= S || (d == 1 && dsym[1] <= dsym[0])) {
      return OCUDU_DAPP_BYPASS_V1;
    }
    for (unsigned k = 0; k != npil_sym; ++k) {
      const uint16_t* e = c + 2 * (d * npil_sym + k);
      if (e[0] != dsym[d] || e[1] != 2 * k) {
        return OCUDU_DAPP_BYPASS_V1;
      }
    }
  }
  // The pilots are the QPSK DM-RS sequence times the DM-RS scaling: both follow from the reference
  // symbols (signs and magnitude).
  const float beta = std::fabs(r[0]) / kPilotValue;
  if (!(beta > 0.f) || !std::isfinite(beta)) {
    return OCUDU_DAPP_BYPASS_V1;
  }
  const float tol = 1e-5f * std::fabs(r[0]);
  w.pilots.assign(static_cast<size_t>(nd) * L * npil_sym * 2, 0.f);
  for (unsigned d = 0; d != nd; ++d) {
    for (unsigned k = 0; k != npil_sym; ++k) {
      const float re = r[2 * (d * npil_sym + k)], im = r[2 * (d * npil_sym + k) + 1];
      if (std::fabs(std::fabs(re) - std::fabs(r[0])) > tol || std::fabs(std::fabs(im) - std::fabs(r[0])) > tol) {
        return OCUDU_DAPP_BYPASS_V1; // not a QPSK sequence (e.g. a low-PAPR sequence)
      }
      for (unsigned l = 0; l != L; ++l) {
        // Layer 1: the frequency OCC of CDM group 0, port 1 (w_f = +1, -1 on odd pilots).
        const float s = (l == 1 && (k & 1u)) ? -1.f : 1.f;
        float*      p = w.pilots.data() + 2 * ((static_cast<size_t>(d) * L + l) * npil_sym + k);
        p[0]          = s * std::copysign(kPilotValue, re);
        p[1]          = s * std::copysign(kPilotValue, im);
      }
    }
  }

  w.nof_ports    = P;
  w.nof_layers   = L;
  w.nof_symbols  = S;
  w.nof_subc     = N;
  w.first_symbol = pusch.start_symbol;
  const float* x = tensor_data<const float>(rx_grid);
  w.grid.assign(static_cast<size_t>(P) * kSymbols * N, 0u);
  for (unsigned p = 0; p != P; ++p) {
    for (unsigned s = 0; s != S; ++s) {
      const float* src = x + 2 * ((static_cast<size_t>(p) * S + s) * N);
      uint32_t*    dst = w.grid.data() + (static_cast<size_t>(p) * kSymbols + pusch.start_symbol + s) * N;
      for (unsigned k = 0; k != N; ++k) {
        dst[k] = to_cbf16(src[2 * k], src[2 * k + 1]);
      }
    }
  }
  pg_port_estimate_cfg cfg = {};
  cfg.grid_nof_subc        = N;
  cfg.scaling              = beta;
  cfg.rb_start             = 0;
  cfg.nof_rb               = static_cast<uint16_t>(N / 12);
  cfg.dmrs_symbol_mask     = static_cast<uint16_t>(0);
  for (unsigned d = 0; d != nd; ++d) {
    cfg.dmrs_symbol_mask |= static_cast<uint16_t>(1u << (pusch.start_symbol + dsym[d]));
  }
  cfg.first_symbol = static_cast<uint8_t>(pusch.start_symbol);
  cfg.nof_symbols  = static_cast<uint8_t>(S);
  cfg.nof_layers   = static_cast<uint8_t>(L);
  cfg.scs_khz      = static_cast<uint8_t>(scs_khz);
  w.sym_est.assign(static_cast<size_t>(P) * kSymbols * L * N, 0u);
  w.freq.resize(static_cast<size_t>(nd) * L * N * 2);
  for (unsigned p = 0; p != P; ++p) {
    pg_port_estimate_result res = {};
    if (pg_port_channel_estimate_host(w.ctx, &cfg, w.grid.data() + static_cast<size_t>(p) * kSymbols * N,
                                      w.pilots.data(), w.freq.data(),
                                      w.sym_est.data() + static_cast<size_t>(p) * kSymbols * L * N, &res) != PG_OK) {
      return OCUDU_DAPP_DEVICE_ERROR_V1;
    }
    // The port's noise variance as the estimator reports it (the host applies its own floor to the
    // estimator interface's output; the receiver equalises with it unfloored, as the host's own
    // demodulator does).
    w.noise[p] = res.noise_var;
  }
  return OCUDU_DAPP_OK_V1;
}

float scs_khz_of(const ocudu_dapp_pusch_metadata_v1& pusch, uint32_t numerology)
{
  const uint64_t hz = pusch.reserved[OCUDU_DAPP_PUSCH_RESERVED_SUBCARRIER_SPACING_HZ_V1];
  if (hz != 0) {
    return static_cast<float>(hz / 1000u);
  }
  return static_cast<float>(15u << (numerology < 4 ? numerology : 1));
}

ocudu_dapp_status_v1 create_worker(void* instance, uint32_t worker_id, void** out)
{
  if (instance == nullptr || out == nullptr) {
    return OCUDU_DAPP_INVALID_INPUT_V1;
  }
  auto* w = new (std::nothrow) worker_state;
  if (w == nullptr) {
    return OCUDU_DAPP_RESOURCE_V1;
  }
  w->inst      = static_cast<instance_state*>(instance);
  w->worker_id = worker_id;
  pg_config cfg = {w->inst->device, 4, 0};
  if (pg_create(&cfg, &w->ctx) != PG_OK) {
    delete w;
    return OCUDU_DAPP_DEVICE_ERROR_V1;
  }
  // Host scratch for the largest allocation, so that invocations do not allocate.
  const size_t re_max = static_cast<size_t>(kSymbols) * kMaxPrb * 12;
  w->grid.reserve(kMaxPorts * re_max);
  w->sym_est.reserve(kMaxPorts * kMaxLayers * re_max);
  w->freq.reserve(2 * kMaxLayers * kMaxPrb * 12 * 2);
  w->pilots.reserve(2 * kMaxLayers * kMaxPrb * 6 * 2);
  w->y.reserve(kMaxPorts * re_max);
  w->h.reserve(kMaxPorts * kMaxLayers * re_max);
  w->eq.reserve(2 * kMaxLayers * re_max);
  w->eq_var.reserve(kMaxLayers * re_max);
  w->idx.reserve(re_max);
  *out = w;
  return OCUDU_DAPP_OK_V1;
}

void destroy_worker(void*, void* context)
{
  auto* w = static_cast<worker_state*>(context);
  if (w != nullptr) {
    pg_destroy(w->ctx);
    delete w;
  }
}

ocudu_dapp_status_v1 estimator_invoke(void* context, const ocudu_dapp_channel_estimator_input_v1* in,
                                      ocudu_dapp_channel_estimator_output_v1* out)
{
  auto* w = static_cast<worker_state*>(context);
  if (w == nullptr || in == nullptr || out == nullptr || in->invocation.worker_id != w->worker_id) {
    return OCUDU_DAPP_INVALID_INPUT_V1;
  }
  try {
    const auto* pusch = typed_metadata<ocudu_dapp_pusch_metadata_v1>(in->pusch, OCUDU_DAPP_METADATA_PUSCH_V1);
    const auto* dmrs  = typed_metadata<ocudu_dapp_dmrs_metadata_v1>(in->dmrs, OCUDU_DAPP_METADATA_DMRS_V1);
    if (pusch == nullptr || dmrs == nullptr) {
      return OCUDU_DAPP_INVALID_INPUT_V1;
    }
    const unsigned P = pusch->nof_rx_ports, L = pusch->nof_layers, S = pusch->nof_symbols, N = pusch->nof_subcarriers;
    const int      ce = check_tensor(out->channel_estimates, OCUDU_DAPP_ELEMENT_CF32_V1, 8, {P, L, S, N},
                                     OCUDU_DAPP_ACCESS_WRITE_V1);
    const int nv = check_tensor(out->noise_variances, OCUDU_DAPP_ELEMENT_F32_V1, 4, {P, L}, OCUDU_DAPP_ACCESS_WRITE_V1);
    if (ce <= 0 || nv <= 0) {
      return ce == 0 || nv == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
    }
    const ocudu_dapp_status_v1 st = estimate(*w, in->rx_grid, *pusch, *dmrs, scs_khz_of(*pusch, in->invocation.radio_time.numerology));
    if (st != OCUDU_DAPP_OK_V1) {
      return st;
    }
    float* h = tensor_data<float>(out->channel_estimates);
    float* n = tensor_data<float>(out->noise_variances);
    for (unsigned p = 0; p != P; ++p) {
      for (unsigned l = 0; l != L; ++l) {
        n[p * L + l] = w->noise[p];
        for (unsigned s = 0; s != S; ++s) {
          const uint32_t* src = w->sym_est.data() + ((static_cast<size_t>(p) * kSymbols + pusch->start_symbol + s) * L + l) * N;
          float*          dst = h + 2 * (((static_cast<size_t>(p) * L + l) * S + s) * N);
          for (unsigned k = 0; k != N; ++k) {
            dst[2 * k]     = bf16_part(src[k], 0);
            dst[2 * k + 1] = bf16_part(src[k], 1);
          }
        }
      }
    }
    return OCUDU_DAPP_OK_V1;
  } catch (...) {
    return OCUDU_DAPP_EXCEPTION_V1;
  }
}

ocudu_dapp_status_v1 receiver_invoke(void* context, const ocudu_dapp_receiver_input_v1* in,
                                     ocudu_dapp_receiver_output_v1* out)
{
  auto* w = static_cast<worker_state*>(context);
  if (w == nullptr || in == nullptr || out == nullptr || in->invocation.worker_id != w->worker_id) {
    return OCUDU_DAPP_INVALID_INPUT_V1;
  }
  try {
    const auto* pusch = typed_metadata<ocudu_dapp_pusch_metadata_v1>(in->pusch, OCUDU_DAPP_METADATA_PUSCH_V1);
    const auto* dmrs  = typed_metadata<ocudu_dapp_dmrs_metadata_v1>(in->dmrs, OCUDU_DAPP_METADATA_DMRS_V1);
    if (pusch == nullptr || dmrs == nullptr) {
      return OCUDU_DAPP_INVALID_INPUT_V1;
    }
    const int Qm = static_cast<int>(pusch->modulation);
    if (Qm != 2 && Qm != 4 && Qm != 6 && Qm != 8) {
      return OCUDU_DAPP_BYPASS_V1;
    }
    const unsigned P = pusch->nof_rx_ports, L = pusch->nof_layers, S = pusch->nof_symbols, N = pusch->nof_subcarriers;
    const unsigned nre = pusch->nof_data_re;
    if (nre == 0 || nre > S * N) {
      return OCUDU_DAPP_INVALID_INPUT_V1;
    }
    // The data REs, flattened (symbol, subcarrier) indices relative to rx_grid, in LLR order.
    std::vector<uint32_t>& idx = w->idx;
    idx.resize(nre);
    if (pusch->data_re_indices.struct_size != 0) {
      const int t = check_tensor(pusch->data_re_indices, OCUDU_DAPP_ELEMENT_U32_V1, 4, {nre}, OCUDU_DAPP_ACCESS_READ_V1);
      if (t <= 0) {
        return t == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
      }
      std::memcpy(idx.data(), tensor_data<const uint32_t>(pusch->data_re_indices), nre * 4u);
    } else {
      const int t = check_tensor(pusch->data_re_mask, OCUDU_DAPP_ELEMENT_U8_V1, 1, {S, N}, OCUDU_DAPP_ACCESS_READ_V1);
      if (t <= 0) {
        return t == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
      }
      const uint8_t* m = tensor_data<const uint8_t>(pusch->data_re_mask);
      unsigned       k = 0;
      for (unsigned i = 0; i != S * N && k <= nre; ++i) {
        if (m[i] != 0) {
          if (k < nre) {
            idx[k] = i;
          }
          ++k;
        }
      }
      if (k != nre) {
        return OCUDU_DAPP_INVALID_INPUT_V1;
      }
    }
    for (uint32_t i : idx) {
      if (i >= S * N) {
        return OCUDU_DAPP_INVALID_INPUT_V1;
      }
    }
    const int lt = check_tensor(out->llrs, OCUDU_DAPP_ELEMENT_I8_V1, 1, {static_cast<uint64_t>(nre) * L * Qm},
                                OCUDU_DAPP_ACCESS_WRITE_V1);
    if (lt <= 0) {
      return lt == 0 ? OCUDU_DAPP_BYPASS_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
    }
    const ocudu_dapp_status_v1 st = estimate(*w, in->rx_grid, *pusch, *dmrs, scs_khz_of(*pusch, in->invocation.radio_time.numerology));
    if (st != OCUDU_DAPP_OK_V1) {
      return st;
    }
    // Equaliser inputs: received REs [port][re] and estimates [port][layer][re] (cbf16).
    w->y.resize(static_cast<size_t>(P) * nre);
    w->h.resize(static_cast<size_t>(P) * L * nre);
    for (unsigned p = 0; p != P; ++p) {
      for (unsigned i = 0; i != nre; ++i) {
        const unsigned s = idx[i] / N, k = idx[i] % N;
        w->y[static_cast<size_t>(p) * nre + i] =
            w->grid[(static_cast<size_t>(p) * kSymbols + pusch->start_symbol + s) * N + k];
        for (unsigned l = 0; l != L; ++l) {
          w->h[(static_cast<size_t>(p) * L + l) * nre + i] =
              w->sym_est[((static_cast<size_t>(p) * kSymbols + pusch->start_symbol + s) * L + l) * N + k];
        }
      }
    }
    w->eq.resize(static_cast<size_t>(nre) * L * 2);
    w->eq_var.resize(static_cast<size_t>(nre) * L);
    if (pg_equalize_host(w->ctx, PG_EQ_MMSE, static_cast<int>(nre), static_cast<int>(P), static_cast<int>(L),
                         w->y.data(), w->h.data(), w->noise, 1.0f, w->eq.data(), w->eq_var.data()) != PG_OK) {
      return OCUDU_DAPP_DEVICE_ERROR_V1;
    }
    int8_t* llr = tensor_data<int8_t>(out->llrs);
    if (pg_demodulate_soft_host(w->ctx, Qm, static_cast<int>(nre * L), w->eq.data(), w->eq_var.data(), llr) != PG_OK) {
      return OCUDU_DAPP_DEVICE_ERROR_V1;
    }
    // Optional metrics: post-equalisation noise and equalised symbols, [data_re, layer].
    out->reserved0 = 0;
    const auto* metrics = static_cast<const ocudu_dapp_receiver_metrics_v1*>(out->metrics.metadata.data);
    if (metrics != nullptr && out->metrics.metadata_schema_id == OCUDU_DAPP_METADATA_RECEIVER_METRICS_V1 &&
        out->metrics.metadata.size >= offsetof(ocudu_dapp_receiver_metrics_v1, reserved) &&
        metrics->struct_size >= offsetof(ocudu_dapp_receiver_metrics_v1, reserved)) {
      if (check_tensor(metrics->post_equalization_noise, OCUDU_DAPP_ELEMENT_F32_V1, 4, {nre, L},
                       OCUDU_DAPP_ACCESS_WRITE_V1) > 0) {
        std::memcpy(tensor_data<float>(metrics->post_equalization_noise), w->eq_var.data(), w->eq_var.size() * 4);
        out->reserved0 |= OCUDU_DAPP_RECEIVER_METRICS_VALID_V1;
      }
      if (out->metrics.metadata.size >= OCUDU_DAPP_RECEIVER_EQUALIZED_SYMBOLS_MIN_SIZE_V1 &&
          metrics->struct_size >= OCUDU_DAPP_RECEIVER_EQUALIZED_SYMBOLS_MIN_SIZE_V1 &&
          metrics->equalized_symbols.struct_size != 0 &&
          check_tensor(metrics->equalized_symbols, OCUDU_DAPP_ELEMENT_CF32_V1, 8, {nre, L},
                       OCUDU_DAPP_ACCESS_WRITE_V1) > 0) {
        std::memcpy(tensor_data<float>(metrics->equalized_symbols), w->eq.data(), w->eq.size() * 4);
        out->reserved0 |= OCUDU_DAPP_RECEIVER_EQUALIZED_SYMBOLS_VALID_V1;
      }
    }
    return OCUDU_DAPP_OK_V1;
  } catch (...) {
    return OCUDU_DAPP_EXCEPTION_V1;
  }
}

ocudu_dapp_status_v1 module_create(const ocudu_dapp_host_api_v1*, const void*, void** instance)
{
  if (instance == nullptr) {
    return OCUDU_DAPP_INVALID_INPUT_V1;
  }
  auto* s = new (std::nothrow) instance_state;
  if (s == nullptr) {
    return OCUDU_DAPP_RESOURCE_V1;
  }
  // The GPU of the module's workers: PG_DAPP_DEVICE (default 0).
  if (const char* d = std::getenv("PG_DAPP_DEVICE")) {
    s->device = std::atoi(d);
  }
  *instance = s;
  return OCUDU_DAPP_OK_V1;
}

ocudu_dapp_status_v1 module_noop(void* instance)
{
  return instance != nullptr ? OCUDU_DAPP_OK_V1 : OCUDU_DAPP_INVALID_INPUT_V1;
}
ocudu_dapp_status_v1 module_configure(void* instance, const void*)
{
  return module_noop(instance);
}
ocudu_dapp_status_v1 module_quiesce(void* instance, uint64_t)
{
  return module_noop(instance);
}
void module_destroy(void* instance)
{
  delete static_cast<instance_state*>(instance);
}

const ocudu_dapp_worker_api_v1 kWorkerApi = {sizeof(ocudu_dapp_worker_api_v1), OCUDU_DAPP_ABI_MAJOR_V1,
                                             OCUDU_DAPP_ABI_MINOR_V1, create_worker, destroy_worker, {}};
const ocudu_dapp_channel_estimator_interface_v1 kEstimator = {kWorkerApi, estimator_invoke, {}};
const ocudu_dapp_receiver_interface_v1          kReceiver  = {kWorkerApi, receiver_invoke, {}};

const ocudu_dapp_pusch_profile_v1 kProfile = {
    sizeof(ocudu_dapp_pusch_profile_v1),
    OCUDU_DAPP_ABI_MAJOR_V1,
    OCUDU_DAPP_ABI_MINOR_V1,
    OCUDU_DAPP_PUSCH_PROFILE_V1,
    kMaxPrb,
    kMaxPorts,
    kMaxLayers,
    OCUDU_DAPP_PUSCH_MODULATION_QPSK_V1 | OCUDU_DAPP_PUSCH_MODULATION_QAM16_V1 | OCUDU_DAPP_PUSCH_MODULATION_QAM64_V1 |
        OCUDU_DAPP_PUSCH_MODULATION_QAM256_V1,
    OCUDU_DAPP_PUSCH_DMRS_TYPE1_V1,
    0,
    0,
    {}};

const ocudu_dapp_interface_descriptor_v1 kInterfaces[2] = {
    {sizeof(ocudu_dapp_interface_descriptor_v1), OCUDU_DAPP_ABI_MAJOR_V1, OCUDU_DAPP_ABI_MINOR_V1,
     OCUDU_DAPP_INTERFACE_CHANNEL_ESTIMATOR_V1, 1, 0, OCUDU_DAPP_CLASS_A_INLINE_V1,
     1u << (OCUDU_DAPP_PLACEMENT_IN_PROCESS_V1 - 1), OCUDU_DAPP_THREADING_PER_WORKER_V1, 0, &kEstimator, 0, &kProfile,
     {}},
    {sizeof(ocudu_dapp_interface_descriptor_v1), OCUDU_DAPP_ABI_MAJOR_V1, OCUDU_DAPP_ABI_MINOR_V1,
     OCUDU_DAPP_INTERFACE_RECEIVER_V1, 1, 0, OCUDU_DAPP_CLASS_A_INLINE_V1,
     1u << (OCUDU_DAPP_PLACEMENT_IN_PROCESS_V1 - 1), OCUDU_DAPP_THREADING_PER_WORKER_V1, 0, &kReceiver, 0, &kProfile,
     {}}};

} // namespace

extern "C" OCUDU_DAPP_EXPORT_V1 ocudu_dapp_status_v1 ocudu_dapp_query_v1(const ocudu_dapp_host_info_v1*,
                                                                         ocudu_dapp_module_v1* module)
{
  if (module == nullptr) {
    return OCUDU_DAPP_INVALID_INPUT_V1;
  }
  *module                = ocudu_dapp_module_v1{};
  module->struct_size    = sizeof(ocudu_dapp_module_v1);
  module->abi_major      = OCUDU_DAPP_ABI_MAJOR_V1;
  module->abi_minor      = OCUDU_DAPP_ABI_MINOR_V1;
  module->global_name    = "pusch_b200.dapp";
  module->vendor         = "pusch_b200";
  module->version        = "1.0.0";
  module->nof_interfaces = 2;
  module->interfaces     = kInterfaces;
  module->create         = module_create;
  module->configure      = module_configure;
  module->prepare        = module_configure;
  module->warmup         = module_configure;
  module->start          = module_noop;
  module->stop           = module_noop;
  module->quiesce        = module_quiesce;
  module->destroy        = module_destroy;
  module->management     = nullptr;
  return OCUDU_DAPP_OK_V1;
}

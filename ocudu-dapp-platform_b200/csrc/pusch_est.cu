// DM-RS channel estimation for PUSCH on sm_100a, following the reference's
// port_channel_estimator_average_impl with FD smoothing "filter", TD "interpolate" and no CFO
// compensation (lib/phy/upper/signal_processors/channel_estimator/port_channel_estimator_average_impl.cpp:322-557,
// port_channel_estimator_helpers.cpp:29-300, lib/phy/support/interpolator/interpolator_linear_impl.cpp:15-123)
// and the pilot generation of dmrs_pusch_estimator_impl (dmrs_pusch_estimator_impl.cpp:69-169).
//
// One CTA per (UE, receive port). Per DM-RS symbol d and layer l (CDM group 0: layers 0 and 1):
//   LS          lse = rx * conj(pilot_l); with two layers, adjacent pilot pairs are averaged
//               (the frequency OCC [+1, -1] cancels the other layer); scaled by 1/beta;
//   smoothing   the pilots are extended at both ends by nv virtual pilots (linear fit of magnitude
//               and unwrapped phase of the nv outermost pilots) and convolved with the normalised
//               raised-cosine taps (roll-off 0.2) resampled at the pilot stride;
//   RSRP        sum |smoothed|^2 * beta^2;
//   frequency   linear interpolation from the even subcarriers to every subcarrier;
//   noise       sum over DM-RS symbols of |sum_l mean_d(smoothed) * beta * pilot_l - rx|^2.
// Per port: rsrp /= N, epre = sum |rx|^2 / N, noise /= (N * nof_cdm - 1) floored at rsrp / 1e10,
// snr = rsrp * layers / beta^2 / noise, with N = pilots per symbol x DM-RS symbols.
// Pilot bits come from the Gold sequence c(n) of TS 38.211 Section 5.2.1, evaluated as
// x1(n + Nc) xor (xor over the set bits i of c_init of the x2 sequence started from state e_i):
// c is linear in c_init, so 32 precomputed basis sequences give any sequence word by word.
#include "pg_internal.h"
#include "pg_device.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kEstThreads = 512;
constexpr int kMaxV       = 12;
constexpr int kMaxPil     = 6 * 275;
constexpr int kMaxDmrs    = 2;

__constant__ float c_rc_taps[3][16]; // normalised taps for 1, 2 and >= 3 PRBs (5, 11, 15 taps)

__device__ __forceinline__ float2 cbf16_load(const uint32_t* p)
{
  const uint32_t v = __ldg(p);
  return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xffff0000u));
}

__device__ __forceinline__ uint32_t float_to_bf16_rne(float f)
{
  uint32_t u = __float_as_uint(f);
  if ((u & 0x7fffffffu) > 0x7f800000u) {
    return (u >> 16) | 0x40u; // quiet NaN
  }
  return (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
}

} // namespace

namespace pg {

// Host: x1 from (1, 0, ..., 0) and x2 from each unit state e_i, positions Nc .. Nc + 32*words.
void gold_tables_host(std::vector<uint32_t>& tab, uint32_t words)
{
  tab.assign((size_t)32 * words, 0);
  const uint32_t nc = 1600;
  for (int seq = 0; seq < 32; ++seq) {
    // State holds x(n) .. x(n+30) in bits 0..30.
    uint32_t st = seq == 0 ? 1u : (1u << (seq - 1));
    uint32_t* out = tab.data() + (size_t)seq * words;
    for (uint32_t n = 0; n < nc + 32u * words; ++n) {
      const uint32_t bit = st & 1u;
      uint32_t       nb;
      if (seq == 0) {
        nb = ((st >> 3) ^ st) & 1u;
      } else {
        nb = ((st >> 3) ^ (st >> 2) ^ (st >> 1) ^ st) & 1u;
      }
      st = (st >> 1) | (nb << 30);
      if (n >= nc) {
        const uint32_t m = n - nc;
        out[m >> 5] |= bit << (m & 31);
      }
    }
  }
}

} // namespace pg

namespace {

// Dynamic shared memory of one CTA, sized for the largest allocation of the launch (npil_max
// pilots per DM-RS symbol): pilot bits per DM-RS symbol, then the LS estimates of each (DM-RS
// symbol, layer) extended by kMaxV virtual pilots at both ends, then the reduction scratch.
struct est_layout {
  uint32_t* bits; // [kMaxDmrs][bit_words]
  float2*   ext;  // [kMaxDmrs][2][npil_max + 2 kMaxV]
  float*    red;  // [3][kEstThreads / 32]
  int       bit_words, ext_stride;
};

__host__ __device__ inline size_t est_smem_bytes(int npil_max)
{
  const size_t bit_words  = (size_t)(2 * npil_max) / 32 + 2;
  const size_t ext_stride = (size_t)npil_max + 2 * kMaxV;
  return 16 + kMaxDmrs * bit_words * 4 + kMaxDmrs * 2 * ext_stride * 8 + 3 * (kEstThreads / 32) * 4;
}

__device__ inline est_layout est_carve(unsigned char* raw, int npil_max)
{
  est_layout l;
  l.bit_words  = (2 * npil_max) / 32 + 2;
  l.ext_stride = npil_max + 2 * kMaxV;
  l.bits       = reinterpret_cast<uint32_t*>(raw);
  size_t off   = (size_t)kMaxDmrs * l.bit_words * 4;
  off          = (off + 7) & ~(size_t)7;
  l.ext        = reinterpret_cast<float2*>(raw + off);
  off += (size_t)kMaxDmrs * 2 * l.ext_stride * 8;
  l.red = reinterpret_cast<float*>(raw + off);
  return l;
}

__device__ __forceinline__ float block_sum(float v, float* red, int slot_unused)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  (void)slot_unused;
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = v;
  }
  __syncthreads();
  float t = 0.f;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kEstThreads / 32; ++i) {
      t += red[i];
    }
  }
  __syncthreads();
  return t;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmulconjf(float2 a, float2 b) // a * conj(b)
{
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

__device__ void virtual_pilots(float2* out, const float2* base, int nv, bool is_start)
{
  // Linear fit of |h| and of the unwrapped arg(h) over nv pilots (port_channel_estimator_helpers.cpp
  // compute_v_pilots / add_v_pilots), evaluated at the nv positions before or after them.
  float arg_prev = 0.f, acc = 0.f;
  float mean_abs = 0.f, mean_arg = 0.f, sxa = 0.f, sxg = 0.f;
  float args[kMaxV], abss[kMaxV];
  for (int i = 0; i < nv; ++i) {
    const float a = hypotf(base[i].x, base[i].y);
    float       g = atan2f(base[i].y, base[i].x);
    if (i > 0) {
      // unwrap: keep consecutive differences within (-pi, pi].
      float d = g - arg_prev;
      if (d > 3.14159265358979f) {
        acc -= 6.28318530717959f;
      } else if (d < -3.14159265358979f) {
        acc += 6.28318530717959f;
      }
    }
    arg_prev = g;
    abss[i]  = a;
    args[i]  = g + acc;
  }
  for (int i = 0; i < nv; ++i) {
    mean_abs += abss[i];
    mean_arg += args[i];
    sxa += abss[i] * (float)i;
    sxg += args[i] * (float)i;
  }
  mean_abs /= (float)nv;
  mean_arg /= (float)nv;
  const float mean_x = (float)(nv * (nv - 1)) / 2.0f / (float)nv;
  const float nxsq   = (float)((nv - 1) * nv * (2 * nv - 1)) / 6.0f;
  const float den    = nxsq - (float)nv * mean_x * mean_x;
  const float sa     = (sxa - mean_x * mean_abs * (float)nv) / den;
  const float ia     = mean_abs - sa * mean_x;
  const float sg     = (sxg - mean_x * mean_arg * (float)nv) / den;
  const float ig     = mean_arg - sg * mean_x;
  const int   voff   = is_start ? -nv : nv;
  for (int i = 0; i < nv; ++i) {
    const float iv  = (float)(i + voff);
    const float rho = sa * iv + ia;
    float       s, c;
    sincosf(sg * iv + ig + (rho > 0.f ? 0.f : 3.14159265358979f), &s, &c);
    out[i] = make_float2(fabsf(rho) * c, fabsf(rho) * s);
  }
}

__global__ void __launch_bounds__(kEstThreads) pusch_estimate_kernel(const pg_pusch_ue* __restrict__ ues,
                                                                     const uint32_t* __restrict__ grids,
                                                                     float2* __restrict__ est_all,
                                                                     float2* __restrict__ ls_all,
                                                                     pg_port_result* __restrict__ results,
                                                                     const uint32_t* __restrict__ gold,
                                                                     uint32_t gold_words, int npil_max,
                                                                     const float2* __restrict__ pilots,
                                                                     float2* __restrict__ cfo_acc)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const est_layout  sm   = est_carve(smem_raw, npil_max);
  const int         u    = blockIdx.x;
  const int         port = blockIdx.y;
  const pg_pusch_ue ue   = ues[u];
  if (port >= ue.nof_rx_ports) {
    return;
  }
  const int tid  = threadIdx.x;
  const int nl   = ue.nof_layers;
  const int nrb  = ue.nof_rb;
  const int npil = 6 * nrb;
  const int nsc  = 12 * nrb;
  if (npil > npil_max) {
    return; // not reached: the host sizes the shared memory for the largest allocation
  }
  int dsym[kMaxDmrs];
  int nd = 0;
  for (int s = ue.first_symbol; s < ue.first_symbol + ue.nof_symbols && nd < kMaxDmrs; ++s) {
    if ((ue.dmrs_symbol_mask >> s) & 1) {
      dsym[nd++] = s;
    }
  }
  const float     beta = ue.dmrs_scaling;
  const uint32_t* grid = grids + ue.grid_offset + (size_t)port * 14 * ue.grid_nof_subc;
  auto ext = [&](int d, int l) { return sm.ext + ((size_t)d * 2 + l) * sm.ext_stride; };
  auto bit = [&](int d, int i) { return (sm.bits[d * sm.bit_words + (i >> 5)] >> (i & 31)) & 1u; };
  auto rxp = [&](int d, int k) {
    return cbf16_load(grid + (size_t)dsym[d] * ue.grid_nof_subc + 12 * ue.rb_start + 2 * k);
  };
  // Pilot of layer l at DM-RS symbol d, pilot k: given by the caller ([d][l][k], dmrs_pusch_estimator's
  // sequences) or generated here (QPSK of the Gold sequence, the frequency OCC on layer 1).
  const float a = 0.707106781186547524f; // 1/sqrt(2) (M_SQRT1_2 in float)
  auto pilot = [&](int d, int l, int k) {
    if (pilots != nullptr) {
      return pilots[((size_t)d * nl + l) * npil + k];
    }
    const float2 p0 = make_float2(bit(d, 2 * k) ? -a : a, bit(d, 2 * k + 1) ? -a : a);
    return (l == 1 && (k & 1)) ? make_float2(-p0.x, -p0.y) : p0;
  };

  // Pilot bits c(2 m0) .. c(2 m0 + 2 npil - 1) per DM-RS symbol, m0 = 6 rb_start.
  const int nwords = (2 * npil + 31) / 32;
  for (int i = tid; i < nd * nwords; i += kEstThreads) {
    const int      d      = i / nwords;
    const int      w      = i - d * nwords;
    const uint32_t c_init = (uint32_t)(((14ull * ue.slot + dsym[d] + 1) * (2ull * ue.n_id + 1) * (1ull << 17) +
                                        (2ull * ue.n_id + ue.n_scid)) %
                                       (1ull << 31));
    sm.bits[d * sm.bit_words + w] = pg::gold_word(gold, gold_words, c_init, 12u * ue.rb_start + 32u * w);
  }
  __syncthreads();

  // LS estimates.
  const float inv_beta = 1.0f / beta;
  float       epre     = 0.f;
  for (int i = tid; i < nd * npil; i += kEstThreads) {
    const int    d  = i / npil;
    const int    k  = i - d * npil;
    const float2 y  = rxp(d, k);
    epre += y.x * y.x + y.y * y.y;
    ext(d, 0)[kMaxV + k] = cmulconjf(y, pilot(d, 0, k));
    if (nl > 1) {
      ext(d, 1)[kMaxV + k] = cmulconjf(y, pilot(d, 1, k));
    }
  }
  __syncthreads();
  if (cfo_acc != nullptr && nd == 2) {
    // CFO observation: the sum over layers and pilots of LS(second DM-RS symbol) x conj(LS(first)),
    // before any averaging (port_channel_estimator_average_impl.cpp:593-615).
    float cr = 0.f, ci = 0.f;
    for (int i = tid; i < nl * npil; i += kEstThreads) {
      const int    l  = i / npil;
      const int    k  = i - l * npil;
      const float2 q  = cmulconjf(ext(1, l)[kMaxV + k], ext(0, l)[kMaxV + k]);
      cr += q.x;
      ci += q.y;
    }
    const float tr = block_sum(cr, sm.red, 0);
    const float ti = block_sum(ci, sm.red, 0);
    if (tid == 0) {
      cfo_acc[(size_t)u * 4 + port] = make_float2(tr, ti);
    }
  }
  for (int i = tid; i < nd * nl * (npil / 2); i += kEstThreads) {
    const int d  = i / (nl * (npil / 2));
    const int r  = i - d * nl * (npil / 2);
    const int l  = r / (npil / 2);
    const int k  = 2 * (r - l * (npil / 2));
    float2*   e  = ext(d, l);
    float2    v0 = e[kMaxV + k], v1 = e[kMaxV + k + 1];
    if (nl > 1) {
      const float2 av = make_float2((v0.x + v1.x) / 2.0f, (v0.y + v1.y) / 2.0f);
      v0 = v1 = av;
    }
    e[kMaxV + k]     = make_float2(v0.x * inv_beta, v0.y * inv_beta);
    e[kMaxV + k + 1] = make_float2(v1.x * inv_beta, v1.y * inv_beta);
  }
  __syncthreads();
  if (ls_all != nullptr) {
    // The LS estimates themselves (input of the learned estimator): the pilots' subcarriers
    // (even) of the frequency-response layout, zero on the odd ones.
    float2* ls = ls_all + ue.est_offset + (size_t)port * nd * nl * nsc;
    for (int i = tid; i < nd * nl * nsc; i += kEstThreads) {
      const int d = i / (nl * nsc);
      const int r = i - d * nl * nsc;
      const int l = r / nsc;
      const int j = r - l * nsc;
      ls[i]       = (j & 1) ? make_float2(0.f, 0.f) : ext(d, l)[kMaxV + (j >> 1)];
    }
  }

  // Smoothing filter and virtual pilots.
  const int tsel  = nrb >= 3 ? 2 : nrb - 1;
  const int ntaps = tsel == 2 ? 15 : (tsel == 1 ? 11 : 5);
  const int mid   = ntaps / 2;
  const int nv    = nrb == 1 ? npil : mid;
  if (tid < nd * nl * 2) {
    const int d = tid / (nl * 2), l = (tid / 2) % nl, side = tid & 1;
    float2*   e = ext(d, l);
    if (side == 0) {
      virtual_pilots(e + kMaxV - nv, e + kMaxV, nv, true);
    } else {
      virtual_pilots(e + kMaxV + npil, e + kMaxV + npil - nv, nv, false);
    }
  }
  __syncthreads();
  // The smoothed pilots go straight to the even subcarriers of the output; the odd ones are filled
  // below from their even neighbours, which this CTA reads back after a barrier.
  float2* est          = est_all + ue.est_offset + (size_t)port * nd * nl * nsc;
  float   rsrp_part[2] = {0.f, 0.f};
  for (int i = tid; i < nd * nl * npil; i += kEstThreads) {
    const int     d   = i / (nl * npil);
    const int     r   = i - d * nl * npil;
    const int     l   = r / npil;
    const int     k   = r - l * npil;
    const float2* e   = ext(d, l);
    float2        acc = make_float2(0.f, 0.f);
    for (int t = 0; t < ntaps; ++t) {
      const float2 x = e[kMaxV + k - mid + t];
      acc.x += x.x * c_rc_taps[tsel][t];
      acc.y += x.y * c_rc_taps[tsel][t];
    }
    est[((size_t)d * nl + l) * nsc + 2 * k] = acc;
    rsrp_part[l] += acc.x * acc.x + acc.y * acc.y;
  }
  __syncthreads();

  // Frequency interpolation to the odd subcarriers and noise estimation.
  for (int i = tid; i < nd * nl * npil; i += kEstThreads) {
    const int d   = i / (nl * npil);
    const int r   = i - d * nl * npil;
    const int l   = r / npil;
    const int k   = r - l * npil;
    float2*   row = est + ((size_t)d * nl + l) * nsc;
    float2    v   = row[2 * k];
    if (k + 1 < npil) {
      const float2 n = row[2 * k + 2];
      v              = make_float2((n.x - v.x) * 0.5f + v.x, (n.y - v.y) * 0.5f + v.y);
    }
    row[2 * k + 1] = v;
  }
  float       noise = 0.f;
  const float sf    = beta / (float)nd;
  for (int i = tid; i < nd * npil; i += kEstThreads) {
    const int    d    = i / npil;
    const int    k    = i - d * npil;
    float2       pred = make_float2(0.f, 0.f);
    for (int l = 0; l < nl; ++l) {
      float2 sacc = make_float2(0.f, 0.f);
      for (int dd = 0; dd < nd; ++dd) {
        const float2 f = est[((size_t)dd * nl + l) * nsc + 2 * k];
        sacc.x += f.x * sf;
        sacc.y += f.y * sf;
      }
      const float2 q = cmulf(sacc, pilot(d, l, k));
      pred.x += q.x;
      pred.y += q.y;
    }
    const float2 y = rxp(d, k);
    const float2 e = make_float2(pred.x - y.x, pred.y - y.y);
    noise += e.x * e.x + e.y * e.y;
  }
  float*      red       = sm.red;
  const float tot_noise = block_sum(noise, red, 0);
  const float tot_epre  = block_sum(epre, red + (kEstThreads / 32), 1);
  const float tot_r0    = block_sum(rsrp_part[0], red + 2 * (kEstThreads / 32), 2);
  const float tot_r1    = block_sum(rsrp_part[1], red, 0);
  if (tid == 0) {
    const float    n_pil = (float)(npil * nd);
    pg_port_result pr;
    pr.rsrp[0]       = tot_r0 * beta * beta / n_pil;
    pr.rsrp[1]       = nl > 1 ? tot_r1 * beta * beta / n_pil : 0.f;
    pr.epre          = tot_epre / n_pil;
    const float ravg = nl > 1 ? (pr.rsrp[0] + pr.rsrp[1]) / 2.f : pr.rsrp[0];
    float       nvar = (pg::is_normal(tot_noise) ? tot_noise : 0.f) / (n_pil * (float)((nl + 1) / 2) - 1.f);
    nvar             = fmaxf(ravg / 1e10f, nvar);
    pr.noise_var     = nvar;
    pr.snr           = pg::is_normal(nvar) ? (ravg * (float)nl / beta / beta) / nvar : 0.f;
    results[(size_t)u * 4 + port] = pr;
  }
}

// Chunked form of pusch_estimate_kernel for batches: one CTA per (UE, receive port, chunk of
// kChunk pilots), so that a slot of many allocations runs as one short wave of small CTAs instead
// of one long CTA per (UE, port). Each CTA computes the LS estimates of its chunk plus a halo of
// kHalo pilots either side (the smoothing filter's reach), the virtual pilots where the filter
// reaches past either end of the allocation, the smoothed estimates of its own pilots and of the
// next one (for the frequency interpolation of its last odd subcarrier), and its partial sums of
// RSRP, EPRE and noise. Per element the arithmetic and its order are those of
// pusch_estimate_kernel, so the frequency responses are identical. The last CTA of each (UE, port)
// to finish (a per-port arrival counter, reset by that CTA for the next launch) adds the port's
// partial sums in chunk order (deterministic) and forms the scalars.
// c_init of the DM-RS sequence of OFDM symbol `sym` (TS 38.211 Section 6.4.1.1.1.1).
__device__ __host__ __forceinline__ uint32_t dmrs_c_init(const pg_pusch_ue& ue, int sym)
{
  return (uint32_t)(((14ull * ue.slot + sym + 1) * (2ull * ue.n_id + 1) * (1ull << 17) + (2ull * ue.n_id + ue.n_scid)) %
                    (1ull << 31));
}

// Words per DM-RS symbol of a UE's precomputed pilot bits: the allocation's 12 nof_rb sequence bits
// plus two words, so that a 32-bit window at any bit offset below 12 nof_rb reads in bounds.
__device__ __host__ __forceinline__ int dmrs_bit_words(int nof_rb)
{
  return (12 * nof_rb + 31) / 32 + 2;
}

constexpr int kChunk        = 128;
constexpr int kHalo         = 8;  // even, >= the largest filter half-length (7)
constexpr int kTileOff      = 16; // tile position of pilot k is k - (k0 - kTileOff)
constexpr int kChunkTile    = kChunk + 2 * kTileOff;
constexpr int kChunkThreads = 128;

__global__ void __launch_bounds__(kChunkThreads) pusch_estimate_chunk_kernel(const pg_pusch_ue* __restrict__ ues,
                                                                             const uint32_t* __restrict__ work,
                                                                             const uint32_t* __restrict__ grids,
                                                                             float2* __restrict__ est_all,
                                                                             float2* __restrict__ ls_all,
                                                                             float4* __restrict__ partials,
                                                                             const uint32_t* __restrict__ gold,
                                                                             uint32_t gold_words,
                                                                             int* __restrict__ arrivals,
                                                                             pg_port_result* __restrict__ results,
                                                                             const uint32_t* __restrict__ pilot_bits,
                                                                             int nof_ues)
{
  __shared__ uint32_t s_bits[kMaxDmrs][(2 * kChunkTile) / 32 + 2];
  __shared__ float2   s_y[kMaxDmrs][kChunk]; // the received pilots of the chunk (LS, then noise)
  __shared__ float2   s_ls[kMaxDmrs][2][kChunkTile];
  __shared__ float2   s_sm[kMaxDmrs][2][kChunk + 1];
  __shared__ float    s_red[kChunkThreads / 32][4];

  const uint32_t    wi   = work[blockIdx.x];
  const int         u    = (int)(wi & 0xffffu);
  const int         port = (int)((wi >> 16) & 0xfu);
  const int         ch   = (int)(wi >> 20);
  const pg_pusch_ue ue   = ues[u];
  const int         tid  = threadIdx.x;
  const int         nl   = ue.nof_layers;
  const int         nrb  = ue.nof_rb;
  const int         npil = 6 * nrb;
  const int         nsc  = 12 * nrb;
  const int         k0   = ch * kChunk;
  const int         k1   = min(npil, k0 + kChunk);
  const int         t0   = k0 - kTileOff;
  const int         pb   = max(0, k0 - kHalo);   // first LS pilot of the tile (even)
  const int         pe   = min(npil, k1 + kHalo); // one past the last (even)
  int dsym[kMaxDmrs];
  int nd = 0;
  for (int s = ue.first_symbol; s < ue.first_symbol + ue.nof_symbols && nd < kMaxDmrs; ++s) {
    if ((ue.dmrs_symbol_mask >> s) & 1) {
      dsym[nd++] = s;
    }
  }
  const float     beta = ue.dmrs_scaling;
  const uint32_t* grid = grids + ue.grid_offset + (size_t)port * 14 * ue.grid_nof_subc;
  auto rxp = [&](int d, int k) {
    return cbf16_load(grid + (size_t)dsym[d] * ue.grid_nof_subc + 12 * ue.rb_start + 2 * k);
  };
  const float a = 0.707106781186547524f;
  auto bit = [&](int d, int i) { // pilot bit i of the allocation, i >= 2 pb
    const int j = i - 2 * pb;
    return (s_bits[d][j >> 5] >> (j & 31)) & 1u;
  };
  auto pilot = [&](int d, int l, int k) {
    const float2 p0 = make_float2(bit(d, 2 * k) ? -a : a, bit(d, 2 * k + 1) ? -a : a);
    return (l == 1 && (k & 1)) ? make_float2(-p0.x, -p0.y) : p0;
  };

  // Pilot bits c(2 (m0 + pb)) .. of the tile, m0 = 6 rb_start: from the UE's precomputed pilot
  // bits (dmrs_bits_launch; bit b of symbol d's row = c(12 rb_start + b)) or from the Gold basis.
  const int nwords = (2 * (pe - pb) + 31) / 32;
  if (pilot_bits != nullptr) {
    const uint32_t* pbits = pilot_bits + work[gridDim.x + 4 * nof_ues + 1 + u];
    const int       W     = dmrs_bit_words(nrb);
    const int       w0    = (2 * pb) >> 5;
    const int       sh    = (2 * pb) & 31;
    for (int i = tid; i < nd * nwords; i += kChunkThreads) {
      const int      d  = i / nwords;
      const int      w  = i - d * nwords;
      const uint32_t lo = __ldg(pbits + d * W + w0 + w), hi = __ldg(pbits + d * W + w0 + w + 1);
      s_bits[d][w]      = sh ? __funnelshift_r(lo, hi, sh) : lo;
    }
  } else {
    for (int i = tid; i < nd * nwords; i += kChunkThreads) {
      const int      d      = i / nwords;
      const int      w      = i - d * nwords;
      s_bits[d][w] = pg::gold_word(gold, gold_words, dmrs_c_init(ue, dsym[d]), 12u * ue.rb_start + 2u * pb + 32u * w);
    }
  }
  __syncthreads();

  // LS estimates of the tile, a pilot pair (k, k + 1) per thread step: averaged over the pair with
  // two layers (the frequency OCC), scaled by 1/beta.
  const float inv_beta = 1.0f / beta;
  float       epre     = 0.f;
  const int   npairs   = (pe - pb) / 2;
  for (int i = tid; i < nd * npairs; i += kChunkThreads) {
    const int    d  = i / npairs;
    const int    k  = pb + 2 * (i - d * npairs);
    const float2 y0 = rxp(d, k), y1 = rxp(d, k + 1);
    if (k >= k0 && k < k1) {
      epre += y0.x * y0.x + y0.y * y0.y;
      epre += y1.x * y1.x + y1.y * y1.y;
      s_y[d][k - k0]     = y0;
      s_y[d][k + 1 - k0] = y1;
    }
    for (int l = 0; l < nl; ++l) {
      float2 v0 = cmulconjf(y0, pilot(d, l, k)), v1 = cmulconjf(y1, pilot(d, l, k + 1));
      if (nl > 1) {
        const float2 av = make_float2((v0.x + v1.x) / 2.0f, (v0.y + v1.y) / 2.0f);
        v0 = v1 = av;
      }
      v0                       = make_float2(v0.x * inv_beta, v0.y * inv_beta);
      v1                       = make_float2(v1.x * inv_beta, v1.y * inv_beta);
      s_ls[d][l][k - t0]       = v0;
      s_ls[d][l][k + 1 - t0]   = v1;
      if (ls_all != nullptr && k >= k0 && k < k1) {
        float2* ls = ls_all + ue.est_offset + (size_t)port * nd * nl * nsc + ((size_t)d * nl + l) * nsc;
        ls[2 * k]     = v0;
        ls[2 * k + 1] = make_float2(0.f, 0.f);
        ls[2 * k + 2] = v1;
        ls[2 * k + 3] = make_float2(0.f, 0.f);
      }
    }
  }
  __syncthreads();

  // Virtual pilots where the filter reaches past the allocation's ends.
  const int tsel  = nrb >= 3 ? 2 : nrb - 1;
  const int ntaps = tsel == 2 ? 15 : (tsel == 1 ? 11 : 5);
  const int mid   = ntaps / 2;
  const int nv    = nrb == 1 ? npil : mid;
  const int ks    = min(k1 + 1, npil); // smoothed pilots k0 .. ks - 1
  if (tid < nd * nl * 2) {
    const int d = tid / (nl * 2), l = (tid / 2) % nl, side = tid & 1;
    float2*   e = s_ls[d][l];
    if (side == 0 && k0 == 0) {
      virtual_pilots(e - nv - t0, e - t0, nv, true);
    } else if (side == 1 && ks - 1 + mid >= npil) {
      virtual_pilots(e + npil - t0, e + npil - nv - t0, nv, false);
    }
  }
  __syncthreads();

  // Smoothing: pilots k0 .. ks - 1; the chunk's own ones go to the even subcarriers of the output.
  float2* est          = est_all + ue.est_offset + (size_t)port * nd * nl * nsc;
  float   rsrp_part[2] = {0.f, 0.f};
  const int nsm        = ks - k0;
  for (int i = tid; i < nd * nl * nsm; i += kChunkThreads) {
    const int     d   = i / (nl * nsm);
    const int     r   = i - d * nl * nsm;
    const int     l   = r / nsm;
    const int     k   = k0 + r - l * nsm;
    const float2* e   = s_ls[d][l];
    float2        acc = make_float2(0.f, 0.f);
    for (int t = 0; t < ntaps; ++t) {
      const float2 x = e[k - mid + t - t0];
      acc.x += x.x * c_rc_taps[tsel][t];
      acc.y += x.y * c_rc_taps[tsel][t];
    }
    s_sm[d][l][k - k0] = acc;
    if (k < k1) {
      est[((size_t)d * nl + l) * nsc + 2 * k] = acc;
      rsrp_part[l] += acc.x * acc.x + acc.y * acc.y;
    }
  }
  __syncthreads();

  // Frequency interpolation to the odd subcarriers and noise, own pilots.
  for (int i = tid; i < nd * nl * (k1 - k0); i += kChunkThreads) {
    const int d = i / (nl * (k1 - k0));
    const int r = i - d * nl * (k1 - k0);
    const int l = r / (k1 - k0);
    const int k = k0 + r - l * (k1 - k0);
    float2    v = s_sm[d][l][k - k0];
    if (k + 1 < npil) {
      const float2 n = s_sm[d][l][k + 1 - k0];
      v              = make_float2((n.x - v.x) * 0.5f + v.x, (n.y - v.y) * 0.5f + v.y);
    }
    est[((size_t)d * nl + l) * nsc + 2 * k + 1] = v;
  }
  float       noise = 0.f;
  const float sf    = beta / (float)nd;
  for (int i = tid; i < nd * (k1 - k0); i += kChunkThreads) {
    const int d    = i / (k1 - k0);
    const int k    = k0 + i - d * (k1 - k0);
    float2    pred = make_float2(0.f, 0.f);
    for (int l = 0; l < nl; ++l) {
      float2 sacc = make_float2(0.f, 0.f);
      for (int dd = 0; dd < nd; ++dd) {
        const float2 f = s_sm[dd][l][k - k0];
        sacc.x += f.x * sf;
        sacc.y += f.y * sf;
      }
      const float2 q = cmulf(sacc, pilot(d, l, k));
      pred.x += q.x;
      pred.y += q.y;
    }
    const float2 y = s_y[d][k - k0];
    const float2 e = make_float2(pred.x - y.x, pred.y - y.y);
    noise += e.x * e.x + e.y * e.y;
  }
  float v4[4] = {rsrp_part[0], rsrp_part[1], epre, noise};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v4[q] += __shfl_xor_sync(0xffffffffu, v4[q], o);
    }
  }
  if ((tid & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      s_red[tid >> 5][q] = v4[q];
    }
  }
  __syncthreads();
  __shared__ int s_last;
  const int       pi    = 4 * u + port;
  const uint32_t* first = work + gridDim.x; // the work list (one item per CTA), then each port's first item
  if (tid == 0) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int w = 0; w < kChunkThreads / 32; ++w) {
      t.x += s_red[w][0];
      t.y += s_red[w][1];
      t.z += s_red[w][2];
      t.w += s_red[w][3];
    }
    partials[blockIdx.x] = t;
    __threadfence();
    const int nch = (int)(first[pi + 1] - first[pi]);
    s_last        = atomicAdd(&arrivals[pi], 1) == nch - 1;
  }
  __syncthreads();
  if (s_last && tid < 32) {
    // Last chunk of this port: every other chunk's partials are visible (fence before arrival).
    // The first warp loads them at once (lane i takes chunks i, i + 32, ...) and adds them in a
    // fixed tree, so the port's scalars do not depend on which chunk arrived last.
    __threadfence();
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t w = first[pi] + tid; w < first[pi + 1]; w += 32) {
      const float4 p = __ldcg(partials + w);
      s.x += p.x;
      s.y += p.y;
      s.z += p.z;
      s.w += p.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      s.z += __shfl_xor_sync(0xffffffffu, s.z, o);
      s.w += __shfl_xor_sync(0xffffffffu, s.w, o);
    }
    if (tid == 0) {
      arrivals[pi]      = 0;
      const float n_pil = (float)(npil * nd);
      pg_port_result pr;
      pr.rsrp[0]       = s.x * beta * beta / n_pil;
      pr.rsrp[1]       = nl > 1 ? s.y * beta * beta / n_pil : 0.f;
      pr.epre          = s.z / n_pil;
      const float ravg = nl > 1 ? (pr.rsrp[0] + pr.rsrp[1]) / 2.f : pr.rsrp[0];
      float       nvar = (pg::is_normal(s.w) ? s.w : 0.f) / (n_pil * (float)((nl + 1) / 2) - 1.f);
      nvar             = fmaxf(ravg / 1e10f, nvar);
      pr.noise_var     = nvar;
      pr.snr           = pg::is_normal(nvar) ? (ravg * (float)nl / beta / beta) / nvar : 0.f;
      results[pi]      = pr;
    }
  }
}

// Pilot bits of every UE of a plan, computed once: row d (DM-RS symbol d of the allocation) word w =
// c(12 rb_start + 32 w) .. c(12 rb_start + 32 w + 31), rows of dmrs_bit_words(nof_rb) words from
// off[u].
__global__ void dmrs_bits_kernel(const pg_pusch_ue* __restrict__ ues, const uint32_t* __restrict__ off,
                                 uint32_t* __restrict__ bits, const uint32_t* __restrict__ gold, uint32_t gold_words)
{
  const pg_pusch_ue ue = ues[blockIdx.y];
  const int         W  = dmrs_bit_words(ue.nof_rb);
  int               d  = 0;
  for (int s = ue.first_symbol; s < ue.first_symbol + ue.nof_symbols && d < kMaxDmrs; ++s) {
    if ((ue.dmrs_symbol_mask >> s) & 1) {
      const uint32_t c_init = dmrs_c_init(ue, s);
      for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        bits[off[blockIdx.y] + d * W + w] = pg::gold_word(gold, gold_words, c_init, 12u * ue.rb_start + 32u * w);
      }
      ++d;
    }
  }
}

// Per-symbol estimates of one UE: f[i] + (f[i+1] - f[i]) w rounded to bf16 (the reference's
// apply_td_domain_strategy + conversion to cbf16_t); with the learned estimator's time-basis
// coefficients (basis, two DM-RS symbols) + a_1 w (1 - w) + a_2 w (1 - w) (2 w - 1) before the
// rounding, in the demodulator's operation order.
__global__ void symbol_estimates_kernel(pg_pusch_ue ue, const float2* __restrict__ est,
                                        const float2* __restrict__ basis, uint32_t* __restrict__ out, int nd,
                                        int dsym0, int dsym1)
{
  const int nsc = 12 * ue.nof_rb;
  const int nl  = ue.nof_layers;
  const int s   = blockIdx.y;
  const int p   = blockIdx.z;
  int       i0  = 0;
  float     w   = 0.f;
  if (nd == 2) {
    w = (float)(s - dsym0) / (float)(dsym1 - dsym0);
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nl * nsc; t += gridDim.x * blockDim.x) {
    const int     l  = t / nsc;
    const int     j  = t - l * nsc;
    const float2* f0 = est + (((size_t)p * nd + i0) * nl + l) * nsc;
    float2        v  = f0[j];
    if (nd == 2) {
      const float2 v1 = f0[(size_t)nl * nsc + j];
      v               = make_float2(__fmaf_rn(v1.x - v.x, w, v.x), __fmaf_rn(v1.y - v.y, w, v.y));
      if (basis != nullptr) {
        const int L = nl;
          // The learned estimator's time-basis terms a_1 w (1 - w) + a_2 w (1 - w) (2 w - 1).
          const float2* b0 = basis + (((size_t)p * nd) * L + l) * nsc;
          const float2  a1 = b0[j], a2 = b0[(size_t)L * nsc + j];
          const float   f1 = __fmul_rn(w, __fsub_rn(1.f, w));
          const float   f2 = __fmul_rn(f1, __fsub_rn(__fmul_rn(2.f, w), 1.f));
          v                = make_float2(__fmaf_rn(a2.x, f2, __fmaf_rn(a1.x, f1, v.x)),
                                         __fmaf_rn(a2.y, f2, __fmaf_rn(a1.y, f1, v.y)));
      }
    }
    out[(((size_t)p * 14 + s) * nl + l) * nsc + j] = float_to_bf16_rne(v.x) | (float_to_bf16_rne(v.y) << 16);
  }
}

// ---------------------------------------------------------------------------------------------
// Time alignment of one receive port (time_alignment_estimator_dft_impl.cpp:97-233, called by
// port_channel_estimator_helpers.cpp:235-272 with the smoothed pilots and stride 2).
constexpr int kTaMaxDft = 4096; // pow2(log2_ceil(MAX_NOF_SUBCARRIERS = 3300))

// Power of the inverse DFT of every (DM-RS symbol, layer) sequence of smoothed pilots, summed over
// the sequences: corr[n] = sum_q |sum_k x_q[k] e^{+j 2 pi k n / N}|^2 (the pilots zero-padded to
// N, a power of two). x_q[k] = est[q][2 k], the filter output at pilot k.
__global__ void ta_correlation_kernel(const float2* __restrict__ est, int nseq, int nsc, int npil, int N,
                                      float* __restrict__ corr)
{
  __shared__ float2 tw[kTaMaxDft];
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    float sn, cs;
    sincospif(2.0f * (float)m / (float)N, &sn, &cs);
    tw[m] = make_float2(cs, sn);
  }
  __syncthreads();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) {
    return;
  }
  float power = 0.f;
  for (int q = 0; q < nseq; ++q) {
    const float2* x   = est + (size_t)q * nsc;
    float         re  = 0.f, im = 0.f;
    unsigned      idx = 0; // k n mod N
    for (int k = 0; k < npil; ++k) {
      const float2 v = __ldg(x + 2 * k);
      const float2 w = tw[idx];
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
      idx = (idx + (unsigned)n) & (unsigned)(N - 1);
    }
    power += re * re + im * im;
  }
  corr[n] = power;
}

struct ta_cfo_out {
  double time_alignment_s;
  float  cfo_hz;
  float  pad;
};

// Peak of the correlation among the max_ta delayed and the max_ta advanced samples, refined by the
// reference's five- (three-) point curve fit (lib/support/math/curve_fitting_find_max.cpp) unless N
// is the largest DFT size; and the CFO from the phase of the DM-RS-symbol correlation:
// arg / (2 pi (epoch_1 - epoch_0)) * scs (port_channel_estimator_average_impl.cpp:612-615, :53).
__global__ void ta_cfo_kernel(const float* __restrict__ corr, int N, int max_ta, double fs,
                              const float2* __restrict__ cfo_acc, float epoch_diff, float scs_hz,
                              ta_cfo_out* __restrict__ out)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  int   di = 0, ai = 0;
  float dv = 0.f, av = 0.f;
  for (int i = 0; i < max_ta; ++i) {
    const float v = corr[i];
    if (i == 0 || v > dv) {
      dv = v;
      di = i;
    }
    const float w = corr[N - max_ta + i];
    if (i == 0 || w > av) {
      av = w;
      ai = i;
    }
  }
  int idx = -(max_ta - ai);
  if (dv >= av) {
    idx = di;
  }
  float frac = 0.f;
  if (N != kTaMaxDft) {
    const float nw5[5] = {-0.400000f, -0.200000f, 0.000000f, 0.200000f, 0.400000f};
    const float dw5[5] = {0.571429f, -0.285714f, -0.571429f, -0.285714f, 0.571429f};
    const float nw3[3] = {-0.5f, 0.0f, 0.5f};
    const float dw3[3] = {0.5f, -1.0f, 0.5f};
    const int   taps   = max_ta > 2 ? 5 : 3;
    float       num = 0.f, den = 0.f;
    for (int i = 0; i < taps; ++i) {
      const float smp = corr[(unsigned)(idx + i + N - taps / 2) & (unsigned)(N - 1)];
      num             = __fadd_rn(num, __fmul_rn(taps == 5 ? nw5[i] : nw3[i], smp));
      den             = __fadd_rn(den, __fmul_rn(taps == 5 ? dw5[i] : dw3[i], smp));
    }
    const float r = -(taps == 5 ? 1.0f : 0.5f) * num / den;
    frac          = (isnan(r) || isinf(r) || fabsf(r) > 1.0f) ? 0.f : r;
  }
  out->time_alignment_s = ((double)idx + (double)frac) / fs;
  if (cfo_acc != nullptr) {
    const float2 c = cfo_acc[0];
    out->cfo_hz    = atan2f(c.y, c.x) / 6.28318530717959f / epoch_diff * scs_hz;
  } else {
    out->cfo_hz = __int_as_float(0x7fc00000); // NaN: one DM-RS symbol, no CFO observation
  }
}

} // namespace

namespace pg {

int est_upload_tables(pg_context* ctx)
{
  // Raised-cosine impulse, roll-off 0.2, 10 samples per symbol, 31 samples centred at 15; the
  // taps of n PRBs (n = 1, 2, >= 3) are every second sample around the centre, normalised.
  double rc[31];
  for (int n = 0; n < 31; ++n) {
    const double t = (n - 15) / 10.0, b = 0.2;
    const double s = t == 0 ? 1.0 : std::sin(M_PI * t) / (M_PI * t);
    const double q = 1 - (2 * b * t) * (2 * b * t);
    rc[n]          = std::fabs(q) < 1e-12 ? 0.0 : s * std::cos(M_PI * b * t) / q;
  }
  float taps[3][16] = {};
  for (int sel = 0; sel < 3; ++sel) {
    const int nrb = sel + 1, ncoef = nrb * 10 + 1, nout = ncoef / 2 / 2, first = 15 - nout * 2, n = 2 * nout + 1;
    float     tot = 0.f;
    for (int i = 0; i < n; ++i) {
      taps[sel][i] = (float)rc[first + 2 * i];
      tot += taps[sel][i];
    }
    for (int i = 0; i < n; ++i) {
      taps[sel][i] *= 1.0f / tot;
    }
  }
  int rc2 = check_cuda(ctx,
                       cudaFuncSetAttribute(pusch_estimate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)est_smem_bytes(kMaxPil)),
                       "cudaFuncSetAttribute(pusch_estimate_kernel)");
  if (rc2 != PG_OK) {
    return rc2;
  }
  rc2 = check_cuda(ctx, cudaMemcpyToSymbol(c_rc_taps, taps, sizeof(taps)), "cudaMemcpyToSymbol(rc taps)");
  if (rc2 != PG_OK) {
    return rc2;
  }
  std::vector<uint32_t> gold;
  gold_tables_host(gold, kGoldWords);
  rc2 = check_cuda(ctx, cudaMalloc(&ctx->dev.gold, gold.size() * 4), "cudaMalloc(gold)");
  if (rc2 == PG_OK) {
    rc2 = check_cuda(ctx, cudaMemcpy(ctx->dev.gold, gold.data(), gold.size() * 4, cudaMemcpyHostToDevice),
                     "cudaMemcpy(gold)");
  }
  return rc2;
}

int validate_ues(pg_context* ctx, const pg_pusch_ue* ues, int n)
{
  if (n < 0 || (n > 0 && ues == nullptr)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid UE list");
  }
  if (n > kDemodMaxUes) {
    // The estimator's and demodulator's work lists carry the UE index in 16 bits.
    return set_error(ctx, PG_ERR_INVALID, "more than 65535 UEs in one batch");
  }
  for (int i = 0; i < n; ++i) {
    const pg_pusch_ue& u = ues[i];
    int                nd = 0;
    for (int s = u.first_symbol; s < u.first_symbol + u.nof_symbols; ++s) {
      nd += (u.dmrs_symbol_mask >> s) & 1;
    }
    const bool ok = u.nof_rb >= 1 && u.rb_start + u.nof_rb <= 275 && 12u * (u.rb_start + u.nof_rb) <= u.grid_nof_subc &&
                    (u.nof_layers == 1 || u.nof_layers == 2) &&
                    (u.nof_rx_ports == 1 || u.nof_rx_ports == 2 || u.nof_rx_ports == 4) &&
                    u.nof_layers <= u.nof_rx_ports && nd >= 1 && nd <= kMaxDmrs && u.first_symbol + u.nof_symbols <= 14 &&
                    u.dmrs_scaling > 0.f && (u.modulation_order == 2 || u.modulation_order == 4 ||
                                             u.modulation_order == 6 || u.modulation_order == 8);
    if (!ok) {
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(i) + ": unsupported PUSCH configuration");
    }
  }
  return PG_OK;
}

int est_work_build(const pg_pusch_ue* ues, int n, std::vector<uint32_t>& blob, uint32_t* pilot_words)
{
  std::vector<uint32_t> first((size_t)4 * n + 1);
  blob.clear();
  for (int u = 0; u < n; ++u) {
    const int nch = (6 * (int)ues[u].nof_rb + kChunk - 1) / kChunk;
    for (int p = 0; p < 4; ++p) {
      first[(size_t)4 * u + p] = (uint32_t)blob.size();
      if (p < ues[u].nof_rx_ports) {
        for (int c = 0; c < nch; ++c) {
          blob.push_back((uint32_t)u | ((uint32_t)p << 16) | ((uint32_t)c << 20));
        }
      }
    }
  }
  first[(size_t)4 * n] = (uint32_t)blob.size();
  const int nwork      = (int)blob.size();
  blob.insert(blob.end(), first.begin(), first.end());
  uint32_t words = 0;
  for (int u = 0; u < n; ++u) {
    blob.push_back(words);
    words += (uint32_t)(kMaxDmrs * dmrs_bit_words(ues[u].nof_rb));
  }
  if (pilot_words != nullptr) {
    *pilot_words = words;
  }
  return nwork;
}

int dmrs_bits_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, const uint32_t* work_dev, int nwork,
                     uint32_t* bits_dev, cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  dmrs_bits_kernel<<<dim3(1, n), 128, 0, s>>>(ues_dev, work_dev + nwork + 4 * (size_t)n + 1, bits_dev, ctx->dev.gold,
                                              kGoldWords);
  return check_cuda(ctx, cudaGetLastError(), "dmrs_bits_kernel launch");
}

int estimate_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, const uint32_t* work_dev, int nwork,
                    void* partials, int* arrivals, const uint32_t* grids, float* est, float* ls,
                    pg_port_result* results, cudaStream_t s, const uint32_t* pilot_bits)
{
  if (n == 0 || nwork == 0) {
    return PG_OK;
  }
  pusch_estimate_chunk_kernel<<<nwork, kChunkThreads, 0, s>>>(
      ues_dev, work_dev, grids, reinterpret_cast<float2*>(est), reinterpret_cast<float2*>(ls),
      static_cast<float4*>(partials), ctx->dev.gold, kGoldWords, arrivals, results, pilot_bits, n);
  return check_cuda(ctx, cudaGetLastError(), "pusch_estimate_chunk_kernel launch");
}

int estimate_launch_host(pg_context* ctx, const pg_pusch_ue* ues, int n, const uint32_t* grids, float* est, float* ls,
                         pg_port_result* results, cudaStream_t s)
{
  std::vector<uint32_t> blob;
  const int             nwork = est_work_build(ues, n, blob);
  std::vector<uint8_t>  staged((size_t)n * sizeof(pg_pusch_ue) + blob.size() * 4);
  std::memcpy(staged.data(), ues, (size_t)n * sizeof(pg_pusch_ue));
  std::memcpy(staged.data() + (size_t)n * sizeof(pg_pusch_ue), blob.data(), blob.size() * 4);
  void* dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_UE, staged.data(), staged.size(), s, &dev)) {
    return rc;
  }
  // Partial sums (nwork float4), then the per-port arrival counters (4 n ints, zeroed here; each
  // port's last chunk leaves its counter at zero again).
  const size_t part_bytes = (size_t)nwork * sizeof(float4);
  if (int rc = ensure_scratch(ctx, &ctx->est_partials, &ctx->est_partials_cap,
                              std::max<size_t>(16, part_bytes + (size_t)16 * n), "cudaMalloc(estimate partials)")) {
    return rc;
  }
  int* arrivals = reinterpret_cast<int*>(static_cast<uint8_t*>(ctx->est_partials) + part_bytes);
  if (int rc = check_cuda(ctx, cudaMemsetAsync(arrivals, 0, (size_t)16 * n, s), "cudaMemsetAsync(arrivals)")) {
    return rc;
  }
  const pg_pusch_ue* d_ues  = static_cast<const pg_pusch_ue*>(dev);
  const uint32_t*    d_work = reinterpret_cast<const uint32_t*>(static_cast<uint8_t*>(dev) + (size_t)n * sizeof(pg_pusch_ue));
  if (int rc = estimate_launch(ctx, d_ues, n, d_work, nwork, ctx->est_partials, arrivals, grids, est, ls, results, s)) {
    return rc;
  }
  return release_slot_after(ctx, SLOT_UE, s);
}

int max_nof_rb(const pg_pusch_ue* ues, int n)
{
  int m = 1;
  for (int i = 0; i < n; ++i) {
    m = std::max(m, (int)ues[i].nof_rb);
  }
  return m;
}

int dmrs_count(const pg_pusch_ue& u, int* d0, int* d1)
{
  int nd = 0;
  for (int s = u.first_symbol; s < u.first_symbol + u.nof_symbols; ++s) {
    if ((u.dmrs_symbol_mask >> s) & 1) {
      if (nd == 0) {
        *d0 = s;
      } else if (nd == 1) {
        *d1 = s;
      }
      ++nd;
    }
  }
  return nd;
}

} // namespace pg

using namespace pg;

extern "C" {

size_t pg_pusch_est_size(const pg_pusch_ue* ue)
{
  if (ue == nullptr) {
    return 0;
  }
  int d0 = 0, d1 = 0;
  return (size_t)ue->nof_rx_ports * dmrs_count(*ue, &d0, &d1) * ue->nof_layers * 12 * ue->nof_rb;
}

int pg_pusch_estimate_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids, float* est,
                             pg_port_result* results, void* stream)
{
  return pg_pusch_estimate_ls_device(ctx, ues, nof_ues, grids, est, nullptr, results, stream);
}

int pg_pusch_estimate_ls_device(pg_context* ctx, const pg_pusch_ue* ues, int nof_ues, const uint32_t* grids,
                                float* est, float* ls, pg_port_result* results, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ues(ctx, ues, nof_ues)) {
    return rc;
  }
  if (nof_ues == 0) {
    return PG_OK;
  }
  return estimate_launch_host(ctx, ues, nof_ues, grids, est, ls, results, static_cast<cudaStream_t>(stream));
}

int pg_pusch_symbol_estimates_device(pg_context* ctx, const pg_pusch_ue* ue, const float* est, const float* basis,
                                     uint32_t* out, void* stream)
{
  if (ctx == nullptr || ue == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ues(ctx, ue, 1)) {
    return rc;
  }
  int       d0 = 0, d1 = 0;
  const int nd = dmrs_count(*ue, &d0, &d1);
  symbol_estimates_kernel<<<dim3((ue->nof_layers * 12 * ue->nof_rb + 255) / 256, 14, ue->nof_rx_ports), 256, 0,
                            static_cast<cudaStream_t>(stream)>>>(*ue, reinterpret_cast<const float2*>(est),
                                                                 reinterpret_cast<const float2*>(basis), out, nd, d0,
                                                                 d1);
  return check_cuda(ctx, cudaGetLastError(), "symbol_estimates_kernel launch");
}

int pg_port_channel_estimate_host(pg_context* ctx, const pg_port_estimate_cfg* cfg, const uint32_t* grid,
                                  const float* pilots, float* freq_response, uint32_t* symbol_estimates,
                                  pg_port_estimate_result* result)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (cfg == nullptr || grid == nullptr || pilots == nullptr || freq_response == nullptr || result == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null argument");
  }
  const int mu = cfg->scs_khz == 15 ? 0 : cfg->scs_khz == 30 ? 1 : cfg->scs_khz == 60 ? 2 : cfg->scs_khz == 120 ? 3 : -1;
  if (mu < 0) {
    return set_error(ctx, PG_ERR_INVALID, "subcarrier spacing must be 15, 30, 60 or 120 kHz");
  }
  pg_pusch_ue ue       = {};
  ue.grid_nof_subc     = cfg->grid_nof_subc;
  ue.dmrs_scaling      = cfg->scaling;
  ue.rb_start          = cfg->rb_start;
  ue.nof_rb            = cfg->nof_rb;
  ue.dmrs_symbol_mask  = cfg->dmrs_symbol_mask;
  ue.first_symbol      = cfg->first_symbol;
  ue.nof_symbols       = cfg->nof_symbols;
  ue.nof_rx_ports      = 1;
  ue.nof_layers        = cfg->nof_layers;
  ue.modulation_order  = 2;
  ue.dc_subcarrier     = -1;
  {
    // One receive port is estimated whatever the layer count: validate the allocation as if the
    // UE had enough ports for its layers.
    pg_pusch_ue chk  = ue;
    chk.nof_rx_ports = 4;
    if (int rc = validate_ues(ctx, &chk, 1)) {
      return rc;
    }
  }
  int       d0 = 0, d1 = 0;
  const int nd   = dmrs_count(ue, &d0, &d1);
  const int nl   = ue.nof_layers;
  const int npil = 6 * ue.nof_rb;
  const int nsc  = 12 * ue.nof_rb;

  // Inverse-DFT size of the time-alignment estimator: the pilot count scaled by 4096 / 3300 (guard
  // against circular interference), rounded up to a power of two, at least 128
  // (time_alignment_estimator_dft_impl.cpp:19-24, :160-175).
  unsigned req = (unsigned)npil * kTaMaxDft / 3300u;
  unsigned N   = 1;
  while (N < req) {
    N <<= 1;
  }
  N = std::max(N, 128u);
  // Sampling rate of the correlation (stride 2 for the type-1 comb) and the window of half a cyclic
  // prefix (144 kappa / 2^(mu + 1)), with the reference's double arithmetic.
  const double tc          = 1.0 / (480000.0 * 4096.0);
  const double fs          = (double)((uint64_t)N * cfg->scs_khz * 1000u * 2u);
  const int    max_ta      = (int)std::floor((double)((144 * 64) >> (mu + 1)) * tc * fs);
  // OFDM symbol start epochs in useful-symbol durations (normal cyclic prefix): the first symbol of
  // each half subframe has 16 kappa more cyclic prefix.
  auto epoch = [&](int sym) {
    double e = 0.0;
    for (int i = 0; i <= sym; ++i) {
      const int  per_half = 7 << mu;
      const bool longcp   = (i % per_half) == 0;
      const double cp_tc  = (double)((144 * 64) >> mu) + (longcp ? 16.0 * 64.0 : 0.0);
      e += (i == 0 ? 0.0 : 1.0) + cp_tc / (double)((2048 * 64) >> mu);
    }
    return (float)e;
  };
  const float epoch_diff = nd == 2 ? epoch(d1) - epoch(d0) : 0.f;

  const size_t grid_words = (size_t)14 * cfg->grid_nof_subc;
  const size_t pil_bytes  = (size_t)nd * nl * npil * 8;
  const size_t est_bytes  = (size_t)nd * nl * nsc * 8;
  const size_t sym_bytes  = (size_t)14 * nl * nsc * 4;
  auto al                 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_pil      = al(grid_words * 4);
  const size_t o_est      = o_pil + al(pil_bytes);
  const size_t o_sym      = o_est + al(est_bytes);
  const size_t o_res      = o_sym + al(sym_bytes);
  const size_t o_cfo      = o_res + al(4 * sizeof(pg_port_result));
  const size_t o_corr     = o_cfo + al(4 * sizeof(float2));
  const size_t o_out      = o_corr + al((size_t)kTaMaxDft * 4);
  const size_t total      = o_out + al(sizeof(ta_cfo_out));
  cudaStream_t s          = ctx->stream;
  int          rc         = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, total, "cudaMalloc(port estimate)");
  }
  if (rc != PG_OK) {
    return rc;
  }
  char* b = static_cast<char*>(ctx->scratch_a);
  rc      = check_cuda(ctx, cudaMemcpyAsync(b, grid, grid_words * 4, cudaMemcpyHostToDevice, s), "H2D grid");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(b + o_pil, pilots, pil_bytes, cudaMemcpyHostToDevice, s), "H2D pilots");
  }
  void* dev = nullptr;
  if (rc == PG_OK) {
    rc = stage_slot(ctx, SLOT_UE, &ue, sizeof(ue), s, &dev);
  }
  if (rc == PG_OK) {
    pusch_estimate_kernel<<<dim3(1, 1), kEstThreads, est_smem_bytes(npil), s>>>(
        static_cast<const pg_pusch_ue*>(dev), reinterpret_cast<const uint32_t*>(b), reinterpret_cast<float2*>(b + o_est),
        nullptr, reinterpret_cast<pg_port_result*>(b + o_res), ctx->dev.gold, kGoldWords, npil,
        reinterpret_cast<const float2*>(b + o_pil), reinterpret_cast<float2*>(b + o_cfo));
    rc = check_cuda(ctx, cudaGetLastError(), "pusch_estimate_kernel launch");
  }
  if (rc == PG_OK && symbol_estimates != nullptr) {
    symbol_estimates_kernel<<<dim3((nl * nsc + 255) / 256, 14, 1), 256, 0, s>>>(
        ue, reinterpret_cast<const float2*>(b + o_est), nullptr, reinterpret_cast<uint32_t*>(b + o_sym), nd, d0, d1);
    rc = check_cuda(ctx, cudaGetLastError(), "symbol_estimates_kernel launch");
  }
  if (rc == PG_OK) {
    ta_correlation_kernel<<<(N + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float2*>(b + o_est), nd * nl, nsc,
                                                          npil, (int)N, reinterpret_cast<float*>(b + o_corr));
    rc = check_cuda(ctx, cudaGetLastError(), "ta_correlation_kernel launch");
  }
  if (rc == PG_OK) {
    ta_cfo_kernel<<<1, 32, 0, s>>>(reinterpret_cast<const float*>(b + o_corr), (int)N, max_ta, fs,
                                   nd == 2 ? reinterpret_cast<const float2*>(b + o_cfo) : nullptr, epoch_diff,
                                   (float)cfg->scs_khz * 1000.0f, reinterpret_cast<ta_cfo_out*>(b + o_out));
    rc = check_cuda(ctx, cudaGetLastError(), "ta_cfo_kernel launch");
  }
  pg_port_result pr  = {};
  ta_cfo_out     tco = {};
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(freq_response, b + o_est, est_bytes, cudaMemcpyDeviceToHost, s), "D2H est");
  }
  if (rc == PG_OK && symbol_estimates != nullptr) {
    rc = check_cuda(ctx, cudaMemcpyAsync(symbol_estimates, b + o_sym, sym_bytes, cudaMemcpyDeviceToHost, s),
                    "D2H symbol estimates");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(&pr, b + o_res, sizeof(pr), cudaMemcpyDeviceToHost, s), "D2H result");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(&tco, b + o_out, sizeof(tco), cudaMemcpyDeviceToHost, s), "D2H TA");
  }
  if (rc == PG_OK) {
    rc = release_slot_after(ctx, SLOT_UE, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  if (rc != PG_OK) {
    return rc;
  }
  result->noise_var        = pr.noise_var;
  result->epre             = pr.epre;
  result->snr              = pr.snr;
  result->rsrp[0]          = pr.rsrp[0];
  result->rsrp[1]          = pr.rsrp[1];
  result->cfo_hz           = tco.cfo_hz;
  result->time_alignment_s = tco.time_alignment_s;
  return PG_OK;
}

} // extern "C"

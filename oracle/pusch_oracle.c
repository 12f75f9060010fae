/* Test infrastructure only: plain-C CPU restatement of the reference's PUSCH receive-path
 * stages (the checker for the CUDA path; never linked into the product).
 *
 * Each function cites the reference code it restates. The LDPC decoder restates the
 * AVX-512/AVX2 variant (the two are bit-identical; the "generic" variant rounds its scaling
 * differently and is not the target).
 */
#include "pusch_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../ocudu-dapp-platform_b200/csrc/ldpc_base_graphs.inc"

/* ------------------------------------------------------------------------------------------ */
/* CRC: include/ocudu/phy/upper/channel_coding/crc_calculator.h:17-24 (polynomials) and        */
/* lib/phy/upper/channel_coding/crc_calculator_lut_impl.cpp:53-140 (MSB-first, init 0).         */

static void crc_params(int poly, uint32_t* g, int* order)
{
  switch (poly) {
    case PGO_CRC16: *g = 0x11021u; *order = 16; break;
    case PGO_CRC24A: *g = 0x1864cfbu; *order = 24; break;
    case PGO_CRC24B: *g = 0x1800063u; *order = 24; break;
    case PGO_CRC24C: *g = 0x1b2b117u; *order = 24; break;
    case PGO_CRC11: *g = 0xe21u; *order = 11; break;
    default: *g = 0x61u; *order = 6; break;
  }
}

uint32_t pgo_crc(int poly, const uint8_t* packed, int nbits)
{
  uint32_t g;
  int      order;
  crc_params(poly, &g, &order);
  uint32_t mask = (order == 32) ? 0xffffffffu : ((1u << order) - 1u);
  uint32_t rem  = 0;
  for (int i = 0; i < nbits; ++i) {
    uint32_t bit = (packed[i >> 3] >> (7 - (i & 7))) & 1u;
    uint32_t top = ((rem >> (order - 1)) & 1u) ^ bit;
    rem          = (rem << 1) & mask;
    if (top) {
      rem ^= g & mask;
    }
  }
  return rem;
}

/* ------------------------------------------------------------------------------------------ */
/* Base graph access (TS 38.212 Table 5.3.2-1 lifting-size sets).                              */

static int set_index(int Z)
{
  static const int a_tab[8] = {2, 3, 5, 7, 9, 11, 13, 15};
  for (int i = 0; i < 8; ++i) {
    int t = Z;
    while ((t % 2) == 0 && t > a_tab[i]) {
      t /= 2;
    }
    if (t == a_tab[i]) {
      return i;
    }
  }
  return -1;
}

int pgo_ldpc_edge_shift(int bg, int Z, int edge)
{
  int s = set_index(Z);
  int v = (bg == 1) ? PG_BG1_EDGE_V[edge][s] : PG_BG2_EDGE_V[edge][s];
  return v % Z;
}

/* ------------------------------------------------------------------------------------------ */
/* LLR arithmetic: include/ocudu/phy/upper/log_likelihood_ratio.h:235 (LLR_MAX = 120,         */
/* infinity = 127) and lib/phy/upper/log_likelihood_ratio.cpp:21-70 (special sums).           */

#define LLR_MAX 120
#define LLR_INF 127

int8_t pgo_llr_sum(int8_t a, int8_t b)
{
  if (a == -b) {
    return 0;
  }
  if (a == LLR_INF || a == -LLR_INF) {
    return a;
  }
  if (b == LLR_INF || b == -LLR_INF) {
    return b;
  }
  int t = (int)a + (int)b;
  if (t > LLR_MAX) {
    t = LLR_MAX;
  }
  if (t < -LLR_MAX) {
    t = -LLR_MAX;
  }
  return (int8_t)t;
}

/* ------------------------------------------------------------------------------------------ */
/* LDPC decoder.                                                                              */
/*  - decode() control flow: lib/phy/upper/channel_coding/ldpc/ldpc_decoder_impl.cpp:41-145    */
/*  - load_soft_bits (clamp +-64, 2Z punctured zeros): ldpc_decoder_impl.cpp:147-188          */
/*  - per-layer updates: ldpc_decoder_impl.cpp:190-306                                       */
/*  - element arithmetic: lib/phy/upper/channel_coding/ldpc/ldpc_decoder_avx512.cpp:69-253     */
/*  - scaling floor(x * floor(0.8*2^16) / 2^16) for |x| <= 120: avx512_support.h:47-89          */
/* The check-to-variable messages are kept per (row, edge, check lane) instead of the          */
/* reference's rotated-back per (row, variable slot, variable lane) layout; the stored values  */
/* are the same numbers, permuted.                                                            */

static int8_t sat8(int x)
{
  return (int8_t)(x > 127 ? 127 : (x < -128 ? -128 : x));
}

static int8_t v2c_msg(int8_t soft, int8_t c2v)
{
  int v = sat8((int)soft - (int)c2v);
  if (v > LLR_MAX) v = LLR_MAX;
  if (v < -LLR_MAX) v = -LLR_MAX;
  if (soft >= LLR_INF) v = LLR_INF;
  if (soft <= -LLR_INF) v = -LLR_INF;
  return (int8_t)v;
}

static int8_t soft_update(int8_t c2v, int8_t v2c)
{
  int  s      = sat8((int)c2v + (int)v2c);
  int  c_pinf = c2v > LLR_MAX, c_ninf = c2v < -LLR_MAX;
  int  v_pinf = v2c > LLR_MAX, v_ninf = v2c < -LLR_MAX;
  if (s > LLR_MAX || (c_pinf && !v_ninf) || (v_pinf && !c_ninf)) {
    s = LLR_INF;
  }
  if (s < -LLR_MAX || (c_ninf && !v_pinf) || (v_ninf && !c_pinf)) {
    s = -LLR_INF;
  }
  return (int8_t)s;
}

static int scale_mag(int m)
{
  /* 0.8f * 65536 truncated to uint16 = 52428; values above LLR_MAX pass unaltered. */
  return m > LLR_MAX ? m : ((m * 52428) >> 16);
}

static int hard_bits(const int8_t* soft, int nbits, uint8_t* out_packed)
{
  int ok = 1;
  memset(out_packed, 0, (size_t)((nbits + 7) / 8));
  for (int i = 0; i < nbits; ++i) {
    if (soft[i] <= 0) {
      out_packed[i >> 3] |= (uint8_t)(0x80u >> (i & 7));
    }
    if (soft[i] == 0) {
      ok = 0;
    }
  }
  return ok;
}

/* Syndrome check over the processed rows: ldpc_decoder_impl.cpp:329-387. */
static int syndrome_ok(int bg, int Z, const int8_t* soft, int nof_layers)
{
  const unsigned char* deg  = bg == 1 ? PG_BG1_ROW_DEG : PG_BG2_ROW_DEG;
  const unsigned char* cols = bg == 1 ? PG_BG1_EDGE_COL : PG_BG2_EDGE_COL;
  int                  e0   = 0;
  for (int r = 0; r < nof_layers; ++r) {
    for (int j = 0; j < Z; ++j) {
      int parity = 0;
      for (int e = 0; e < deg[r]; ++e) {
        int s = pgo_ldpc_edge_shift(bg, Z, e0 + e);
        int8_t x = soft[cols[e0 + e] * Z + (j + s) % Z];
        if (x == 0) {
          return 0;
        }
        parity ^= (x <= 0);
      }
      if (parity) {
        return 0;
      }
    }
    e0 += deg[r];
  }
  return 1;
}

int pgo_ldpc_decode(int bg, int Z, int nof_filler_bits, int crc_poly, int max_iterations, const int8_t* llrs,
                    int nof_llrs, uint8_t* out_packed)
{
  const int            Kb      = bg == 1 ? 22 : 10;
  const int            Nfull   = bg == 1 ? 68 : 52;
  const int            nrows   = bg == 1 ? 46 : 42;
  const unsigned char* deg     = bg == 1 ? PG_BG1_ROW_DEG : PG_BG2_ROW_DEG;
  const unsigned char* cols    = bg == 1 ? PG_BG1_EDGE_COL : PG_BG2_EDGE_COL;
  const int            nedges  = bg == 1 ? PG_BG1_EDGES : PG_BG2_EDGES;
  const int            msg_len = Kb * Z;

  /* Trim trailing zero LLRs (ldpc_decoder_impl.cpp:66-71). */
  int input_size = nof_llrs;
  while (input_size > 0 && llrs[input_size - 1] == 0) {
    --input_size;
  }
  if (input_size < msg_len) {
    memset(out_packed, 0xff, (size_t)((msg_len + 7) / 8));
    return 0;
  }

  int8_t* soft = (int8_t*)calloc((size_t)(Nfull * Z), 1);
  int8_t* c2v  = (int8_t*)calloc((size_t)(nedges * Z), 1);
  int8_t  v2c[32];

  /* load_soft_bits: full nodes clamped to +-64, a ragged tail copied as is. */
  int nof_full = nof_llrs / Z;
  for (int i = 0; i < nof_full * Z; ++i) {
    int8_t x      = llrs[i];
    soft[2 * Z + i] = (int8_t)(x > 64 ? 64 : (x < -64 ? -64 : x));
  }
  for (int i = nof_full * Z; i < nof_llrs; ++i) {
    soft[2 * Z + i] = llrs[i];
  }

  int cb_len = input_size + 2 * Z;
  if (cb_len < (Kb + 4) * Z) {
    cb_len = (Kb + 4) * Z;
  }
  if (cb_len % Z) {
    cb_len = (cb_len / Z + 1) * Z;
  }
  int nof_layers = cb_len / Z - Kb;
  if (nof_layers > nrows) {
    nof_layers = nrows;
  }

  int result = 0;
  for (int it = 0; it < max_iterations; ++it) {
    int e0 = 0;
    for (int r = 0; r < nof_layers; ++r) {
      int d = deg[r];
      for (int j = 0; j < Z; ++j) {
        int min1 = LLR_MAX, min2 = LLR_MAX, idx = 0;
        int sgn  = 0;
        for (int e = 0; e < d; ++e) {
          int    s   = pgo_ldpc_edge_shift(bg, Z, e0 + e);
          int    pos = cols[e0 + e] * Z + (j + s) % Z;
          int8_t m   = v2c_msg(soft[pos], c2v[(e0 + e) * Z + j]);
          v2c[e]     = m;
          int a      = m < 0 ? -m : m;
          if (min1 > a) {
            min2 = min1;
            min1 = a;
            idx  = e;
          } else if (min2 > a) {
            min2 = a;
          }
          sgn ^= (m < 0);
        }
        int s1 = scale_mag(min1), s2 = scale_mag(min2);
        for (int e = 0; e < d; ++e) {
          int    s   = pgo_ldpc_edge_shift(bg, Z, e0 + e);
          int    pos = cols[e0 + e] * Z + (j + s) % Z;
          int    mag = (idx == e) ? s2 : s1;
          int    neg = sgn ^ (v2c[e] < 0);
          int8_t c   = (int8_t)(neg ? -mag : mag);
          c2v[(e0 + e) * Z + j] = c;
          soft[pos]             = soft_update(c, v2c[e]);
        }
      }
      e0 += d;
    }
    if (crc_poly >= 0) {
      int ok = hard_bits(soft, msg_len, out_packed);
      if (ok && pgo_crc(crc_poly, out_packed, msg_len - nof_filler_bits) == 0) {
        result = it + 1;
        break;
      }
    }
  }
  if (crc_poly < 0) {
    int ok = hard_bits(soft, msg_len, out_packed);
    result = (ok && syndrome_ok(bg, Z, soft, nof_layers)) ? max_iterations : 0;
  }
  free(soft);
  free(c2v);
  return result;
}

/* ------------------------------------------------------------------------------------------ */
/* Rate dematching: lib/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher_impl.cpp:29-250.     */

static void fill(int8_t* p, int n, int8_t v)
{
  for (int i = 0; i < n; ++i) {
    p[i] = v;
  }
}

void pgo_rate_dematch(int bg, int Z, int rv, int qm, int Nref, int nof_filler_bits, int new_data, const int8_t* in,
                      int E, int8_t* out)
{
  static const int k0_bg1[4] = {0, 17, 33, 56};
  static const int k0_bg2[4] = {0, 13, 25, 43};
  const int        Kb        = bg == 1 ? 22 : 10;
  const int        N         = (bg == 1 ? 66 : 50) * Z;
  const int        Ncb       = (Nref > 0 && Nref < N) ? Nref : N;
  const int        nof_sys   = (Kb - 2) * Z;
  const int        nof_info  = nof_sys - nof_filler_bits;
  const int        k0        = (((bg == 1 ? k0_bg1[rv] : k0_bg2[rv]) * Ncb) / N) * Z;

  /* Bit de-interleaving: out[K*j + i] = in[i*Qm + j] (ldpc_rate_dematcher_impl.cpp:196-205). */
  int8_t* aux = (int8_t*)malloc((size_t)(E > 0 ? E : 1));
  if (qm <= 1) {
    memcpy(aux, in, (size_t)E);
  } else {
    int Kq = E / qm;
    for (int i = 0, t = 0; i < Kq; ++i) {
      for (int j = 0; j < qm; ++j, ++t) {
        aux[Kq * j + i] = in[t];
      }
    }
  }

  /* allot_llrs (ldpc_rate_dematcher_impl.cpp:110-194). */
  int          copy = new_data;
  const int8_t* p   = aux;
  int          left = E;
  fill(out + nof_info, nof_filler_bits, LLR_INF);
  int idx = k0;
  while (left > 0) {
    if (idx < nof_info) {
      int n = nof_info - idx < left ? nof_info - idx : left;
      if (copy) {
        fill(out, idx, 0);
        memcpy(out + idx, p, (size_t)n);
      } else {
        for (int i = 0; i < n; ++i) {
          out[idx + i] = pgo_llr_sum(out[idx + i], p[i]);
        }
      }
      idx += n;
      p += n;
      left -= n;
    } else if (copy) {
      fill(out, nof_info, 0);
      if (idx > nof_sys) {
        fill(out + nof_sys, idx - nof_sys, 0);
      }
    }
    if (copy && idx < nof_info) {
      fill(out + idx, nof_info - idx, 0);
    }
    if (idx < nof_sys) {
      idx = nof_sys;
    }
    int n = Ncb - idx < left ? Ncb - idx : left;
    if (copy) {
      memcpy(out + idx, p, (size_t)n);
    } else {
      for (int i = 0; i < n; ++i) {
        out[idx + i] = pgo_llr_sum(out[idx + i], p[i]);
      }
    }
    idx = (idx + n) % Ncb;
    p += n;
    left -= n;
    if (left > 0) {
      copy = 0;
    }
  }
  if (copy && idx != 0) {
    fill(out + idx, Ncb - idx, 0);
  }
  if (new_data && Ncb < N) {
    fill(out + Ncb, N - Ncb, 0);
  }
  free(aux);
}

/* ------------------------------------------------------------------------------------------ */
/* Soft demapping: lib/phy/upper/channel_modulation/demodulation_mapper_{qpsk,qam16,qam64,     */
/* qam256}.cpp (AVX2 kernels) and avx2_helpers.h:103-253 (quantize_ps: scale by 120/R, clip,   */
/* round to nearest even). The 64/256-QAM pieces are the max-log LLRs of the TS 38.211 Gray    */
/* mapping, computed here per call from the constellation.                                   */

static float rcp_noise(float n)
{
  return (n > 0.f) ? 1.0f / n : 0.0f;
}

static int8_t quantize_rne(float v, float scale)
{
  v = v * scale;
  if (v != v) {
    return 0;
  }
  if (v > 120.f) v = 120.f;
  if (v < -120.f) v = -120.f;
  return (int8_t)lrintf(v); /* default rounding mode: nearest, ties to even */
}

static int level_of(int code, int m)
{
  int t = 1;
  for (int k = m - 1; k >= 1; --k) {
    int bk = (code >> (m - 1 - k)) & 1;
    t      = (1 << (m - k)) - (1 - 2 * bk) * t;
  }
  return (1 - 2 * ((code >> (m - 1)) & 1)) * t;
}

/* Max-log LLR (times noise) of dimension bit k for component x, in units of 1/sqrt(E). */
static float maxlog_piece(float x, int m, int k, float unit, float energy)
{
  int   nlev = 1 << m;
  float w    = 2.0f * unit;
  int   idx  = (int)floorf(x / w) + nlev / 2;
  if (idx < 0) idx = 0;
  if (idx > nlev - 1) idx = nlev - 1;
  double xm    = (idx - nlev / 2) * 2 + 1;
  double best0 = 1e30, best1 = 1e30;
  int    s0 = 0, s1 = 0;
  for (int c = 0; c < nlev; ++c) {
    int    bk = (c >> (m - 1 - k)) & 1;
    int    l  = level_of(c, m);
    double d  = (xm - l) * (xm - l);
    if (bk == 0 && d < best0) { best0 = d; s0 = l; }
    if (bk == 1 && d < best1) { best1 = d; s1 = l; }
  }
  float slope     = (float)(2 * (s0 - s1)) * unit;
  float intercept = (float)(s1 * s1 - s0 * s0) / energy;
  return slope * x + intercept;
}

void pgo_demodulate_soft(int qm, const float* symbols, const float* noise_vars, int nof_symbols, int8_t* llrs)
{
  for (int i = 0; i < nof_symbols; ++i) {
    float  x[2] = {symbols[2 * i], symbols[2 * i + 1]};
    float  rcp  = rcp_noise(noise_vars[i]);
    int8_t* out = llrs + (size_t)i * qm;
    if (qm == 2) {
      float g = 2.0f * sqrtf(2.0f);
      out[0]  = quantize_rne((g * x[0]) * rcp, 120.f / 24.f);
      out[1]  = quantize_rne((g * x[1]) * rcp, 120.f / 24.f);
    } else if (qm == 4) {
      float s10 = 1.0f / sqrtf(10.0f);
      for (int c = 0; c < 2; ++c) {
        float first  = (4.0f * s10) * x[c];
        float second = 2.0f * first - copysignf(0.8f, x[c]);
        float v01    = fabsf(x[c]) > 2.0f * s10 ? second : first;
        float v23    = 0.8f - fabsf(first);
        int   z      = fabsf(x[c]) <= 1e-9f;
        out[c]       = quantize_rne(z ? 0.f : v01 * rcp, 6.0f);
        out[2 + c]   = quantize_rne(z ? 0.f : v23 * rcp, 6.0f);
      }
    } else {
      int   m      = qm / 2;
      float energy = qm == 6 ? 42.f : 170.f;
      float unit   = 1.0f / sqrtf(energy);
      for (int c = 0; c < 2; ++c) {
        int z = fabsf(x[c]) <= 1e-9f;
        for (int k = 0; k < m; ++k) {
          float v        = maxlog_piece(x[c], m, k, unit, energy) * rcp;
          out[2 * k + c] = quantize_rne(z ? 0.f : v, 6.0f);
        }
      }
    }
  }
}

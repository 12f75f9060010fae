// PUSCH demodulation on sm_100a: per resource element, the channel estimate of the OFDM symbol
// (time interpolation between the DM-RS symbols, rounded to bf16 as the reference's estimator
// returns it, DC subcarrier zeroed), equalisation, soft demapping and descrambling, fused in one
// kernel that writes the codeword LLRs in the reference's order: data symbols in time order,
// subcarriers in frequency order, layers, bits (pusch_demodulator_impl.cpp:254-461 with
// get_ch_data_estimates :510-545 and revert_scrambling :22-206).
//
// The descrambling sequence c_init = RNTI * 2^15 + n_ID is produced first, one 32-bit word per
// thread from the Gold basis table (pg_device.cuh).
#include "pg_internal.h"
#include "pg_device.cuh"

#include <algorithm>
#include <vector>

namespace {

__constant__ float c_slope_d[3][4][16];
__constant__ float c_intercept_d[3][4][16];
__constant__ float c_width_d[3];

struct cf {
  float r, i;
};
__device__ __forceinline__ cf cmul(cf a, cf b)
{
  return {__fsub_rn(__fmul_rn(a.r, b.r), __fmul_rn(a.i, b.i)), __fadd_rn(__fmul_rn(a.r, b.i), __fmul_rn(a.i, b.r))};
}
__device__ __forceinline__ cf cconjmul(cf a, cf b)
{
  return {__fadd_rn(__fmul_rn(a.r, b.r), __fmul_rn(a.i, b.i)), __fsub_rn(__fmul_rn(a.i, b.r), __fmul_rn(a.r, b.i))};
}
__device__ __forceinline__ cf cadd(cf a, cf b)
{
  return {__fadd_rn(a.r, b.r), __fadd_rn(a.i, b.i)};
}
__device__ __forceinline__ cf csub(cf a, cf b)
{
  return {__fsub_rn(a.r, b.r), __fsub_rn(a.i, b.i)};
}
__device__ __forceinline__ cf cscale(cf a, float s)
{
  return {__fmul_rn(a.r, s), __fmul_rn(a.i, s)};
}
__device__ __forceinline__ float cnorm(cf a)
{
  return __fadd_rn(__fmul_rn(a.r, a.r), __fmul_rn(a.i, a.i));
}
__device__ __forceinline__ cf cbf16(uint32_t v)
{
  return {__uint_as_float(v << 16), __uint_as_float(v & 0xffff0000u)};
}
// A complex FP32 value rounded to bf16 (round to nearest even, both parts in one conversion) and
// widened back to FP32.
__device__ __forceinline__ cf bf16_round2(float re, float im)
{
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(im), "f"(re));
  return {__uint_as_float(r << 16), __uint_as_float(r & 0xffff0000u)};
}

// Hardware reciprocal estimate (relative error below 2^-22): the equaliser and the demapper use
// it where the reference itself uses a 14-bit reciprocal estimate or a division.
__device__ __forceinline__ float rcp_est(float x)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ int8_t quantize(float v, float scale)
{
  v = __fmul_rn(v, scale);
  v = v > 120.f ? 120.f : (v < -120.f ? -120.f : v);
  if (!(v == v)) {
    return 0;
  }
  return (int8_t)__float2int_rn(v);
}

template <int QM>
__device__ __forceinline__ void demap(float xr, float xi, float nvar, int8_t* llr, const float* s_slope,
                                      const float* s_icpt, const float* s_width)
{
  const float rcp = (nvar > 0.f) ? rcp_est(nvar) : 0.f;
  if (QM == 2) {
    const float g = 2.0f * 1.41421353816986083984375f;
    llr[0]        = quantize(__fmul_rn(__fmul_rn(g, xr), rcp), 5.0f);
    llr[1]        = quantize(__fmul_rn(__fmul_rn(g, xi), rcp), 5.0f);
    return;
  }
  if (QM == 4) {
    const float s10  = 0.3162277638912200927734375f;
    const float x[2] = {xr, xi};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float first  = __fmul_rn(4.0f * s10, x[c]);
      const float second = __fsub_rn(__fmul_rn(2.0f, first), copysignf(0.8f, x[c]));
      const float v01    = fabsf(x[c]) > 2.0f * s10 ? second : first;
      const float v23    = __fsub_rn(0.8f, fabsf(first));
      const bool  z      = fabsf(x[c]) <= 1e-9f;
      llr[c]             = quantize(z ? 0.f : __fmul_rn(v01, rcp), 6.0f);
      llr[2 + c]         = quantize(z ? 0.f : __fmul_rn(v23, rcp), 6.0f);
    }
    return;
  }
  constexpr int t     = QM == 6 ? 1 : 2;
  constexpr int nint  = QM == 6 ? 8 : 16;
  // Interval index floor(x / width) as x times the stored reciprocal width: where the two differ
  // (x / width within an ulp of an integer) the neighbouring interval's line meets this one at
  // the boundary (the interval functions are continuous), so the LLR is the same within rounding.
  const float   iwidth = s_width[3 + t];
  const float   x[2]   = {xr, xi};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    int idx      = (int)floorf(__fmul_rn(x[c], iwidth)) + nint / 2;
    idx          = idx < 0 ? 0 : (idx > nint - 1 ? nint - 1 : idx);
    const bool z = fabsf(x[c]) <= 1e-9f;
#pragma unroll
    for (int b = 0; b < QM / 2; ++b) {
      const float v  = __fmul_rn(__fadd_rn(__fmul_rn(s_slope[(t * 4 + b) * 16 + idx], x[c]),
                                           s_icpt[(t * 4 + b) * 16 + idx]),
                                 rcp);
      llr[2 * b + c] = quantize(z ? 0.f : v, 6.0f);
    }
  }
}

__global__ void scrambling_kernel(const pg_pusch_ue* __restrict__ ues, const uint32_t* __restrict__ seq_offsets,
                                  uint32_t* __restrict__ seq, const uint32_t* __restrict__ gold, uint32_t gold_words)
{
  const pg_pusch_ue ue     = ues[blockIdx.y];
  int               ndmrs  = 0;
  for (int s = ue.first_symbol; s < ue.first_symbol + ue.nof_symbols; ++s) {
    ndmrs += (ue.dmrs_symbol_mask >> s) & 1;
  }
  const uint32_t g      = (uint32_t)(ue.nof_symbols - ndmrs) * 12u * ue.nof_rb * ue.nof_layers * ue.modulation_order;
  const uint32_t words  = (g + 31) / 32;
  const uint32_t c_init = ((uint32_t)ue.rnti << 15) + ue.n_id_data;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    seq[seq_offsets[blockIdx.y] + w] = pg::gold_word(gold, gold_words, c_init, 32u * w);
  }
}

// Descrambling of a soft-bit stream: thread i takes soft bits 32 i .. 32 i + 31 and Gold word i.
__global__ void descramble_kernel(uint32_t c_init, const int8_t* __restrict__ in, int8_t* __restrict__ out, size_t n,
                                  const uint32_t* __restrict__ gold, uint32_t gold_words)
{
  const size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (32 * w >= n) {
    return;
  }
  const uint32_t c   = pg::gold_word(gold, gold_words, c_init, 32u * (uint32_t)w);
  const size_t   end = n - 32 * w < 32 ? n - 32 * w : 32;
  for (size_t b = 0; b < end; ++b) {
    const int x        = in[32 * w + b];
    out[32 * w + b]    = (int8_t)(((c >> b) & 1u) ? -x : x);
  }
}

struct demap_tables {
  const float* slope;
  const float* icpt;
  const float* width;
};

template <int L, int P, int QM>
__device__ __forceinline__ void demod_re(const pg_pusch_ue& ue, const uint32_t* __restrict__ grid,
                                         const float2* __restrict__ est, const float2* __restrict__ basis,
                                         const pg_port_result* __restrict__ pres, int nd, float w, int sym, int re_idx,
                                         int j, const uint32_t* __restrict__ seq, int8_t* __restrict__ llr_out,
                                         const demap_tables& tb, const pg::rm_direct* __restrict__ dr,
                                         int8_t* __restrict__ rm_out, int estride, int je)
{
  // est / basis: [port][DM-RS symbol][layer][estride], this RE's subcarrier at index je (the whole
  // allocation, estride = 12 nof_rb and je = j, or a tile of it in shared memory).
  const int nsc     = estride;
  const int sc      = 12 * ue.rb_start + j;
  const bool is_dc  = sc == ue.dc_subcarrier;
  cf        y[P];
  cf        h[P][L];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    y[p] = cbf16(__ldg(grid + ((size_t)p * 14 + sym) * ue.grid_nof_subc + sc));
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const float2* f0 = est + (((size_t)p * nd) * L + l) * nsc;
      float2        v  = f0[je];
      if (nd == 2) {
        const float2 v1 = f0[(size_t)L * nsc + je];
        v               = make_float2(__fmaf_rn(v1.x - v.x, w, v.x), __fmaf_rn(v1.y - v.y, w, v.y));
        if (basis != nullptr) {
          // The learned estimator's time-basis terms a_1 w (1 - w) + a_2 w (1 - w) (2 w - 1).
          const float2* b0 = basis + (((size_t)p * nd) * L + l) * nsc;
          const float2  a1 = b0[je], a2 = b0[(size_t)L * nsc + je];
          const float   f1 = __fmul_rn(w, __fsub_rn(1.f, w));
          const float   f2 = __fmul_rn(f1, __fsub_rn(__fmul_rn(2.f, w), 1.f));
          v                = make_float2(__fmaf_rn(a2.x, f2, __fmaf_rn(a1.x, f1, v.x)),
                                         __fmaf_rn(a2.y, f2, __fmaf_rn(a1.y, f1, v.y)));
        }
      }
      h[p][l] = is_dc ? cf{0.f, 0.f} : bf16_round2(v.x, v.y);
    }
  }
  cf    s[L];
  float nv[L];
  if (L == 1) {
    float ch_mod = 0.f, nacc = 0.f;
    cf    acc    = {0.f, 0.f};
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float n2 = cnorm(h[p][0]);
      if (n2 < INFINITY) {
        ch_mod = __fadd_rn(ch_mod, n2);
        nacc   = __fadd_rn(nacc, __fmul_rn(n2, pres[p].noise_var));
        acc    = cadd(acc, cconjmul(y[p], h[p][0]));
      }
    }
    const bool  ok  = (ch_mod > 0.f) && (ch_mod < INFINITY);
    const float rcp = rcp_est(ch_mod);
    s[0]            = ok ? cscale(acc, rcp) : cf{0.f, 0.f};
    nv[0]           = ok ? __fmul_rn(nacc, __fmul_rn(rcp, rcp)) : INFINITY;
  } else {
    float noise = pres[0].noise_var;
#pragma unroll
    for (int p = 1; p < P; ++p) {
      noise = fmaxf(noise, pres[p].noise_var);
    }
    cf   G[L][L], Gi[L][L];
    bool ok = pg::is_normal(noise) && noise >= 0.f;
#pragma unroll
    for (int i = 0; i < L; ++i) {
#pragma unroll
      for (int k = 0; k < L; ++k) {
        if (k < i) {
          // Hermitian: conj(h_i) h_k and conj(h_k) h_i have equal real parts and opposite
          // imaginary parts in IEEE arithmetic (products commute, a - b = -(b - a)).
          G[i][k] = cf{G[k][i].r, -G[k][i].i};
        } else {
          cf acc = {0.f, 0.f};
#pragma unroll
          for (int p = 0; p < P; ++p) {
            acc = cadd(acc, cconjmul(h[p][i], h[p][k]));
          }
          G[i][k] = acc;
        }
        Gi[i][k] = cf{i == k ? 1.f : 0.f, 0.f};
      }
      ok        = ok && (G[i][i].r > 0.f);
      G[i][i].r = __fadd_rn(G[i][i].r, noise);
    }
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const cf    piv  = G[i][i];
      const float pn   = cnorm(piv);
      ok               = ok && (pn > 0.f);
      const cf    pinv = cscale(cf{piv.r, -piv.i}, rcp_est(pn));
      Gi[i][i]         = cf{1.f, 0.f};
#pragma unroll
      for (int k = i + 1; k < L; ++k) {
        G[i][k] = cmul(G[i][k], pinv);
      }
#pragma unroll
      for (int k = 0; k <= i; ++k) {
        Gi[i][k] = cmul(Gi[i][k], pinv);
      }
#pragma unroll
      for (int r = 0; r < L; ++r) {
        if (r != i) {
          const cf f = G[r][i];
#pragma unroll
          for (int k = i; k < L; ++k) {
            G[r][k] = csub(G[r][k], cmul(f, G[i][k]));
          }
#pragma unroll
          for (int k = 0; k < i; ++k) {
            Gi[r][k] = csub(Gi[r][k], cmul(f, Gi[i][k]));
          }
          const cf t = cmul(f, Gi[i][i]);
          Gi[r][i]   = cf{-t.r, -t.i};
        }
      }
    }
#pragma unroll
    for (int l = 0; l < L; ++l) {
      cf    acc  = {0.f, 0.f};
      float corr = 0.f;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        cf wv = {0.f, 0.f};
#pragma unroll
        for (int k = 0; k < L; ++k) {
          wv = cadd(wv, cconjmul(Gi[k][l], h[p][k]));
        }
        acc  = cadd(acc, cmul(wv, y[p]));
        corr = __fadd_rn(corr, cmul(wv, h[p][l]).r);
      }
      const float c = rcp_est(corr);
      s[l]          = ok ? cscale(acc, c) : cf{0.f, 0.f};
      nv[l]         = ok ? __fsub_rn(c, 1.f) : INFINITY;
    }
  }
  // Demap, descramble, store: LLR index (re * L + l) * QM + b.
  int8_t        llr[L * QM];
#pragma unroll
  for (int l = 0; l < L; ++l) {
    demap<QM>(s[l].r, s[l].i, nv[l], llr + l * QM, tb.slope, tb.icpt, tb.width);
  }
  const uint32_t bit0 = (uint32_t)re_idx * L * QM;
  const uint32_t wa   = __ldg(seq + (bit0 >> 5));
  const uint32_t wb   = __ldg(seq + (bit0 >> 5) + 1);
  const uint32_t sh   = bit0 & 31u;
  const uint32_t cbits = sh ? ((wa >> sh) | (wb << (32 - sh))) : wa;
  if (dr != nullptr) {
    // Fused rate dematching: the RE's L*QM bits lie in one codeblock (E is a multiple of L*QM);
    // bit l*QM + b is de-interleaver row b, column i0 + l, placed in the circular buffer.
    const uint32_t es = dr->e_small, el = dr->e_large, ns = dr->n_small;
    const uint32_t lo = ns * es;
    uint32_t       r, off, E;
    if (bit0 < lo) {
      r   = bit0 / es;
      off = r * es;
      E   = es;
    } else {
      r   = ns + (bit0 - lo) / el;
      off = lo + (r - ns) * el;
      E   = el;
    }
    const uint32_t kq  = E / QM;
    const uint32_t i0  = (bit0 - off) / QM;
    int8_t*        cbo = rm_out + dr->out0 + (size_t)r * dr->cb_len;
#pragma unroll
    for (int b = 0; b < QM; ++b) {
#pragma unroll
      for (int l = 0; l < L; ++l) {
        uint32_t v = dr->v0 + (uint32_t)b * kq + i0 + (uint32_t)l;
        v          = v >= dr->V ? v - dr->V : v;
        const uint32_t pos = v < dr->inf ? v : v + dr->F;
        const int      k   = l * QM + b;
        const int      x   = llr[k];
        cbo[pos]           = (int8_t)(((cbits >> k) & 1u) ? -x : x);
      }
    }
    return;
  }
  int8_t* out = llr_out + ue.llr_offset + bit0;
  // The RE's descrambled LLRs packed four to a word, stored with the widest store their address
  // allows (codewords of plans and batched calls start on 16-byte boundaries, so an RE's NB bytes
  // are NB-aligned for NB = 2, 4, 8, 16 and 4-aligned for 12).
  constexpr int NB = L * QM;
  uint32_t      wd[(NB + 3) / 4];
#pragma unroll
  for (int k = 0; k < (NB + 3) / 4; ++k) {
    wd[k] = 0;
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int v = llr[b];
    wd[b / 4] |= (uint32_t)(uint8_t)(int8_t)(((cbits >> b) & 1u) ? -v : v) << (8 * (b % 4));
  }
  const uintptr_t a = reinterpret_cast<uintptr_t>(out);
  if (NB == 16 && (a & 15u) == 0) {
    *reinterpret_cast<uint4*>(out) = make_uint4(wd[0], wd[1 % ((NB + 3) / 4)], wd[2 % ((NB + 3) / 4)],
                                                wd[3 % ((NB + 3) / 4)]);
  } else if (NB == 8 && (a & 7u) == 0) {
    *reinterpret_cast<uint2*>(out) = make_uint2(wd[0], wd[1 % ((NB + 3) / 4)]);
  } else if ((NB == 4 || NB == 12) && (a & 3u) == 0) {
#pragma unroll
    for (int k = 0; k < NB / 4; ++k) {
      reinterpret_cast<uint32_t*>(out)[k] = wd[k];
    }
  } else if ((NB == 2 || NB == 6) && (a & 1u) == 0) {
#pragma unroll
    for (int k = 0; k < NB / 2; ++k) {
      reinterpret_cast<uint16_t*>(out)[k] = (uint16_t)(wd[k / 2] >> (16 * (k % 2)));
    }
  } else {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      out[b] = (int8_t)(wd[b / 4] >> (8 * (b % 4)));
    }
  }
}

// Demodulation in tiles: one CTA per (UE, kDemodTile consecutive subcarriers of its allocation)
// over every data symbol. The CTA stages the tile's frequency responses (and the learned
// estimator's time-basis coefficients) in shared memory once, so each is read from memory once
// rather than once per data symbol; a warp's threads take consecutive subcarriers of one symbol,
// so grid reads and LLR stores stay coalesced.
constexpr int kDemodTile = 32;

template <int L, int P, int QM>
__device__ __forceinline__ void demod_tile(const pg_pusch_ue& ue, int u, int j0, int nt, int nd, const int* s_sym,
                                           const float* s_w, int nds, const uint32_t* grid, const float2* s_est,
                                           const float2* s_bas, const pg_port_result* pres, const uint32_t* sq,
                                           int8_t* llrs, const demap_tables& tb, const pg::rm_direct* dr,
                                           int8_t* rm_out)
{
  // Work item q = (data symbol q / kDemodTile, subcarrier j0 + q % kDemodTile); the missing
  // subcarriers of a UE's last, narrower tile idle.
  const int nsc = 12 * ue.nof_rb;
  for (int q = threadIdx.x; q < nds * kDemodTile; q += blockDim.x) {
    const int di = q / kDemodTile;
    const int jj = q % kDemodTile;
    if (jj < nt) {
      const int j = j0 + jj;
      demod_re<L, P, QM>(ue, grid, s_est, s_bas, pres, nd, s_w[di], s_sym[di], di * nsc + j, j, sq, llrs, tb, dr,
                         rm_out, kDemodTile, jj);
    }
  }
}

template <int L, int P>
__device__ __forceinline__ void demod_tile_qm(const pg_pusch_ue& ue, int u, int j0, int nt, int nd, const int* s_sym,
                                              const float* s_w, int nds, const uint32_t* grid, const float2* s_est,
                                              const float2* s_bas, const pg_port_result* pres, const uint32_t* sq,
                                              int8_t* llrs, const demap_tables& tb, const pg::rm_direct* dr,
                                              int8_t* rm_out)
{
  switch (ue.modulation_order) {
    case 2: demod_tile<L, P, 2>(ue, u, j0, nt, nd, s_sym, s_w, nds, grid, s_est, s_bas, pres, sq, llrs, tb, dr, rm_out); break;
    case 4: demod_tile<L, P, 4>(ue, u, j0, nt, nd, s_sym, s_w, nds, grid, s_est, s_bas, pres, sq, llrs, tb, dr, rm_out); break;
    case 6: demod_tile<L, P, 6>(ue, u, j0, nt, nd, s_sym, s_w, nds, grid, s_est, s_bas, pres, sq, llrs, tb, dr, rm_out); break;
    default: demod_tile<L, P, 8>(ue, u, j0, nt, nd, s_sym, s_w, nds, grid, s_est, s_bas, pres, sq, llrs, tb, dr, rm_out); break;
  }
}

// tiles_per_cta consecutive tiles of the batch's tile list per CTA (a launch-shape tunable).
// tile_map[t] = UE index | tile index within the UE's allocation << 16.
__global__ void __launch_bounds__(256) pusch_demod_kernel(const pg_pusch_ue* __restrict__ ues, uint32_t ntiles,
                                                          const uint32_t* __restrict__ tile_map,
                                                          const uint32_t* __restrict__ grids,
                                                          const float2* __restrict__ est_all,
                                                          const float2* __restrict__ basis_all,
                                                          const uint8_t* __restrict__ basis_use,
                                                          const pg_port_result* __restrict__ port_results,
                                                          const uint32_t* __restrict__ seq_offsets,
                                                          const uint32_t* __restrict__ seq, int8_t* __restrict__ llrs,
                                                          int tiles_per_cta, const pg::rm_direct* __restrict__ direct,
                                                          int8_t* __restrict__ rm_out)
{
  __shared__ float  s_slope[3 * 4 * 16];
  __shared__ float  s_icpt[3 * 4 * 16];
  __shared__ float  s_width[6]; // interval widths, then their reciprocals
  __shared__ float2 s_est[4 * 2 * 2 * kDemodTile];
  __shared__ float2 s_bas[4 * 2 * 2 * kDemodTile];
  __shared__ int    s_sym[14];
  __shared__ float  s_w[14];
  __shared__ pg_port_result s_pres[4];
  __shared__ pg::rm_direct  s_dr;
  for (int i = threadIdx.x; i < 3 * 4 * 16; i += blockDim.x) {
    s_slope[i] = (&c_slope_d[0][0][0])[i];
    s_icpt[i]  = (&c_intercept_d[0][0][0])[i];
  }
  if (threadIdx.x < 3) {
    s_width[threadIdx.x]     = c_width_d[threadIdx.x];
    s_width[3 + threadIdx.x] = 1.0f / c_width_d[threadIdx.x];
  }
  const demap_tables tb = {s_slope, s_icpt, s_width};
  for (int k = 0; k < tiles_per_cta; ++k) {
    const uint32_t t = blockIdx.x * (uint32_t)tiles_per_cta + (uint32_t)k;
    if (t >= ntiles) {
      break;
    }
    const uint32_t    tm  = __ldg(tile_map + t);
    const int         u   = (int)(tm & 0xffffu);
    const pg_pusch_ue ue  = ues[u];
    const int         nsc = 12 * ue.nof_rb;
    const int         j0  = (int)(tm >> 16) * kDemodTile;
    const int         nt  = min(kDemodTile, nsc - j0);
    // The allocation's DM-RS symbols (the first two are the interpolation's ends) and data symbols.
    const uint32_t alloc = ((1u << (ue.first_symbol + ue.nof_symbols)) - 1u) & ~((1u << ue.first_symbol) - 1u);
    const uint32_t dm    = ue.dmrs_symbol_mask & alloc;
    const uint32_t data  = alloc & ~dm;
    const int      nd    = __popc(dm);
    const int      nds   = __popc(data);
    const int      d0    = __ffs(dm) - 1;
    const int      d1    = __ffs(dm & (dm - 1u)) - 1;
    __syncthreads(); // the previous tile's readers are done with the shared arrays
    const bool placed = direct != nullptr && direct[u].enabled != 0;
    if (placed && threadIdx.x < sizeof(pg::rm_direct) / 4) {
      reinterpret_cast<uint32_t*>(&s_dr)[threadIdx.x] = reinterpret_cast<const uint32_t*>(direct + u)[threadIdx.x];
    }
    if (threadIdx.x < 14 && ((data >> threadIdx.x) & 1u)) {
      const int s      = (int)threadIdx.x;
      const int r      = __popc(data & ((1u << s) - 1u));
      s_sym[r]         = s;
      s_w[r]           = nd == 2 ? (float)(s - d0) / (float)(d1 - d0) : 0.f;
    }
    if (threadIdx.x >= 32 && threadIdx.x < 32 + ue.nof_rx_ports) {
      s_pres[threadIdx.x - 32] = port_results[(size_t)u * 4 + threadIdx.x - 32];
    }
    const int ne = nd == 2 ? 2 : 1;
    const bool use_basis = basis_all != nullptr && basis_use != nullptr && nd == 2 && basis_use[u] != 0;
    const float2* est = est_all + ue.est_offset;
    const float2* bas = use_basis ? basis_all + ue.est_offset : nullptr;
    for (int i = threadIdx.x; i < ue.nof_rx_ports * ne * ue.nof_layers * kDemodTile; i += blockDim.x) {
      const int row = i / kDemodTile;
      const int jj  = i % kDemodTile;
      if (jj < nt) {
        // row = (p * ne + d) * L + l of the tile; the allocation's est rows are (p * nd + d) * L + l.
        const int    l   = row % ue.nof_layers;
        const int    pd  = row / ue.nof_layers;
        const int    d   = pd % ne;
        const int    p   = pd / ne;
        const size_t src = ((size_t)(p * nd + d) * ue.nof_layers + l) * nsc + j0 + jj;
        s_est[row * kDemodTile + jj] = est[src];
        if (bas != nullptr) {
          s_bas[row * kDemodTile + jj] = bas[src];
        }
      }
    }
    __syncthreads();
    const pg::rm_direct*  dr   = placed ? &s_dr : nullptr;
    const uint32_t*       grid = grids + ue.grid_offset;
    const uint32_t*       sq   = seq + seq_offsets[u];
    const float2*         sb   = bas != nullptr ? s_bas : nullptr;
    if (ue.nof_layers == 1) {
      switch (ue.nof_rx_ports) {
        case 1: demod_tile_qm<1, 1>(ue, u, j0, nt, ne, s_sym, s_w, nds, grid, s_est, sb, s_pres, sq, llrs, tb, dr, rm_out); break;
        case 2: demod_tile_qm<1, 2>(ue, u, j0, nt, ne, s_sym, s_w, nds, grid, s_est, sb, s_pres, sq, llrs, tb, dr, rm_out); break;
        default: demod_tile_qm<1, 4>(ue, u, j0, nt, ne, s_sym, s_w, nds, grid, s_est, sb, s_pres, sq, llrs, tb, dr, rm_out); break;
      }
    } else {
      switch (ue.nof_rx_ports) {
        case 2: demod_tile_qm<2, 2>(ue, u, j0, nt, ne, s_sym, s_w, nds, grid, s_est, sb, s_pres, sq, llrs, tb, dr, rm_out); break;
        default: demod_tile_qm<2, 4>(ue, u, j0, nt, ne, s_sym, s_w, nds, grid, s_est, sb, s_pres, sq, llrs, tb, dr, rm_out); break;
      }
    }
  }
}

} // namespace

namespace pg {

int demod_upload_tables(pg_context* ctx, const void* slope, const void* intercept, const void* width)
{
  int rc = check_cuda(ctx, cudaMemcpyToSymbol(c_slope_d, slope, sizeof(c_slope_d)), "cudaMemcpyToSymbol");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_intercept_d, intercept, sizeof(c_intercept_d)), "cudaMemcpyToSymbol");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_width_d, width, sizeof(c_width_d)), "cudaMemcpyToSymbol");
  }
  return rc;
}

uint32_t ue_codeword_bits(const pg_pusch_ue& u)
{
  int ndmrs = 0;
  for (int s = u.first_symbol; s < u.first_symbol + u.nof_symbols; ++s) {
    ndmrs += (u.dmrs_symbol_mask >> s) & 1;
  }
  return (uint32_t)(u.nof_symbols - ndmrs) * 12u * u.nof_rb * u.nof_layers * u.modulation_order;
}

int descramble_launch(pg_context* ctx, uint32_t c_init, const int8_t* in, int8_t* out, size_t n, cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  // The Gold basis covers kGoldWords - 2 words from position 0.
  if ((n + 31) / 32 + 2 > kGoldWords) {
    return set_error(ctx, PG_ERR_INVALID, "soft-bit stream longer than the scrambling sequence table");
  }
  const size_t words = (n + 31) / 32;
  descramble_kernel<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(c_init, in, out, n, ctx->dev.gold, kGoldWords);
  return check_cuda(ctx, cudaGetLastError(), "descramble_kernel launch");
}

int scrambling_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t max_words,
                      const uint32_t* seq_offsets_dev, uint32_t* seq_dev, cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  scrambling_kernel<<<dim3(std::max(1u, std::min(64u, (max_words + 255) / 256)), n), 256, 0, s>>>(
      ues_dev, seq_offsets_dev, seq_dev, ctx->dev.gold, kGoldWords);
  return check_cuda(ctx, cudaGetLastError(), "scrambling_kernel launch");
}

int demod_only_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t total_tiles,
                      const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                      const pg_port_result* port_results, const uint32_t* seq_offsets_dev, const uint32_t* seq_dev,
                      int8_t* llrs, cudaStream_t s)
{
  return demod_only_launch(ctx, ues_dev, n, total_tiles, tile_map_dev, grids, est, port_results, seq_offsets_dev, seq_dev,
                           llrs, s, 256, 1);
}

int demod_only_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t total_tiles,
                      const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                      const pg_port_result* port_results, const uint32_t* seq_offsets_dev, const uint32_t* seq_dev,
                      int8_t* llrs, cudaStream_t s, int block, int res_per_thread, const float* basis,
                      const uint8_t* basis_use, const rm_direct* direct, int8_t* rm_out)
{
  if (n == 0 || total_tiles == 0) {
    return PG_OK;
  }
  if (n > kDemodMaxUes) {
    return set_error(ctx, PG_ERR_INVALID, "more than 65535 UEs in one demodulation batch");
  }
  if (block != 64 && block != 128 && block != 256) {
    block = 256;
  }
  res_per_thread       = std::max(1, std::min(8, res_per_thread));
  const uint32_t per   = (uint32_t)res_per_thread; // tiles per CTA
  pusch_demod_kernel<<<(total_tiles + per - 1) / per, block, 0, s>>>(
      ues_dev, total_tiles, tile_map_dev, grids, reinterpret_cast<const float2*>(est), reinterpret_cast<const float2*>(basis),
      basis_use, port_results, seq_offsets_dev, seq_dev, llrs, res_per_thread, direct, rm_out);
  return check_cuda(ctx, cudaGetLastError(), "pusch_demod_kernel launch");
}

// Enqueues scrambling-sequence generation and demodulation; seq_offsets_dev / seq_dev are
// device scratch sized by the caller from ue_codeword_bits, tile_map_dev holds the batch's
// demodulation tiles (demod_tile_map).
int demod_launch(pg_context* ctx, const pg_pusch_ue* ues_dev, int n, uint32_t max_words, uint32_t total_tiles,
                 const uint32_t* tile_map_dev, const uint32_t* grids, const float* est,
                 const pg_port_result* port_results, const uint32_t* seq_offsets_dev, uint32_t* seq_dev, int8_t* llrs,
                 cudaStream_t s)
{
  if (int rc = scrambling_launch(ctx, ues_dev, n, max_words, seq_offsets_dev, seq_dev, s)) {
    return rc;
  }
  return demod_only_launch(ctx, ues_dev, n, total_tiles, tile_map_dev, grids, est, port_results, seq_offsets_dev,
                           seq_dev, llrs, s);
}

// The batch's demodulation tiles (kDemodTile subcarriers each), UE by UE; returns their number.
uint32_t demod_tile_map(const pg_pusch_ue* ues, int n, std::vector<uint32_t>& map)
{
  uint32_t t = 0;
  for (int i = 0; i < n; ++i) {
    const uint32_t k = (12u * ues[i].nof_rb + kDemodTile - 1) / kDemodTile;
    for (uint32_t j = 0; j < k; ++j) {
      map.push_back((uint32_t)i | (j << 16));
    }
    t += k;
  }
  return t;
}

} // namespace pg

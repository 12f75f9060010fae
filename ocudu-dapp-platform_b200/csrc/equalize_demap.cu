// Channel equalisation and soft demapping for sm_100a.
//
// Equaliser (one thread per resource element), following channel_equalizer_generic_impl
// (lib/phy/upper/equalization/channel_equalizer_generic_impl.cpp:511-653):
//  * one layer (ZF or "MMSE"): maximum-ratio combining with per-port noise,
//    s = sum_p y_p conj(h_p) / (tx * sum_p |h_p|^2), var = sum_p |h_p|^2 n_p / (tx * sum |h|^2)^2,
//    ports with a non-finite |h|^2 skipped, (0, +inf) when the denominator is not positive and
//    finite (equalize_zf_1xn.h:25-153, SIMD path);
//  * two or more layers, MMSE: G = (tx H)^H (tx H) + n I with n the largest port noise
//    variance, Gauss-Jordan inverse, W = G^-1 (tx H)^H, s_l = (W y)_l / Re(W tx H)_ll,
//    var_l = 1 / Re(W tx H)_ll - 1 (equalize_mmse_mxn_simd.h:14-75, matrix_inverse.h).
// Reciprocals are IEEE-exact here (the reference uses the approximate rcp14/rcp instructions on
// some paths: its outputs carry up to 2^-14 relative error from that alone).
//
// Demapper (one thread per symbol), following demodulation_mapper_impl and the AVX2 kernels
// (lib/phy/upper/channel_modulation/demodulation_mapper_{qpsk,qam16,qam64,qam256}.cpp,
// avx2_helpers.h:103-253): max-log piecewise-linear LLRs times 1/noise (0 when the noise
// variance is not positive), scaled by 120/R (R = 24 for QPSK, 20 otherwise), clipped to
// +-120 and rounded to the nearest integer, ties to even. 16-, 64- and 256-QAM LLRs of a component
// whose magnitude is at most 1e-9 are zero.
#include "pg_internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

__device__ __forceinline__ float2 bf16x2_to_float2(uint32_t v)
{
  return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xffff0000u));
}

struct cf {
  float r, i;
};
__device__ __forceinline__ cf cmul(cf a, cf b)
{
  return {__fsub_rn(__fmul_rn(a.r, b.r), __fmul_rn(a.i, b.i)), __fadd_rn(__fmul_rn(a.r, b.i), __fmul_rn(a.i, b.r))};
}
__device__ __forceinline__ cf cconjmul(cf a, cf b) // a * conj(b)
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

struct port_noise {
  float v[8];
};

template <int P>
__global__ void equalize_1layer_kernel(int nof_re, const uint32_t* __restrict__ y, const uint32_t* __restrict__ h,
                                       port_noise nvar_port, float tx, float2* __restrict__ out,
                                       float* __restrict__ out_var)
{
  const int re = blockIdx.x * blockDim.x + threadIdx.x;
  if (re >= nof_re) {
    return;
  }
  float ch_mod = 0.f, nacc = 0.f;
  cf    acc    = {0.f, 0.f};
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const float2 yy = bf16x2_to_float2(__ldg(y + (size_t)p * nof_re + re));
    const float2 hh = bf16x2_to_float2(__ldg(h + (size_t)p * nof_re + re));
    const cf     yc = {yy.x, yy.y}, hc = {hh.x, hh.y};
    const float  n2 = cnorm(hc);
    if (n2 < INFINITY) {
      ch_mod = __fadd_rn(ch_mod, n2);
      nacc   = __fadd_rn(nacc, __fmul_rn(n2, nvar_port.v[p]));
      acc    = cadd(acc, cconjmul(yc, hc));
    }
  }
  const float d   = __fmul_rn(tx, ch_mod);
  const bool  ok  = (d > 0.f) && (d < INFINITY);
  const float rcp = __frcp_rn(d);
  out[re]         = ok ? make_float2(__fmul_rn(acc.r, rcp), __fmul_rn(acc.i, rcp)) : make_float2(0.f, 0.f);
  out_var[re]     = ok ? __fmul_rn(nacc, __fmul_rn(rcp, rcp)) : INFINITY;
}

template <int L, int P>
__global__ void equalize_mmse_kernel(int nof_re, const uint32_t* __restrict__ y, const uint32_t* __restrict__ h,
                                     float noise, float tx, float2* __restrict__ out, float* __restrict__ out_var)
{
  const int re = blockIdx.x * blockDim.x + threadIdx.x;
  if (re >= nof_re) {
    return;
  }
  cf H[P][L], Y[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const float2 yy = bf16x2_to_float2(__ldg(y + (size_t)p * nof_re + re));
    Y[p]            = {yy.x, yy.y};
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const float2 hh = bf16x2_to_float2(__ldg(h + ((size_t)p * L + l) * nof_re + re));
      H[p][l]         = cscale(cf{hh.x, hh.y}, tx);
    }
  }
  // Gram matrix in the reference's convention G[i][j] = sum_p H[p][i] conj(H[p][j]) (the transpose
  // of H^H H, gram_matrix.h), diagonal loaded with the noise variance.
  cf   G[L][L], Gi[L][L];
  bool ok = true;
#pragma unroll
  for (int i = 0; i < L; ++i) {
#pragma unroll
    for (int j = 0; j < L; ++j) {
      cf acc = {0.f, 0.f};
#pragma unroll
      for (int p = 0; p < P; ++p) {
        acc = cadd(acc, cconjmul(H[p][i], H[p][j]));
      }
      G[i][j]  = acc;
      Gi[i][j] = cf{i == j ? 1.f : 0.f, 0.f};
    }
    ok = ok && (G[i][i].r > 0.f);
    G[i][i].r = __fadd_rn(G[i][i].r, noise);
  }
  // Gauss-Jordan elimination in the reference's order (matrix_inverse.h).
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const cf    piv  = G[i][i];
    const float pn   = cnorm(piv);
    ok               = ok && (pn > 0.f);
    const cf    pinv = cscale(cf{piv.r, -piv.i}, __frcp_rn(pn));
    Gi[i][i]         = cf{1.f, 0.f};
#pragma unroll
    for (int j = i + 1; j < L; ++j) {
      G[i][j] = cmul(G[i][j], pinv);
    }
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      Gi[i][j] = cmul(Gi[i][j], pinv);
    }
#pragma unroll
    for (int k = 0; k < L; ++k) {
      if (k != i) {
        const cf f = G[k][i];
#pragma unroll
        for (int j = i; j < L; ++j) {
          G[k][j] = csub(G[k][j], cmul(f, G[i][j]));
        }
#pragma unroll
        for (int j = 0; j < i; ++j) {
          Gi[k][j] = csub(Gi[k][j], cmul(f, Gi[i][j]));
        }
        const cf t = cmul(f, Gi[i][i]);
        Gi[k][i]   = cf{-t.r, -t.i};
      }
    }
  }
  // W[l][p] = sum_k Gi[k][l] conj(H[p][k]) (Gi is the inverse of the transposed Gram matrix).
#pragma unroll
  for (int l = 0; l < L; ++l) {
    cf    s    = {0.f, 0.f};
    float corr = 0.f;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      cf w = {0.f, 0.f};
#pragma unroll
      for (int k = 0; k < L; ++k) {
        w = cadd(w, cconjmul(Gi[k][l], H[p][k]));
      }
      s    = cadd(s, cmul(w, Y[p]));
      corr = __fadd_rn(corr, cmul(w, H[p][l]).r);
    }
    const float c = __frcp_rn(corr);
    out[(size_t)re * L + l]     = ok ? make_float2(__fmul_rn(s.r, c), __fmul_rn(s.i, c)) : make_float2(0.f, 0.f);
    out_var[(size_t)re * L + l] = ok ? __fsub_rn(c, 1.f) : INFINITY;
  }
}

// ---------------------------------------------------------------------------------------------
// Demapper tables: slopes and intercepts of the max-log LLR per interval of width 2/sqrt(E)
// (E = 10, 42, 170), derived on the host from the TS 38.211 Gray mapping.
__constant__ float c_slope[3][4][16];     // [16/64/256QAM][bit pair][interval]
__constant__ float c_intercept[3][4][16];
__constant__ float c_width[3];

__device__ __forceinline__ float quant_scale(int qm)
{
  return qm == 2 ? 120.f / 24.f : 120.f / 20.f;
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
__device__ __forceinline__ void demap_symbol(float xr, float xi, float nvar, int8_t* llr)
{
  const float rcp   = (nvar > 0.f) ? __frcp_rn(nvar) : 0.f;
  const float scale = quant_scale(QM);
  if (QM == 2) {
    const float g = 2.0f * 1.41421353816986083984375f; // 2 * sqrt(2) in float
    llr[0]        = quantize(__fmul_rn(__fmul_rn(g, xr), rcp), scale);
    llr[1]        = quantize(__fmul_rn(__fmul_rn(g, xi), rcp), scale);
    return;
  }
  if (QM == 4) {
    const float s10   = 0.3162277638912200927734375f; // 1/sqrt(10) in float
    const float x[2]  = {xr, xi};
    float       l01[2], l23[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float first  = __fmul_rn(4.0f * s10, x[c]);
      const float second = __fsub_rn(__fmul_rn(2.0f, first), copysignf(0.8f, x[c]));
      float       v01    = fabsf(x[c]) > 2.0f * s10 ? second : first;
      float       v23    = __fsub_rn(0.8f, fabsf(first));
      v01                = __fmul_rn(v01, rcp);
      v23                = __fmul_rn(v23, rcp);
      const bool z       = fabsf(x[c]) <= 1e-9f;
      l01[c]             = z ? 0.f : v01;
      l23[c]             = z ? 0.f : v23;
    }
    llr[0] = quantize(l01[0], scale);
    llr[1] = quantize(l01[1], scale);
    llr[2] = quantize(l23[0], scale);
    llr[3] = quantize(l23[1], scale);
    return;
  }
  constexpr int t     = QM == 6 ? 1 : 2;
  constexpr int nint  = QM == 6 ? 8 : 16;
  const float   width = c_width[t];
  const float   x[2]  = {xr, xi};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    int idx = (int)floorf(__fdiv_rn(x[c], width)) + nint / 2;
    idx     = idx < 0 ? 0 : (idx > nint - 1 ? nint - 1 : idx);
    const bool z = fabsf(x[c]) <= 1e-9f;
#pragma unroll
    for (int b = 0; b < QM / 2; ++b) {
      float v = __fmul_rn(__fadd_rn(__fmul_rn(c_slope[t][b][idx], x[c]), c_intercept[t][b][idx]), rcp);
      llr[2 * b + c] = quantize(z ? 0.f : v, scale);
    }
  }
}

template <int QM>
__global__ void demap_kernel(int n, const float2* __restrict__ sym, const float* __restrict__ nvar,
                             int8_t* __restrict__ llr)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const float2 s = sym[i];
  int8_t       out[QM];
  demap_symbol<QM>(s.x, s.y, nvar[i], out);
#pragma unroll
  for (int b = 0; b < QM; ++b) {
    llr[(size_t)i * QM + b] = out[b];
  }
}

} // namespace

namespace pg {

// Max-log LLR pieces for square QAM with Gray mapping per dimension (TS 38.211 Section 5.1):
// level(b_0, b_2, ...) = (1-2b_0)(2^(m-1) - (1-2b_2)(2^(m-2) - ...)) / sqrt(E). On interval i of
// width 2/sqrt(E) the LLR of bit pair k is LLR*noise = (x - s1)^2 - (x - s0)^2 with s0 / s1 the
// nearest levels whose bit k is 0 / 1: slope 2 (s0 - s1), intercept s1^2 - s0^2.
int demap_upload_tables(pg_context* ctx)
{
  float slope[3][4][16]     = {};
  float intercept[3][4][16] = {};
  float width[3]            = {};
  const int   bits_dim[3]   = {2, 3, 4};
  const float energy[3]     = {10.f, 42.f, 170.f};
  for (int t = 0; t < 3; ++t) {
    const int   m    = bits_dim[t];
    const int   nlev = 1 << m;
    const float unit = 1.0f / std::sqrt(energy[t]);
    width[t]         = 2 * unit;
    // Level of every code (bits b_0 (MSB) .. b_{m-1} of this dimension):
    // t = 1; for k = m-1 .. 1: t = 2^(m-k) - (1 - 2 b_k) t; level = (1 - 2 b_0) t.
    int lev[16], bits[16];
    for (int code = 0; code < nlev; ++code) {
      int tv = 1;
      for (int k = m - 1; k >= 1; --k) {
        const int bk = (code >> (m - 1 - k)) & 1;
        tv           = (1 << (m - k)) - (1 - 2 * bk) * tv;
      }
      const int b0 = (code >> (m - 1)) & 1;
      lev[code]    = (1 - 2 * b0) * tv;
      bits[code]   = code;
    }
    const int nint = nlev; // intervals of width 2 units covering [-nlev, nlev)
    for (int i = 0; i < nint && i < 16; ++i) {
      const double xm = (i - nint / 2) * 2 + 1; // interval midpoint in units
      for (int k = 0; k < m; ++k) {
        double best0 = 1e30, best1 = 1e30;
        int    s0 = 0, s1 = 0;
        for (int c = 0; c < nlev; ++c) {
          const int    bk = (bits[c] >> (m - 1 - k)) & 1;
          const double d  = (xm - lev[c]) * (xm - lev[c]);
          if (bk == 0 && d < best0) {
            best0 = d;
            s0    = lev[c];
          }
          if (bk == 1 && d < best1) {
            best1 = d;
            s1    = lev[c];
          }
        }
        slope[t][k][i]     = (float)(2 * (s0 - s1)) * unit;
        intercept[t][k][i] = (float)(s1 * s1 - s0 * s0) / energy[t];
      }
    }
  }
  int rc = demod_upload_tables(ctx, slope, intercept, width);
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_slope, slope, sizeof(slope)), "cudaMemcpyToSymbol(slope)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_intercept, intercept, sizeof(intercept)), "cudaMemcpyToSymbol");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_width, width, sizeof(width)), "cudaMemcpyToSymbol(width)");
  }
  return rc;
}

int equalize_launch(pg_context* ctx, int nof_re, int nof_ports, int nof_layers, const uint32_t* y, const uint32_t* h,
                    const float* nvar_port_host, float tx, float2* out, float* out_var, cudaStream_t s)
{
  if (nof_re == 0) {
    return PG_OK;
  }
  if (nof_ports < 1 || nof_ports > 8) {
    return set_error(ctx, PG_ERR_INVALID, "unsupported number of receive ports");
  }
  port_noise nvar_port_dev = {};
  float      noise_max     = 0.f;
  for (int p = 0; p < nof_ports; ++p) {
    nvar_port_dev.v[p] = nvar_port_host[p];
    noise_max          = p == 0 ? nvar_port_host[p] : std::max(noise_max, nvar_port_host[p]);
  }
  const int threads = 256, blocks = (nof_re + threads - 1) / threads;
  if (nof_layers == 1) {
    switch (nof_ports) {
      case 1: equalize_1layer_kernel<1><<<blocks, threads, 0, s>>>(nof_re, y, h, nvar_port_dev, tx, out, out_var); break;
      case 2: equalize_1layer_kernel<2><<<blocks, threads, 0, s>>>(nof_re, y, h, nvar_port_dev, tx, out, out_var); break;
      case 4: equalize_1layer_kernel<4><<<blocks, threads, 0, s>>>(nof_re, y, h, nvar_port_dev, tx, out, out_var); break;
      case 8: equalize_1layer_kernel<8><<<blocks, threads, 0, s>>>(nof_re, y, h, nvar_port_dev, tx, out, out_var); break;
      default: return set_error(ctx, PG_ERR_INVALID, "unsupported number of receive ports");
    }
  } else if (nof_layers == 2) {
    switch (nof_ports) {
      case 2: equalize_mmse_kernel<2, 2><<<blocks, threads, 0, s>>>(nof_re, y, h, noise_max, tx, out, out_var); break;
      case 4: equalize_mmse_kernel<2, 4><<<blocks, threads, 0, s>>>(nof_re, y, h, noise_max, tx, out, out_var); break;
      case 8: equalize_mmse_kernel<2, 8><<<blocks, threads, 0, s>>>(nof_re, y, h, noise_max, tx, out, out_var); break;
      default: return set_error(ctx, PG_ERR_INVALID, "unsupported port count for two layers");
    }
  } else if (nof_layers == 4) {
    switch (nof_ports) {
      case 4: equalize_mmse_kernel<4, 4><<<blocks, threads, 0, s>>>(nof_re, y, h, noise_max, tx, out, out_var); break;
      case 8: equalize_mmse_kernel<4, 8><<<blocks, threads, 0, s>>>(nof_re, y, h, noise_max, tx, out, out_var); break;
      default: return set_error(ctx, PG_ERR_INVALID, "unsupported port count for four layers");
    }
  } else {
    return set_error(ctx, PG_ERR_INVALID, "unsupported number of layers");
  }
  return check_cuda(ctx, cudaGetLastError(), "equalize kernel launch");
}

int demap_launch(pg_context* ctx, int qm, int n, const float2* sym, const float* nvar, int8_t* llr, cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  const int threads = 256, blocks = (n + threads - 1) / threads;
  switch (qm) {
    case 2: demap_kernel<2><<<blocks, threads, 0, s>>>(n, sym, nvar, llr); break;
    case 4: demap_kernel<4><<<blocks, threads, 0, s>>>(n, sym, nvar, llr); break;
    case 6: demap_kernel<6><<<blocks, threads, 0, s>>>(n, sym, nvar, llr); break;
    case 8: demap_kernel<8><<<blocks, threads, 0, s>>>(n, sym, nvar, llr); break;
    default: return set_error(ctx, PG_ERR_INVALID, "unsupported modulation order");
  }
  return check_cuda(ctx, cudaGetLastError(), "demap kernel launch");
}

} // namespace pg

using namespace pg;

extern "C" {

static int check_eq_args(pg_context* ctx, int algorithm, int nof_re, int nof_ports, int nof_layers,
                         const float* noise_var_per_port, float tx_scaling)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (nof_re < 0 || noise_var_per_port == nullptr || !(tx_scaling > 0.f) ||
      (algorithm != PG_EQ_ZF && algorithm != PG_EQ_MMSE)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid equaliser arguments");
  }
  if (nof_layers > 1 && algorithm == PG_EQ_ZF) {
    return set_error(ctx, PG_ERR_INVALID, "zero-forcing with several layers is not provided; use MMSE");
  }
  if (!((nof_layers == 1 && (nof_ports == 1 || nof_ports == 2 || nof_ports == 4 || nof_ports == 8)) ||
        (nof_layers == 2 && (nof_ports == 2 || nof_ports == 4 || nof_ports == 8)) ||
        (nof_layers == 4 && (nof_ports == 4 || nof_ports == 8)))) {
    return set_error(ctx, PG_ERR_INVALID, "unsupported ports/layers combination");
  }
  return PG_OK;
}

int pg_equalize_device(pg_context* ctx, int algorithm, int nof_re, int nof_ports, int nof_layers,
                       const uint32_t* ch_symbols, const uint32_t* ch_estimates, const float* noise_var_per_port,
                       float tx_scaling, float* eq_symbols, float* eq_noise_vars, void* stream)
{
  if (int rc = check_eq_args(ctx, algorithm, nof_re, nof_ports, nof_layers, noise_var_per_port, tx_scaling)) {
    return rc;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (nof_layers > 1) {
    float nmax = noise_var_per_port[0];
    for (int p = 1; p < nof_ports; ++p) {
      nmax = std::max(nmax, noise_var_per_port[p]);
    }
    if (!std::isnormal(nmax) || nmax < 0.f) {
      // The reference returns zeros and infinite variances (channel_equalizer_generic_impl.cpp:300-304).
      std::vector<float> inf((size_t)nof_re * nof_layers, INFINITY);
      int rc = check_cuda(ctx, cudaMemsetAsync(eq_symbols, 0, (size_t)nof_re * nof_layers * 8, s), "cudaMemsetAsync");
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaMemcpyAsync(eq_noise_vars, inf.data(), inf.size() * 4, cudaMemcpyHostToDevice, s),
                        "cudaMemcpyAsync");
      }
      if (rc == PG_OK) {
        rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
      }
      return rc;
    }
  }
  return equalize_launch(ctx, nof_re, nof_ports, nof_layers, ch_symbols, ch_estimates, noise_var_per_port, tx_scaling,
                         reinterpret_cast<float2*>(eq_symbols), eq_noise_vars, s);
}

int pg_equalize_host(pg_context* ctx, int algorithm, int nof_re, int nof_ports, int nof_layers,
                     const uint32_t* ch_symbols, const uint32_t* ch_estimates, const float* noise_var_per_port,
                     float tx_scaling, float* eq_symbols, float* eq_noise_vars)
{
  if (int rc = check_eq_args(ctx, algorithm, nof_re, nof_ports, nof_layers, noise_var_per_port, tx_scaling)) {
    return rc;
  }
  const size_t n_y  = (size_t)nof_re * nof_ports * 4;
  const size_t n_h  = (size_t)nof_re * nof_ports * nof_layers * 4;
  const size_t n_eq = (size_t)nof_re * nof_layers * 8;
  const size_t n_nv = (size_t)nof_re * nof_layers * 4;
  auto         al   = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t tot  = al(n_y) + al(n_h) + al(n_eq) + al(n_nv);
  if (int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
    return rc;
  }
  if (int rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(tot, 256), "cudaMalloc")) {
    return rc;
  }
  uint8_t*     b  = static_cast<uint8_t*>(ctx->scratch_a);
  uint32_t*    dy = reinterpret_cast<uint32_t*>(b);
  uint32_t*    dh = reinterpret_cast<uint32_t*>(b + al(n_y));
  float*       de = reinterpret_cast<float*>(b + al(n_y) + al(n_h));
  float*       dn = reinterpret_cast<float*>(b + al(n_y) + al(n_h) + al(n_eq));
  cudaStream_t s  = ctx->stream;
  int          rc = check_cuda(ctx, cudaMemcpyAsync(dy, ch_symbols, n_y, cudaMemcpyHostToDevice, s), "H2D symbols");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(dh, ch_estimates, n_h, cudaMemcpyHostToDevice, s), "H2D estimates");
  }
  if (rc == PG_OK) {
    rc = pg_equalize_device(ctx, algorithm, nof_re, nof_ports, nof_layers, dy, dh, noise_var_per_port, tx_scaling, de,
                            dn, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(eq_symbols, de, n_eq, cudaMemcpyDeviceToHost, s), "D2H symbols");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(eq_noise_vars, dn, n_nv, cudaMemcpyDeviceToHost, s), "D2H noise");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

int pg_demodulate_soft_device(pg_context* ctx, int modulation_order, int nof_symbols, const float* symbols,
                              const float* noise_vars, int8_t* llrs, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (nof_symbols < 0 || !(modulation_order == 2 || modulation_order == 4 || modulation_order == 6 ||
                           modulation_order == 8)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid demapper arguments");
  }
  return demap_launch(ctx, modulation_order, nof_symbols, reinterpret_cast<const float2*>(symbols), noise_vars, llrs,
                      static_cast<cudaStream_t>(stream));
}

int pg_demodulate_soft_host(pg_context* ctx, int modulation_order, int nof_symbols, const float* symbols,
                            const float* noise_vars, int8_t* llrs)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (nof_symbols < 0 || !(modulation_order == 2 || modulation_order == 4 || modulation_order == 6 ||
                           modulation_order == 8)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid demapper arguments");
  }
  const size_t n_s = (size_t)nof_symbols * 8, n_n = (size_t)nof_symbols * 4,
               n_l = (size_t)nof_symbols * modulation_order;
  auto         al  = [](size_t x) { return (x + 255) & ~(size_t)255; };
  if (int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
    return rc;
  }
  if (int rc = ensure_scratch(ctx, &ctx->scratch_a, &ctx->scratch_a_cap, std::max<size_t>(al(n_s) + al(n_n) + al(n_l), 256),
                              "cudaMalloc")) {
    return rc;
  }
  uint8_t*     b  = static_cast<uint8_t*>(ctx->scratch_a);
  cudaStream_t s  = ctx->stream;
  int          rc = check_cuda(ctx, cudaMemcpyAsync(b, symbols, n_s, cudaMemcpyHostToDevice, s), "H2D");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(b + al(n_s), noise_vars, n_n, cudaMemcpyHostToDevice, s), "H2D");
  }
  if (rc == PG_OK) {
    rc = demap_launch(ctx, modulation_order, nof_symbols, reinterpret_cast<const float2*>(b),
                      reinterpret_cast<const float*>(b + al(n_s)), reinterpret_cast<int8_t*>(b + al(n_s) + al(n_n)), s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(llrs, b + al(n_s) + al(n_n), n_l, cudaMemcpyDeviceToHost, s), "D2H");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

} // extern "C"

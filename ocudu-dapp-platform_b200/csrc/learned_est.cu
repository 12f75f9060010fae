// Learned DM-RS channel estimator: a residual 1-D convolutional network over the subcarriers of
// each (UE, receive port, layer) allocation that refines the frequency responses of the plain
// estimator (LS + RC smoothing + linear interpolation, pusch_est.cu) at the DM-RS symbols. The
// plain estimate stays the per-allocation fallback: the network only adds a correction, allocations
// can be left out, and a correction that is not finite is dropped. No counterpart in the
// reference (its estimator is port_channel_estimator_average_impl; the learned part is an
// addition of this library).
//
// Network (14 layers, kernel 5, 'same' padding, BF16 activations, FP32 accumulation on the tensor
// cores, tc_conv1d.cu):
//   x (16 features) -> conv 16->64, ReLU -> 6 x [conv 64->64, ReLU -> conv 64->64, + block input,
//   ReLU] -> conv 64->16 (linear); output channels 0..3 = correction of the DM-RS symbol 0 and 1
//   responses (re, im), in units of the allocation's RMS channel amplitude.
// Features per subcarrier k of an allocation of L = 12 nof_rb subcarriers, normalised by
// g = beta / sqrt(RSRP_layer) (the inverse RMS amplitude of the plain estimate):
//   0-3  plain estimate at DM-RS symbols 0 and 1 (re, im; symbol 1 repeats symbol 0 with one DM-RS symbol)
//   4-7  LS estimate at the pilots (even k; zero on odd k), DM-RS symbols 0 and 1
//   8    log10(noise_var g^2 / beta^2) / 2, clamped to [-4, 4] (the LS noise level)
//   9    1 on pilot subcarriers
//   10   max(0, 1 - k / 8), 11 max(0, 1 - (L - 1 - k) / 8)   (allocation edges)
//   12   1 with two layers (pair-averaged LS), 13 1 with two DM-RS symbols, 14-15 zero
// Row layout: the allocations one after another, two zero rows before each.
//
// Training (all on the GPU with this file's kernels and tc_conv1d.cu): features -> forward ->
// MSE of the correction against g (H_true - plain) -> backward (input gradients through the
// transposed convolutions with the ReLU masks, weight gradients on the tensor cores) -> Adam.
#include "pg_internal.h"
#include "tc_common.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

using namespace pg::tc;

constexpr int kLayers = 14;
constexpr int kBlocks = 6;
constexpr int kCh     = 64;
constexpr int kInCh   = 16;
constexpr int kOutCh  = 16;
constexpr int kTaps   = 5;
constexpr int kGap    = 2; // zero rows before each allocation

struct layer_desc {
  int cin, cout;
  int w_off; // floats: weights [5][cin][cout] at w_off, bias [cout] at w_off + 5 cin cout
  int p_off; // bf16 elements of this layer's packed weights
};

struct layer_table {
  layer_desc l[kLayers];
  int        nparams = 0, npacked = 0;
  layer_table()
  {
    int off = 0, poff = 0;
    for (int i = 0; i < kLayers; ++i) {
      const int cin  = i == 0 ? kInCh : kCh;
      const int cout = i == kLayers - 1 ? kOutCh : kCh;
      l[i]           = {cin, cout, off, poff};
      off += kTaps * cin * cout + cout;
      poff += kTaps * cin * cout;
    }
    nparams = off;
    npacked = poff;
  }
};

const layer_table& layers()
{
  static const layer_table t;
  return t;
}

__constant__ layer_desc c_layers[kLayers];

} // namespace

using pg::le_seq;

struct pg_le_net {
  pg_context* ctx      = nullptr;
  int         max_rows = 0;
  int         step     = 0;
  void*       dev      = nullptr;
  float*      params   = nullptr;
  float*      grads    = nullptr;
  float*      adam_m   = nullptr;
  float*      adam_v   = nullptr;
  uint16_t*   wf       = nullptr; // packed forward weights
  uint16_t*   wt       = nullptr; // packed transposed weights (input gradients)
  uint16_t*   wp       = nullptr; // packed weights of the fused inference kernel (taps along N)
  uint16_t*   x        = nullptr; // [2][R][8]
  uint16_t*   act[8]   = {};      // act[1..7]: [8][R][8] (act[0] = x)
  uint16_t*   mid[kBlocks] = {};  // [8][R][8]
  uint16_t*   y        = nullptr; // [2][R][8]
  uint16_t*   dy       = nullptr; // [2][R][8]
  uint16_t*   g0 = nullptr, *g1 = nullptr, *h = nullptr; // [8][R][8] gradients
  uint8_t*    row_valid = nullptr;
  pg::le_seq* seqs      = nullptr;
  float*      gseq      = nullptr;
  int*        err       = nullptr;
  float*      loss      = nullptr; // [2]
  int         max_seqs  = 0;
};

namespace {

using namespace pg::tc;

__device__ __forceinline__ int find_seq(const le_seq* __restrict__ seqs, int nseq, uint32_t r)
{
  int lo = 0, hi = nseq - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seqs[mid].row0 <= r) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float seq_gain(const le_seq& q, const pg_port_result* __restrict__ pr)
{
  const float rsrp = pr[q.pr].rsrp[q.layer];
  return (rsrp > 0.f && isfinite(rsrp)) ? q.beta * rsqrtf(rsrp) : 0.f;
}

__global__ void le_features_kernel(const le_seq* __restrict__ seqs, int nseq, int R, const float2* __restrict__ est,
                                   const float2* __restrict__ ls, const pg_port_result* __restrict__ pr,
                                   uint4* __restrict__ x, uint8_t* __restrict__ row_valid, float* __restrict__ gseq)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) {
    return;
  }
  const int    s = find_seq(seqs, nseq, (uint32_t)r);
  const le_seq q = seqs[s];
  const int    k = r - (int)q.row0;
  uint4        c0 = make_uint4(0, 0, 0, 0), c1 = make_uint4(0, 0, 0, 0);
  const bool   valid = k >= 0 && k < (int)q.len;
  if (valid) {
    const float  g   = seq_gain(q, pr);
    const size_t o0  = q.est0 + (size_t)k;
    const size_t o1  = o0 + (q.nd > 1 ? q.dstride : 0u);
    const float2 p0 = est[o0], p1 = est[o1], l0 = ls[o0], l1 = ls[o1];
    const float  nv  = pr[q.pr].noise_var;
    float        nf  = 0.f;
    if (g > 0.f) {
      nf = log10f(fmaxf(nv * g * g / (q.beta * q.beta), 1e-12f)) * 0.5f;
      nf = fminf(4.f, fmaxf(-4.f, isfinite(nf) ? nf : 0.f));
    }
    const float L = (float)q.len;
    c0            = make_uint4(pack_bf16x2(g * p0.x, g * p0.y), pack_bf16x2(g * p1.x, g * p1.y),
                               pack_bf16x2(g * l0.x, g * l0.y), pack_bf16x2(g * l1.x, g * l1.y));
    c1 = make_uint4(pack_bf16x2(g > 0.f ? nf : 0.f, (k & 1) ? 0.f : 1.f),
                    pack_bf16x2(fmaxf(0.f, 1.f - (float)k / 8.f), fmaxf(0.f, 1.f - (L - 1.f - (float)k) / 8.f)),
                    pack_bf16x2(q.nof_layers > 1 ? 1.f : 0.f, q.nd > 1 ? 1.f : 0.f), 0u);
    if (g <= 0.f) {
      c0 = make_uint4(0, 0, 0, 0);
      c1 = make_uint4(0, 0, 0, 0);
    }
    if (k == 0) {
      gseq[s] = g;
    }
  }
  x[r]                = c0;
  x[(size_t)R + r]    = c1;
  row_valid[r]        = valid ? 1 : 0;
}

// The eight bf16 channels of one 16-byte activation row.
__device__ __forceinline__ void unpack8(const uint4 v, float* o)
{
  const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    o[j] = __bfloat162float(b[j]);
  }
}

// Corrected estimates: est += correction / g at the DM-RS symbols; with two DM-RS symbols and a
// basis buffer (same layout as est), the time-basis coefficients a_1, a_2 / g of the rows go to
// basis[(port, b, layer)] (b = 0, 1): the channel at OFDM symbol s is then
//   h(s) = h_0 + (h_1 - h_0) w + a_1 w (1 - w) + a_2 w (1 - w) (2 w - 1),  w = (s - d0) / (d1 - d0),
// the linear interpolation of the reference's estimator plus two terms that vanish at the DM-RS
// symbols.
__global__ void le_apply_kernel(const le_seq* __restrict__ seqs, int nseq, int R, const uint4* __restrict__ y,
                                const float* __restrict__ gseq, float2* __restrict__ est, float2* __restrict__ basis)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) {
    return;
  }
  const int    s = find_seq(seqs, nseq, (uint32_t)r);
  const le_seq q = seqs[s];
  const int    k = r - (int)q.row0;
  const float  g = gseq[s];
  if (k < 0 || k >= (int)q.len || !(g > 0.f)) {
    return;
  }
  float o[8];
  unpack8(y[r], o);
  const float inv = 1.f / g;
  for (int d = 0; d < q.nd; ++d) {
    const float dx = o[2 * d] * inv, dyv = o[2 * d + 1] * inv;
    if (isfinite(dx) && isfinite(dyv)) {
      float2& e = est[q.est0 + (size_t)d * q.dstride + k];
      e.x += dx;
      e.y += dyv;
    }
  }
  if (basis != nullptr && q.nd == 2) {
    for (int b = 0; b < 2; ++b) {
      float ax = o[4 + 2 * b] * inv, ay = o[5 + 2 * b] * inv;
      if (!isfinite(ax) || !isfinite(ay)) {
        ax = ay = 0.f;
      }
      basis[q.est0 + (size_t)b * q.dstride + k] = make_float2(ax, ay);
    }
  }
}

// Mean squared error of the channel the network's outputs give at every data symbol of the slot
// (the DM-RS symbols carry no data) against the true channel, in the units of the features (x g):
// target t(s) = g (H(s) - plain(s)), plain(s) = the reference's linear interpolation of the plain
// estimates, prediction p(s) = c_0 + (c_1 - c_0) w + a_1 phi_1(w) + a_2 phi_2(w) with the output pairs
// (0,1) c_0, (2,3) c_1, (4,5) a_1, (6,7) a_2 (one DM-RS symbol: p(s) = c_0). dy = the gradient of
// sum |p - t|^2 inv_n; loss[0] += sum |p - t|^2 inv_n, loss[1] += sum |t|^2 inv_n (the plain
// estimator's error). h_full: [port][14][layer][subcarrier] per UE (le_seq::h0).
__global__ void le_loss_kernel(const le_seq* __restrict__ seqs, int nseq, int R, const uint4* __restrict__ y,
                               const float* __restrict__ gseq, const float2* __restrict__ est,
                               const float2* __restrict__ h_full, float inv_n, uint4* __restrict__ dy,
                               float* __restrict__ loss)
{
  const int r   = blockIdx.x * blockDim.x + threadIdx.x;
  float     l0  = 0.f, l1 = 0.f;
  if (r < R) {
    const int    s = find_seq(seqs, nseq, (uint32_t)r);
    const le_seq q = seqs[s];
    const int    k = r - (int)q.row0;
    const float  g = gseq[s];
    float        d8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (k >= 0 && k < (int)q.len && g > 0.f) {
      float o[8];
      unpack8(y[r], o);
      const int    d0 = q.dsym & 15, d1 = q.dsym >> 4;
      const float2 p0 = est[q.est0 + k];
      const float2 p1 = q.nd > 1 ? est[q.est0 + q.dstride + k] : p0;
      for (int sy = 0; sy < 14; ++sy) {
        if (sy == d0 || (q.nd > 1 && sy == d1)) {
          continue;
        }
        const float  w  = q.nd > 1 ? (float)(sy - d0) / (float)(d1 - d0) : 0.f;
        const float  f1 = q.nd > 1 ? w * (1.f - w) : 0.f;
        const float  f2 = f1 * (2.f * w - 1.f);
        const float2 h  = h_full[q.h0 + (size_t)sy * q.dstride + k];
        const float  tx = g * (h.x - (p0.x + (p1.x - p0.x) * w));
        const float  ty = g * (h.y - (p0.y + (p1.y - p0.y) * w));
        const float  px = q.nd > 1 ? o[0] + (o[2] - o[0]) * w + o[4] * f1 + o[6] * f2 : o[0];
        const float  py = q.nd > 1 ? o[1] + (o[3] - o[1]) * w + o[5] * f1 + o[7] * f2 : o[1];
        const float  ex = (px - tx) * 2.f * inv_n, ey = (py - ty) * 2.f * inv_n;
        if (q.nd > 1) {
          d8[0] += ex * (1.f - w);
          d8[1] += ey * (1.f - w);
          d8[2] += ex * w;
          d8[3] += ey * w;
          d8[4] += ex * f1;
          d8[5] += ey * f1;
          d8[6] += ex * f2;
          d8[7] += ey * f2;
        } else {
          d8[0] += ex;
          d8[1] += ey;
        }
        l0 += ((px - tx) * (px - tx) + (py - ty) * (py - ty)) * inv_n;
        l1 += (tx * tx + ty * ty) * inv_n;
      }
    }
    dy[r]             = make_uint4(pack_bf16x2(d8[0], d8[1]), pack_bf16x2(d8[2], d8[3]), pack_bf16x2(d8[4], d8[5]),
                                   pack_bf16x2(d8[6], d8[7]));
    dy[(size_t)R + r] = make_uint4(0, 0, 0, 0);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l0 += __shfl_xor_sync(0xffffffffu, l0, o);
    l1 += __shfl_xor_sync(0xffffffffu, l1, o);
  }
  if ((threadIdx.x & 31) == 0 && (l0 != 0.f || l1 != 0.f)) {
    atomicAdd(&loss[0], l0);
    atomicAdd(&loss[1], l1);
  }
}

__device__ __forceinline__ uint16_t bf16_bits(float f)
{
  const __nv_bfloat16 b = __float2bfloat16_rn(f);
  return *reinterpret_cast<const uint16_t*>(&b);
}

// Adam step (when update != 0) on every parameter, then the packed BF16 copies of the weights for
// the forward and the input-gradient convolutions and for the fused inference kernel; the gradients
// are cleared for the next step.
__global__ void le_adam_kernel(float* __restrict__ p, float* __restrict__ grad, float* __restrict__ m,
                               float* __restrict__ v, uint16_t* __restrict__ wf, uint16_t* __restrict__ wt,
                               uint16_t* __restrict__ wp, int total,
                               int update, float lr, float b1, float b2, float eps, float wd, float bc1, float bc2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) {
    return;
  }
  int li = 0;
#pragma unroll 1
  while (li + 1 < kLayers && c_layers[li + 1].w_off <= i) {
    ++li;
  }
  const layer_desc L  = c_layers[li];
  const int        j  = i - L.w_off;
  const int        nw = kTaps * L.cin * L.cout;
  float            w  = p[i];
  if (update) {
    const float gr = grad[i];
    const float mm = b1 * m[i] + (1.f - b1) * gr;
    const float vv = b2 * v[i] + (1.f - b2) * gr * gr;
    m[i]           = mm;
    v[i]           = vv;
    const float upd = (mm / bc1) / (sqrtf(vv / bc2) + eps) + (j < nw ? wd * w : 0.f);
    w -= lr * upd;
    p[i]    = w;
    grad[i] = 0.f;
  }
  if (j < nw) {
    const int t  = j / (L.cin * L.cout);
    const int r  = j - t * L.cin * L.cout;
    const int ci = r / L.cout;
    const int co = r - ci * L.cout;
    const uint16_t b = bf16_bits(w);
    wf[L.p_off + ((t * (L.cin / 8) + ci / 8) * L.cout + co) * 8 + (ci & 7)]              = b;
    wt[L.p_off + (((kTaps - 1 - t) * (L.cout / 8) + co / 8) * L.cin + ci) * 8 + (co & 7)] = b;
    wp[L.p_off + (((ci / 8) * kTaps + (kTaps - 1 - t)) * L.cout + co) * 8 + (ci & 7)]     = b;
  }
}

size_t al(size_t x)
{
  return (x + 255) & ~(size_t)255;
}
// ---------------------------------------------------------------------------------------------
// Fused inference: the whole network per window of 512 rows in one kernel, activations in shared
// memory, accumulators in tensor memory, each layer's weights brought in by 1-D bulk copies while
// the previous layer computes. Every layer loses two exact rows at each window edge (its taps reach
// two rows beyond), so after 14 layers the central 456 rows are exact and are the ones stored:
// windows overlap by 56 rows.
//
// Row pairs: an MMA row (M) is a pair of rows (2 r', 2 r' + 1) and its 2 x 64 accumulator columns
// are the output channels of both rows, so one MMA of N = 128 reads each A row once for two output
// rows. Shared memory keeps each buffer in two phase planes (even rows, odd rows), 8-channel chunks
// of row-pair lines of 16 bytes, with one pad pair before and after the window in each plane. The A
// operand x[2 r' + s] (s = -2 .. 3) is plane s & 1 starting floor(s / 2) pairs from r', a plain
// start-address offset. It feeds output row 2 r' through tap s + 2 and row 2 r' + 1 through tap
// s + 1, so the B operand of shift s is [W(s + 2) | W(s + 1)]: the weights are packed with the taps
// in descending order along N (taps 4, 3, 2, 1, 0, cout rows each) and B is 2 cout rows starting at
// tap s + 2. The two end shifts feed one row each (s = -2 row 2 r' through tap 0, s = 3 row
// 2 r' + 1 through tap 4) and are N = cout MMAs into their half of the accumulator; they come first
// in each tile, without accumulation, and initialise the two halves. Per 128-pair tile and 16 input
// channels: 4 MMAs of N = 128 and 2 of N = 64, against 10 of N = 64 with one row per MMA row.
//
// Buffers: A (block input and output; the second layer of a block adds the block input, kept as
// packed bf16 in tensor memory by the layer that wrote it, and writes A in place) and B (block
// middle; the 16 input features share its first two chunks, dead once layer 0's MMAs have
// completed, which precedes every write of B).
//
// Dataflow: the window is two M tiles of 128 pairs; the taps of either tile reach one pair into the
// other. A producer warp waits for tile 0's epilogue barrier of layer l - 1 and issues the shifts
// of tile 0 that read tile 0 only, loads the next layer's weights once layer l - 1's MMAs are
// complete, waits for tile 1's epilogue barrier, issues tile 0's two remaining shifts (they read
// tile 1's first pair) and commits tile 0, then issues and commits tile 1. Sixteen epilogue warps
// (four per TMEM lane quarter, 32 accumulator columns each) take tile 0 as soon as its MMAs
// complete - while tile 1's run - then tile 1: they add bias and residual, apply the ReLU and the
// row mask, store bf16 to shared memory, make the stores visible to the tensor cores and arrive on
// the tile's barrier. MMAs complete in issue order, so the epilogue of layer l writes its
// destination only after every MMA of layer l - 1 that read it.
constexpr int      kFTiles    = 2;
constexpr int      kFPairs    = 128 * kFTiles;
constexpr int      kFWin      = 2 * kFPairs;
constexpr int      kFPRows    = kFPairs + 2; // + one pad pair before and after, per plane
constexpr int      kFMargin   = 2 * kLayers;
constexpr int      kFOut      = kFWin - 2 * kFMargin;
constexpr int      kFOutHalf  = kFWin / 2 - 2 * kFMargin; // exact rows of a one-tile window
constexpr int      kFEpiWarps = 16;
constexpr int      kFThreads  = 32 * (kFEpiWarps + 1); // + producer warp
constexpr uint32_t kFChunkB   = kFPRows * 16;         // one 8-channel chunk of one plane
constexpr uint32_t kFActB     = 2 * 8 * kFChunkB;     // [plane][chunk][pair]
constexpr uint32_t kFWB       = kTaps * 8 * kCh * 16;
constexpr uint32_t kFOffW     = 2 * kFActB;
constexpr uint32_t kFOffBias  = kFOffW + 2 * kFWB;
constexpr uint32_t kFOffVal   = kFOffBias + kLayers * kCh * 4;
constexpr uint32_t kFOffBar   = kFOffVal + kFWin;
constexpr int      kFBars     = 2 * kFTiles + 2; // MMA done [2], epilogue done [2], weights [2]
constexpr size_t   kFSmem     = kFOffBar + 8 * kFBars + 16;
constexpr uint32_t kFCopy     = kFWB;  // bytes per bulk copy: one per layer (16 KB copies measured
                                       // 2 % slower, 4 KB copies 10 %)
constexpr uint32_t kFCols     = 512;   // TMEM columns: 128 accumulators per M tile, then 64 per tile
                                       // of packed bf16 block input (the residual two layers on)
constexpr uint32_t kFColRes   = 256;
static_assert(kFOffW % 16 == 0 && kFOffBias % 16 == 0 && kFOffBar % 8 == 0, "smem layout");
static_assert(kFSmem <= 227 * 1024, "shared memory of the fused kernel");
static_assert(kFChunkB % 16 == 0 && kFSmem < (1u << 18), "descriptor start addresses: 14 bits of 16-byte units");

__device__ __forceinline__ uint32_t layer_weight_bytes(int l)
{
  return (uint32_t)(kTaps * c_layers[l].cin * c_layers[l].cout * 2);
}

// Bulk copy of layer l's packed weights into `dst`, completing on `bar`.
__device__ __forceinline__ void fused_load_weights(const uint16_t* __restrict__ wp, int l, uint32_t dst, uint32_t bar)
{
  const uint32_t bytes = layer_weight_bytes(l);
  const char*    src   = reinterpret_cast<const char*>(wp + c_layers[l].p_off);
  mbar_expect_tx(bar, bytes);
  for (uint32_t o = 0; o < bytes; o += kFCopy) {
    bulk_g2s(dst + o, src + o, min(kFCopy, bytes - o), bar);
  }
}

// The MMAs of one input shift s (x[2 r' + s], all input chunks) of M tile c. The descriptors are
// formed once; each MMA adds its constant offset (16-byte units) to the start-address field, which
// stays below 2^14 (shared memory < 256 KB), so no carry reaches the LBO field. Shift -1 comes first
// in each tile and initialises both halves of the accumulator (N = 2 cout, no accumulation on the
// first chunk); every other MMA accumulates.
template <int CIN, int COUT, int S>
__device__ __forceinline__ void fused_issue_shift(uint64_t a0, uint64_t b0, uint32_t d)
{
  constexpr uint32_t idesc_pair = make_idesc(128, 2 * COUT, false, false);
  constexpr uint32_t idesc_one  = make_idesc(128, COUT, false, false);
  constexpr uint32_t lbo_b      = (uint32_t)kTaps * COUT * 16; // between 8-channel chunks of the weights
  constexpr uint32_t plane      = (uint32_t)(S & 1);
  constexpr uint32_t pofs       = (uint32_t)(1 + (S >> 1));      // 1 + floor(S / 2), pairs
  constexpr uint32_t tap_hi     = S == 3 ? 0u : (uint32_t)(2 - S); // first B tap block (descending taps)
#pragma unroll
  for (int kc = 0; kc < CIN / 16; ++kc) {
    const uint32_t a_off = (plane * 8u + 2u * (uint32_t)kc) * kFChunkB + pofs * 16u;
    const uint32_t b_off = 2u * (uint32_t)kc * lbo_b + tap_hi * COUT * 16u;
    const uint64_t ad    = a0 + (uint64_t)(a_off >> 4);
    const uint64_t bd    = b0 + (uint64_t)(b_off >> 4);
    if (S == 3) {
      mma_bf16(d + COUT, ad, bd, idesc_one, 1u);
    } else if (S == -2) {
      mma_bf16(d, ad, bd, idesc_one, 1u);
    } else {
      mma_bf16(d, ad, bd, idesc_pair, (S == -1 && kc == 0) ? 0u : 1u);
    }
  }
}

// The MMAs of M tile c of one layer: part 0 the shifts that read no pair beyond the tile's end
// (-1, -2, 0, 1), part 1 the two that read the next tile's first pair (2, 3), part 2 all six.
template <int CIN, int COUT>
__device__ __forceinline__ void fused_issue_tile(int c, int part, uint32_t src, uint32_t wb, uint32_t tmem)
{
  const uint64_t a0 = make_desc(src + (uint32_t)(c * 128) * 16u, kFChunkB, 128);
  const uint64_t b0 = make_desc(wb, (uint32_t)kTaps * COUT * 16, 128);
  const uint32_t d  = tmem + (uint32_t)(c * 128);
  if (part != 1) {
    fused_issue_shift<CIN, COUT, -1>(a0, b0, d);
    fused_issue_shift<CIN, COUT, -2>(a0, b0, d);
    fused_issue_shift<CIN, COUT, 0>(a0, b0, d);
    fused_issue_shift<CIN, COUT, 1>(a0, b0, d);
  }
  if (part != 0) {
    fused_issue_shift<CIN, COUT, 2>(a0, b0, d);
    fused_issue_shift<CIN, COUT, 3>(a0, b0, d);
  }
}

// Bounded wait that gives up at once when another thread has recorded a failure.
__device__ __forceinline__ bool fused_wait(uint32_t bar, uint32_t parity, volatile uint32_t* abort_sm,
                                           int* __restrict__ err)
{
  if (*abort_sm != 0) {
    return false;
  }
  if (mbar_wait_bounded(bar, parity)) {
    return true;
  }
  *abort_sm = 1;
  atomicExch(err, 1);
  return false;
}

__device__ __forceinline__ uint32_t fused_line(int plane, int chunk, int pair) // byte offset in a buffer
{
  return ((uint32_t)(plane * 8 + chunk)) * kFChunkB + (uint32_t)pair * 16u;
}

__global__ void __launch_bounds__(kFThreads, 1) le_fused_forward_kernel(const uint4* __restrict__ x,
                                                                        const uint8_t* __restrict__ row_valid,
                                                                        const uint16_t* __restrict__ wp,
                                                                        const float* __restrict__ params, int R,
                                                                        int n_full, int n_win, uint4* __restrict__ y,
                                                                        int* __restrict__ err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char*     buf_a    = smem;
  unsigned char*     buf_b    = smem + kFActB;
  float*             bias_s   = reinterpret_cast<float*>(smem + kFOffBias);
  uint8_t*           valid_s  = smem + kFOffVal;
  uint64_t*          bars     = reinterpret_cast<uint64_t*>(smem + kFOffBar);
  uint32_t*          tmem_sm  = reinterpret_cast<uint32_t*>(bars + kFBars);
  volatile uint32_t* abort_sm = tmem_sm + 1;
  const int          tid      = threadIdx.x;
  const int          warp     = tid >> 5;
  const int          lane     = tid & 31;
  if ((int)blockIdx.x >= n_win) {
    return;
  }
  // Pad pairs of every plane and chunk of both buffers: zero (those of B's first two chunks take
  // the input features of the rows beyond the window, loaded with each window).
  for (int i = tid; i < 2 * 2 * 8 * 2; i += kFThreads) {
    const int b = i >> 5, pl = (i >> 4) & 1, ch = (i >> 1) & 7, e = i & 1;
    *reinterpret_cast<uint4*>(smem + b * kFActB + fused_line(pl, ch, e ? kFPRows - 1 : 0)) = make_uint4(0, 0, 0, 0);
  }
  for (int i = tid; i < kLayers * kCh; i += kFThreads) {
    const int        l = i / kCh, co = i - l * kCh;
    const layer_desc L = c_layers[l];
    bias_s[i]          = co < L.cout ? params[L.w_off + kTaps * L.cin * L.cout + co] : 0.f;
  }
  const bool     producer = warp == kFEpiWarps;
  const uint32_t bar_mma  = smem_u32(&bars[0]);           // + 8c
  const uint32_t bar_epi  = smem_u32(&bars[kFTiles]);     // + 8c
  const uint32_t bar_w    = smem_u32(&bars[2 * kFTiles]); // + 8b
  const uint32_t wbuf0    = smem_u32(smem + kFOffW);
  const uint32_t act_a    = smem_u32(buf_a);
  const uint32_t act_b    = smem_u32(buf_b);
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_sm), kFCols);
  }
  if (producer && lane == 0) {
    for (int c = 0; c < kFTiles; ++c) {
      mbar_init(bar_mma + 8u * c, 1);
      mbar_init(bar_epi + 8u * c, kFEpiWarps);
    }
    mbar_init(bar_w, 1);
    mbar_init(bar_w + 8u, 1);
    *abort_sm = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fused_load_weights(wp, 0, wbuf0, bar_w);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_sm;
  // Epilogue role: TMEM lane quarter q, accumulator columns 32 cs .. 32 cs + 31 of each tile (plane
  // cs >> 1, channel half cs & 1; in the last layer warps cs < 2 take plane cs, 16 columns).
  const int      q          = warp & 3;
  const int      cs         = (warp >> 2) & 3;
  uint32_t       step       = 0; // layer steps of this CTA (all roles count alike)
  uint32_t       w_issued   = 1; // producer: weight loads issued (load k went to buffer k & 1)
  uint32_t       mma_issued = 0; // producer: layer steps whose MMAs were issued

  for (int win = blockIdx.x; win < n_win; win += gridDim.x) {
    // Windows 0 .. n_full - 1 have two M tiles, the rest one (kFOutHalf exact rows): the host picks
    // the split that evens out the work of the CTAs. A one-tile window keeps the barrier protocol
    // of two (its tile-1 steps arrive without work), so every barrier phase stays in step.
    const bool two  = win < n_full;
    const int  nout = two ? kFOut : kFOutHalf;
    const int  base = (two ? win * kFOut : n_full * kFOut + (win - n_full) * kFOutHalf) - kFMargin;
    const int  nrow = two ? kFWin : kFWin / 2; // window rows computed
    // Input features: window rows -2 .. nrow + 1 (pairs 0 .. nrow / 2 + 1 of both planes).
    for (int i = tid; i < 2 * (nrow + 4); i += kFThreads) {
      const int ch = i / (nrow + 4), w = i - ch * (nrow + 4) - 2, g = base + w;
      *reinterpret_cast<uint4*>(buf_b + fused_line(w & 1, ch, (w >> 1) + 1)) =
          (g >= 0 && g < R) ? x[(size_t)ch * R + g] : make_uint4(0, 0, 0, 0);
    }
    for (int i = tid; i < kFWin; i += kFThreads) {
      const int g = base + i;
      valid_s[i]  = (g >= 0 && g < R) ? row_valid[g] : 0;
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*abort_sm != 0) {
      break;
    }
    if (producer) {
      if (lane == 0) {
        for (int l = 0; l < kLayers; ++l) {
          const uint32_t s   = step + (uint32_t)l;
          const uint32_t src = (l & 1) ? act_a : act_b;
          if (!fused_wait(bar_w + 8u * (s & 1), (s >> 1) & 1u, abort_sm, err)) {
            break;
          }
          const uint32_t wb    = wbuf0 + (s & 1) * kFWB;
          auto           issue = [&](int c, int part) {
            if (l == 0) {
              fused_issue_tile<kInCh, kCh>(c, part, src, wb, tmem);
            } else if (l == kLayers - 1) {
              fused_issue_tile<kCh, kOutCh>(c, part, src, wb, tmem);
            } else {
              fused_issue_tile<kCh, kCh>(c, part, src, wb, tmem);
            }
          };
          // Layer 0 follows the window barrier. Later layers: tile 0's first part reads tile 0 of
          // layer l - 1 only, its second part and tile 1 also read tile 1 (and tile 1 overwrites
          // tile 1's accumulator), so the epilogue barriers are waited in between.
          if (l > 0) {
            if (!fused_wait(bar_epi, (s - 1) & 1u, abort_sm, err)) {
              break;
            }
            tc_fence_after();
          }
          issue(0, 0);
          // The MMAs of layer l - 1 are complete once its last commit (tile 1's barrier) has
          // arrived, which precedes the epilogue waited next; before layer 0, the window barrier.
          // Then its weight buffer takes the next layer (layer 0 of the next window after the
          // last layer), in flight while this layer's MMAs run.
          if (l > 0 && !fused_wait(bar_mma + 8u, (s - 1) & 1u, abort_sm, err)) {
            mma_commit(bar_mma);
            mma_commit(bar_mma + 8u);
            mma_issued = s + 1;
            break;
          }
          if (l + 1 < kLayers || win + (int)gridDim.x < n_win) {
            fused_load_weights(wp, (l + 1) % kLayers, wbuf0 + ((s + 1) & 1) * kFWB, bar_w + 8u * ((s + 1) & 1));
            ++w_issued;
          }
          if (l > 0) {
            if (!fused_wait(bar_epi + 8u, (s - 1) & 1u, abort_sm, err)) {
              // Tile 0's first part is in flight: both barriers take its completion, so that the
              // wait after a failure below covers it.
              mma_commit(bar_mma);
              mma_commit(bar_mma + 8u);
              mma_issued = s + 1;
              break;
            }
            tc_fence_after();
          }
          issue(0, 1);
          mma_commit(bar_mma);
          if (two) {
            issue(1, 2);
          }
          mma_commit(bar_mma + 8u);
          mma_issued = s + 1;
        }
      }
      __syncwarp();
    } else {
      for (int l = 0; l < kLayers; ++l) {
        const uint32_t s = step + (uint32_t)l;
        for (int c = 0; c < kFTiles; ++c) {
          // One lane polls the barrier and tells the others: probes from all 32 lanes take
          // shared-memory cycles from the tensor cores' operand reads (measured 13 % slower).
          bool ok = false;
          if (lane == 0) {
            ok = fused_wait(bar_mma + 8u * c, s & 1u, abort_sm, err);
          }
          ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
          if (ok && (two || c == 0)) {
            tc_fence_after();
            const int      pr  = c * 128 + q * 32 + lane;                 // window row pair
            const uint32_t tad = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * 128);
            if (l < kLayers - 1) {
              // 32 output channels (chunks 4 hh .. 4 hh + 3) of one row: one TMEM load of the
              // accumulators, then straight-line arithmetic. Layers 0, 2, .. 12 write the block
              // input, kept as packed bf16 in TMEM as well, where the second layer of the next block
              // reads its residual (no shared-memory reads beside the tensor cores').
              const int      plane  = cs >> 1, hh = cs & 1;
              const bool     valid  = valid_s[2 * pr + plane] != 0;
              const bool     second = l >= 2 && (l & 1) == 0;
              const bool     keep   = (l & 1) == 0;
              unsigned char* dst    = (l & 1) ? buf_b : buf_a;
              uint4*         p      = reinterpret_cast<uint4*>(dst + fused_line(plane, hh * 4, pr + 1));
              constexpr int  kStep  = kFChunkB / 16; // uint4 per chunk
              const float*   bl     = bias_s + l * kCh + hh * 32;
              const uint32_t tres   = tmem + ((uint32_t)(q * 32) << 16) + kFColRes + (uint32_t)(c * 64 + cs * 16);
              uint32_t       res[16];
              if (second) {
                float rf[16];
                tmem_ld16(tres, rf);
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                  res[k] = __float_as_uint(rf[k]);
                }
              }
              float v[32];
              tmem_ld32(tad + (uint32_t)(32 * cs), v);
              uint32_t kept[16];
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const float4 b0 = reinterpret_cast<const float4*>(bl)[2 * k];
                const float4 b1 = reinterpret_cast<const float4*>(bl)[2 * k + 1];
                const float  bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                float        o[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                  o[j] = v[8 * k + j] + bb[j];
                }
                if (second) {
#pragma unroll
                  for (int j = 0; j < 4; ++j) {
                    const __nv_bfloat162 rb = *reinterpret_cast<const __nv_bfloat162*>(&res[4 * k + j]);
                    o[2 * j] += __low2float(rb);
                    o[2 * j + 1] += __high2float(rb);
                  }
                }
                uint4 pk = make_uint4(0, 0, 0, 0);
                if (valid) {
                  pk = make_uint4(pack_bf16x2(fmaxf(o[0], 0.f), fmaxf(o[1], 0.f)),
                                  pack_bf16x2(fmaxf(o[2], 0.f), fmaxf(o[3], 0.f)),
                                  pack_bf16x2(fmaxf(o[4], 0.f), fmaxf(o[5], 0.f)),
                                  pack_bf16x2(fmaxf(o[6], 0.f), fmaxf(o[7], 0.f)));
                }
                p[k * kStep] = pk;
                kept[4 * k] = pk.x, kept[4 * k + 1] = pk.y, kept[4 * k + 2] = pk.z, kept[4 * k + 3] = pk.w;
              }
              if (keep) {
                tmem_st16(tres, kept);
                tmem_wait_st();
              }
              fence_async_shared();
            } else if (cs < 2) {
              const int    plane = cs;
              const int    wr    = 2 * pr + plane; // window row
              const bool   valid = valid_s[wr] != 0;
              const float* bl    = bias_s + l * kCh;
              float        v[16];
              tmem_ld16(tad + (uint32_t)(kOutCh * plane), v);
              const int g = base + wr;
              if (wr >= kFMargin && wr < kFMargin + nout && g < R) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  uint4 pk = make_uint4(0, 0, 0, 0);
                  if (valid) {
                    const float* b8 = bl + 8 * h;
                    const float* v8 = v + 8 * h;
                    pk = make_uint4(pack_bf16x2(v8[0] + b8[0], v8[1] + b8[1]), pack_bf16x2(v8[2] + b8[2], v8[3] + b8[3]),
                                    pack_bf16x2(v8[4] + b8[4], v8[5] + b8[5]), pack_bf16x2(v8[6] + b8[6], v8[7] + b8[7]));
                  }
                  y[(size_t)h * R + g] = pk;
                }
              }
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) {
            mbar_arrive(bar_epi + 8u * c);
          }
        }
      }
    }
    step += kLayers;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*abort_sm != 0) {
      break;
    }
  }
  // After a failure: the producer waits (bounded) for the MMAs and weight loads it issued, so that
  // nothing asynchronous is in flight when the tensor memory and shared memory go away.
  if (producer && lane == 0 && *abort_sm != 0) {
    if (mma_issued > 0) {
      for (int c = 0; c < kFTiles; ++c) {
        (void)mbar_wait_bounded(bar_mma + 8u * c, (mma_issued - 1) & 1u);
      }
    }
    for (uint32_t k = mma_issued; k < w_issued; ++k) {
      (void)mbar_wait_bounded(bar_w + 8u * (k & 1), (k >> 1) & 1u);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tmem_dealloc(tmem, kFCols);
  }
}

int fused_forward(pg_le_net* net, int R, cudaStream_t s);


int check_err_status(pg_le_net* net)
{
  int e = 0;
  if (int rc = pg::check_cuda(net->ctx, cudaMemcpy(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost),
                              "D2H learned-estimator status")) {
    return rc;
  }
  return e != 0 ? pg::set_error(net->ctx, PG_ERR_TIMEOUT, "a tensor-core completion wait expired") : PG_OK;
}

int forward(pg_le_net* net, int R, cudaStream_t s)
{
  pg_context*        ctx = net->ctx;
  const layer_table& T   = layers();
  auto w  = [&](int i) { return (const void*)(net->wf + T.l[i].p_off); };
  auto b  = [&](int i) { return (const float*)(net->params + T.l[i].w_off + kTaps * T.l[i].cin * T.l[i].cout); };
  int  rc = pg::conv_forward_launch(ctx, kInCh, kCh, net->x, w(0), b(0), nullptr, nullptr, net->act[1],
                                    net->row_valid, R, 1, net->err, s);
  for (int k = 0; k < kBlocks && rc == PG_OK; ++k) {
    rc = pg::conv_forward_launch(ctx, kCh, kCh, net->act[k + 1], w(1 + 2 * k), b(1 + 2 * k), nullptr, nullptr,
                                 net->mid[k], net->row_valid, R, 1, net->err, s);
    if (rc == PG_OK) {
      rc = pg::conv_forward_launch(ctx, kCh, kCh, net->mid[k], w(2 + 2 * k), b(2 + 2 * k), net->act[k + 1], nullptr,
                                   net->act[k + 2], net->row_valid, R, 1, net->err, s);
    }
  }
  if (rc == PG_OK) {
    rc = pg::conv_forward_launch(ctx, kCh, kOutCh, net->act[kBlocks + 1], w(kLayers - 1), b(kLayers - 1), nullptr,
                                 nullptr, net->y, net->row_valid, R, 0, net->err, s);
  }
  return rc;
}

// Windows of the fused kernel over R rows: n_full two-tile windows, then one-tile windows up to
// n_win, dealt round-robin to min(n_win, sms) CTAs. CTA 0 has the most of both kinds, so its cost
// (two-tile window 2, one-tile window 1) is the kernel's; the split with the lowest cost is taken,
// with the most two-tile windows among equals.
void fused_windows(int R, int sms, int* n_full, int* n_win)
{
  const int f0   = (R + kFOut - 1) / kFOut;
  int       best = -1;
  for (int f = f0; f >= std::max(0, f0 - sms); --f) {
    const int rem  = R - f * kFOut;
    const int w    = f + (rem > 0 ? (rem + kFOutHalf - 1) / kFOutHalf : 0);
    const int g    = std::max(1, std::min(w, sms));
    const int cost = (f + g - 1) / g + (w + g - 1) / g;
    if (best < 0 || cost < best) {
      best    = cost;
      *n_full = f;
      *n_win  = w;
    }
  }
}

int fused_forward(pg_le_net* net, int R, cudaStream_t s)
{
  if (R <= 0) {
    return PG_OK;
  }
  int n_full = 0, n_win = 0;
  fused_windows(R, net->ctx->sm_count, &n_full, &n_win);
  const int grid = std::max(1, std::min(n_win, net->ctx->sm_count));
  le_fused_forward_kernel<<<grid, kFThreads, kFSmem, s>>>(reinterpret_cast<const uint4*>(net->x), net->row_valid,
                                                          net->wp, net->params, R, n_full, n_win,
                                                          reinterpret_cast<uint4*>(net->y), net->err);
  return pg::check_cuda(net->ctx, cudaGetLastError(), "le_fused_forward_kernel launch");
}

// Gradients of every parameter (added to net->grads) from net->dy and the activations of the last
// forward pass.
int backward(pg_le_net* net, int R, cudaStream_t s)
{
  pg_context*        ctx = net->ctx;
  const layer_table& T   = layers();
  auto wt = [&](int i) { return (const void*)(net->wt + T.l[i].p_off); };
  auto gw = [&](int i) { return net->grads + T.l[i].w_off; };
  auto gb = [&](int i) { return net->grads + T.l[i].w_off + kTaps * T.l[i].cin * T.l[i].cout; };
  const int last = kLayers - 1;
  uint16_t* top  = net->act[kBlocks + 1];
  int rc = pg::conv_wgrad_launch(ctx, kCh, kOutCh, top, net->dy, R, gw(last), gb(last), net->err, s);
  if (rc == PG_OK) {
    rc = pg::conv_forward_launch(ctx, kOutCh, kCh, net->dy, wt(last), nullptr, nullptr, top, net->g0, net->row_valid,
                                 R, 0, net->err, s);
  }
  uint16_t* G = net->g0;
  uint16_t* Gn = net->g1;
  for (int k = kBlocks - 1; k >= 0 && rc == PG_OK; --k) {
    const int l2 = 2 + 2 * k, l1 = 1 + 2 * k;
    rc = pg::conv_wgrad_launch(ctx, kCh, kCh, net->mid[k], G, R, gw(l2), gb(l2), net->err, s);
    if (rc == PG_OK) {
      rc = pg::conv_forward_launch(ctx, kCh, kCh, G, wt(l2), nullptr, nullptr, net->mid[k], net->h, net->row_valid, R,
                                   0, net->err, s);
    }
    if (rc == PG_OK) {
      rc = pg::conv_wgrad_launch(ctx, kCh, kCh, net->act[k + 1], net->h, R, gw(l1), gb(l1), net->err, s);
    }
    if (rc == PG_OK) {
      rc = pg::conv_forward_launch(ctx, kCh, kCh, net->h, wt(l1), nullptr, G, net->act[k + 1], Gn, net->row_valid, R,
                                   0, net->err, s);
    }
    std::swap(G, Gn);
  }
  if (rc == PG_OK) {
    rc = pg::conv_wgrad_launch(ctx, kInCh, kCh, net->x, G, R, gw(0), gb(0), net->err, s);
  }
  return rc;
}

int pack_launch(pg_le_net* net, int update, const pg_le_adam* opt, cudaStream_t s)
{
  const int total = layers().nparams;
  float     lr = 0.f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f, wd = 0.f, bc1 = 1.f, bc2 = 1.f;
  if (update) {
    ++net->step;
    lr  = opt->lr;
    b1  = opt->beta1;
    b2  = opt->beta2;
    eps = opt->eps;
    wd  = opt->weight_decay;
    bc1 = 1.f - std::pow(b1, (float)net->step);
    bc2 = 1.f - std::pow(b2, (float)net->step);
  }
  le_adam_kernel<<<(total + 255) / 256, 256, 0, s>>>(net->params, net->grads, net->adam_m, net->adam_v, net->wf,
                                                     net->wt, net->wp, total, update, lr, b1, b2, eps, wd, bc1, bc2);
  return pg::check_cuda(net->ctx, cudaGetLastError(), "le_adam_kernel launch");
}

} // namespace

namespace pg {

// Sequences of the UEs with use[u] != 0 (all when use is null); returns the rows they need.
size_t le_build_seqs(const pg_pusch_ue* ues, int n, const uint8_t* use, std::vector<le_seq>& out, size_t* terms)
{
  out.clear();
  size_t row = 0, nterms = 0, h_base = 0;
  for (int u = 0; u < n; ++u) {
    if (use != nullptr && use[u] == 0) {
      h_base += (size_t)ues[u].nof_rx_ports * 14 * ues[u].nof_layers * 12 * ues[u].nof_rb;
      continue;
    }
    const pg_pusch_ue& ue = ues[u];
    int                d0 = 0, d1 = 0;
    const int          nd = dmrs_count(ue, &d0, &d1);
    const uint32_t     nsc = 12u * ue.nof_rb;
    for (int p = 0; p < ue.nof_rx_ports; ++p) {
      for (int l = 0; l < ue.nof_layers; ++l) {
        le_seq q{};
        row += kGap;
        q.row0       = (uint32_t)row;
        q.len        = nsc;
        q.est0       = ue.est_offset + (uint32_t)(((p * nd) * ue.nof_layers + l) * nsc);
        q.dstride    = (uint32_t)ue.nof_layers * nsc;
        q.pr         = (uint32_t)(u * 4 + p);
        q.beta       = ue.dmrs_scaling;
        q.layer      = (uint8_t)l;
        q.nof_layers = ue.nof_layers;
        q.nd         = (uint8_t)std::min(nd, 2);
        q.dsym       = (uint8_t)(d0 | ((q.nd > 1 ? d1 : d0) << 4));
        q.h0         = (uint32_t)(h_base + (size_t)((p * 14) * ue.nof_layers + l) * nsc);
        out.push_back(q);
        row += nsc;
        nterms += (size_t)nsc * 2 * (14 - q.nd);
      }
    }
    h_base += (size_t)ue.nof_rx_ports * 14 * ue.nof_layers * nsc;
  }
  if (terms != nullptr) {
    *terms = nterms;
  }
  return out.empty() ? 0 : row;
}

int le_refine_launch(pg_le_net* net, const le_seq* seqs_dev, int nseq, int R, const float* ls, float* est,
                     float* basis, const pg_port_result* pr, cudaStream_t s)
{
  if (nseq == 0 || R == 0) {
    return PG_OK;
  }
  le_features_kernel<<<(R + 255) / 256, 256, 0, s>>>(seqs_dev, nseq, R, reinterpret_cast<const float2*>(est),
                                                     reinterpret_cast<const float2*>(ls), pr,
                                                     reinterpret_cast<uint4*>(net->x), net->row_valid, net->gseq);
  int rc = check_cuda(net->ctx, cudaGetLastError(), "le_features_kernel launch");
  if (rc == PG_OK) {
    rc = fused_forward(net, R, s);
  }
  if (rc == PG_OK) {
    le_apply_kernel<<<(R + 255) / 256, 256, 0, s>>>(seqs_dev, nseq, R, reinterpret_cast<const uint4*>(net->y),
                                                    net->gseq, reinterpret_cast<float2*>(est),
                                                    reinterpret_cast<float2*>(basis));
    rc = check_cuda(net->ctx, cudaGetLastError(), "le_apply_kernel launch");
  }
  return rc;
}

int le_capacity(const pg_le_net* net, size_t rows, int nseq)
{
  return rows <= (size_t)net->max_rows && nseq <= net->max_seqs ? PG_OK : PG_ERR_CAPACITY;
}

pg_context* le_context(const pg_le_net* net)
{
  return net->ctx;
}

} // namespace pg

using namespace pg;

extern "C" {

size_t pg_le_nof_params(void)
{
  return (size_t)layers().nparams;
}

size_t pg_le_rows(const pg_pusch_ue* ues, int nof_ues)
{
  if (ues == nullptr || nof_ues <= 0) {
    return 0;
  }
  std::vector<le_seq> s;
  return le_build_seqs(ues, nof_ues, nullptr, s, nullptr);
}

int pg_le_create(pg_context* ctx, int max_rows, pg_le_net** out)
{
  if (ctx == nullptr || out == nullptr) {
    return PG_ERR_INVALID;
  }
  *out = nullptr;
  if (max_rows <= 0) {
    return set_error(ctx, PG_ERR_INVALID, "learned estimator: max_rows must be positive");
  }
  pg_le_net* n = new (std::nothrow) pg_le_net();
  if (n == nullptr) {
    return set_error(ctx, PG_ERR_CAPACITY, "out of host memory");
  }
  n->ctx      = ctx;
  n->max_rows = max_rows;
  n->max_seqs = max_rows / (12 + kGap) + 1;
  const layer_table& T = layers();
  const size_t R       = (size_t)max_rows;
  const size_t P       = (size_t)T.nparams;
  size_t       off     = 0;
  auto take            = [&](size_t bytes) {
    const size_t o = off;
    off += al(bytes);
    return o;
  };
  const size_t o_p = take(P * 4), o_g = take(P * 4), o_m = take(P * 4), o_v = take(P * 4);
  const size_t o_wf = take((size_t)T.npacked * 2), o_wt = take((size_t)T.npacked * 2),
               o_wp = take((size_t)T.npacked * 2);
  const size_t o_x = take(R * 32), o_y = take(R * 32), o_dy = take(R * 32);
  size_t o_act[8] = {}, o_mid[kBlocks] = {};
  for (int i = 1; i <= kBlocks + 1; ++i) {
    o_act[i] = take(R * 128);
  }
  for (int i = 0; i < kBlocks; ++i) {
    o_mid[i] = take(R * 128);
  }
  const size_t o_g0 = take(R * 128), o_g1 = take(R * 128), o_h = take(R * 128);
  const size_t o_rv = take(R), o_seq = take((size_t)n->max_seqs * sizeof(le_seq)),
               o_gs = take((size_t)n->max_seqs * 4), o_err = take(4), o_loss = take(8);
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&n->dev, off), "cudaMalloc(learned estimator)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemset(n->dev, 0, off), "cudaMemset(learned estimator)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaFuncSetAttribute(le_fused_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFSmem),
                    "cudaFuncSetAttribute(le_fused_forward_kernel)");
  }
  if (rc == PG_OK) {
    layer_desc ld[kLayers];
    std::copy(T.l, T.l + kLayers, ld);
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_layers, ld, sizeof(ld)), "cudaMemcpyToSymbol(layers)");
  }
  if (rc != PG_OK) {
    cudaFree(n->dev);
    delete n;
    return rc;
  }
  uint8_t* b   = static_cast<uint8_t*>(n->dev);
  n->params    = reinterpret_cast<float*>(b + o_p);
  n->grads     = reinterpret_cast<float*>(b + o_g);
  n->adam_m    = reinterpret_cast<float*>(b + o_m);
  n->adam_v    = reinterpret_cast<float*>(b + o_v);
  n->wf        = reinterpret_cast<uint16_t*>(b + o_wf);
  n->wt        = reinterpret_cast<uint16_t*>(b + o_wt);
  n->wp        = reinterpret_cast<uint16_t*>(b + o_wp);
  n->x         = reinterpret_cast<uint16_t*>(b + o_x);
  n->y         = reinterpret_cast<uint16_t*>(b + o_y);
  n->dy        = reinterpret_cast<uint16_t*>(b + o_dy);
  for (int i = 1; i <= kBlocks + 1; ++i) {
    n->act[i] = reinterpret_cast<uint16_t*>(b + o_act[i]);
  }
  n->act[0] = n->x;
  for (int i = 0; i < kBlocks; ++i) {
    n->mid[i] = reinterpret_cast<uint16_t*>(b + o_mid[i]);
  }
  n->g0        = reinterpret_cast<uint16_t*>(b + o_g0);
  n->g1        = reinterpret_cast<uint16_t*>(b + o_g1);
  n->h         = reinterpret_cast<uint16_t*>(b + o_h);
  n->row_valid = b + o_rv;
  n->seqs      = reinterpret_cast<le_seq*>(b + o_seq);
  n->gseq      = reinterpret_cast<float*>(b + o_gs);
  n->err       = reinterpret_cast<int*>(b + o_err);
  n->loss      = reinterpret_cast<float*>(b + o_loss);
  *out         = n;
  return PG_OK;
}

void pg_le_destroy(pg_le_net* net)
{
  if (net == nullptr) {
    return;
  }
  cudaDeviceSynchronize();
  cudaFree(net->dev);
  delete net;
}

int pg_le_set_params(pg_le_net* net, const float* params, size_t count)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (params == nullptr || count != (size_t)layers().nparams) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: parameter count mismatch");
  }
  cudaStream_t s  = net->ctx->stream;
  int          rc = check_cuda(net->ctx, cudaMemcpyAsync(net->params, params, count * 4, cudaMemcpyHostToDevice, s),
                               "H2D learned-estimator parameters");
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemsetAsync(net->adam_m, 0, count * 4, s), "cudaMemsetAsync(adam m)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemsetAsync(net->adam_v, 0, count * 4, s), "cudaMemsetAsync(adam v)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemsetAsync(net->grads, 0, count * 4, s), "cudaMemsetAsync(grads)");
  }
  if (rc == PG_OK) {
    net->step = 0;
    rc        = pack_launch(net, 0, nullptr, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

static int copy_out(pg_le_net* net, const float* src, float* dst, size_t count)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (dst == nullptr || count != (size_t)layers().nparams) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: parameter count mismatch");
  }
  if (int rc = check_cuda(net->ctx, cudaDeviceSynchronize(), "cudaDeviceSynchronize")) {
    return rc;
  }
  if (int rc = check_cuda(net->ctx, cudaMemcpy(dst, src, count * 4, cudaMemcpyDeviceToHost), "D2H parameters")) {
    return rc;
  }
  return check_err_status(net);
}

int pg_le_get_params(pg_le_net* net, float* params, size_t count)
{
  return copy_out(net, net != nullptr ? net->params : nullptr, params, count);
}

int pg_le_get_grads(pg_le_net* net, float* grads, size_t count)
{
  return copy_out(net, net != nullptr ? net->grads : nullptr, grads, count);
}

int pg_le_status(pg_le_net* net)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = check_cuda(net->ctx, cudaDeviceSynchronize(), "cudaDeviceSynchronize")) {
    return rc;
  }
  return check_err_status(net);
}

int pg_le_forward_device(pg_le_net* net, const void* x, const uint8_t* row_valid, int rows, void* y, void* stream)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (x == nullptr || row_valid == nullptr || y == nullptr || rows < 0) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: null buffer or negative row count");
  }
  if (rows > net->max_rows) {
    return set_error(net->ctx, PG_ERR_CAPACITY, "learned estimator: more rows than max_rows");
  }
  cudaStream_t s  = static_cast<cudaStream_t>(stream);
  int          rc = check_cuda(net->ctx, cudaMemcpyAsync(net->x, x, (size_t)rows * 32, cudaMemcpyDeviceToDevice, s),
                               "D2D features");
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemcpyAsync(net->row_valid, row_valid, rows, cudaMemcpyDeviceToDevice, s),
                    "D2D row mask");
  }
  if (rc == PG_OK) {
    rc = forward(net, rows, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemcpyAsync(y, net->y, (size_t)rows * 32, cudaMemcpyDeviceToDevice, s), "D2D out");
  }
  return rc;
}

int pg_le_backward_device(pg_le_net* net, const void* dy, int rows, void* stream)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (dy == nullptr || rows < 0 || rows > net->max_rows) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: null gradient or bad row count");
  }
  cudaStream_t s  = static_cast<cudaStream_t>(stream);
  int          rc = check_cuda(net->ctx, cudaMemsetAsync(net->grads, 0, (size_t)layers().nparams * 4, s),
                               "cudaMemsetAsync(grads)");
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemcpyAsync(net->dy, dy, (size_t)rows * 32, cudaMemcpyDeviceToDevice, s),
                    "D2D output gradient");
  }
  if (rc == PG_OK) {
    rc = backward(net, rows, s);
  }
  return rc;
}

static int stage_seqs(pg_le_net* net, const pg_pusch_ue* ues, int nof_ues, const uint8_t* use, int* nseq, int* R,
                      size_t* terms, cudaStream_t s)
{
  if (int rc = validate_ues(net->ctx, ues, nof_ues)) {
    return rc;
  }
  std::vector<le_seq> seqs;
  const size_t        rows = le_build_seqs(ues, nof_ues, use, seqs, terms);
  if (le_capacity(net, rows, (int)seqs.size()) != PG_OK) {
    return set_error(net->ctx, PG_ERR_CAPACITY,
                     "learned estimator: " + std::to_string(rows) + " rows exceed max_rows " +
                         std::to_string(net->max_rows));
  }
  *nseq = (int)seqs.size();
  *R    = (int)rows;
  if (seqs.empty()) {
    return PG_OK;
  }
  // Pageable source: the call returns once the descriptors have been copied out of `seqs`.
  return check_cuda(net->ctx,
                    cudaMemcpyAsync(net->seqs, seqs.data(), seqs.size() * sizeof(le_seq), cudaMemcpyHostToDevice, s),
                    "H2D learned-estimator sequences");
}

int pg_le_refine_device(pg_le_net* net, const pg_pusch_ue* ues, int nof_ues, const float* ls, float* est,
                        float* basis, const pg_port_result* port_results, const uint8_t* use, void* stream)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (ls == nullptr || est == nullptr || port_results == nullptr) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: null device buffer");
  }
  cudaStream_t s    = static_cast<cudaStream_t>(stream);
  int          nseq = 0, R = 0;
  if (int rc = stage_seqs(net, ues, nof_ues, use, &nseq, &R, nullptr, s)) {
    return rc;
  }
  return le_refine_launch(net, net->seqs, nseq, R, ls, est, basis, port_results, s);
}

int pg_le_train_step_device(pg_le_net* net, const pg_pusch_ue* ues, int nof_ues, const float* ls, const float* est,
                            const pg_port_result* port_results, const float* h_true, const pg_le_adam* opt,
                            float* loss, void* stream)
{
  if (net == nullptr) {
    return PG_ERR_INVALID;
  }
  if (ls == nullptr || est == nullptr || port_results == nullptr || h_true == nullptr || opt == nullptr) {
    return set_error(net->ctx, PG_ERR_INVALID, "learned estimator: null buffer");
  }
  cudaStream_t s    = static_cast<cudaStream_t>(stream);
  int          nseq = 0, R = 0;
  size_t       terms = 0;
  if (int rc = stage_seqs(net, ues, nof_ues, nullptr, &nseq, &R, &terms, s)) {
    return rc;
  }
  if (nseq == 0) {
    return PG_OK;
  }
  le_features_kernel<<<(R + 255) / 256, 256, 0, s>>>(net->seqs, nseq, R, reinterpret_cast<const float2*>(est),
                                                     reinterpret_cast<const float2*>(ls), port_results,
                                                     reinterpret_cast<uint4*>(net->x), net->row_valid, net->gseq);
  int rc = check_cuda(net->ctx, cudaGetLastError(), "le_features_kernel launch");
  if (rc == PG_OK) {
    rc = forward(net, R, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(net->ctx, cudaMemsetAsync(net->loss, 0, 8, s), "cudaMemsetAsync(loss)");
  }
  if (rc == PG_OK) {
    le_loss_kernel<<<(R + 255) / 256, 256, 0, s>>>(net->seqs, nseq, R, reinterpret_cast<const uint4*>(net->y),
                                                   net->gseq, reinterpret_cast<const float2*>(est),
                                                   reinterpret_cast<const float2*>(h_true), 1.f / (float)terms,
                                                   reinterpret_cast<uint4*>(net->dy), net->loss);
    rc = check_cuda(net->ctx, cudaGetLastError(), "le_loss_kernel launch");
  }
  if (rc == PG_OK) {
    rc = backward(net, R, s);
  }
  if (rc == PG_OK) {
    rc = pack_launch(net, 1, opt, s);
  }
  if (rc == PG_OK && loss != nullptr) {
    rc = check_cuda(net->ctx, cudaMemcpyAsync(loss, net->loss, 8, cudaMemcpyDeviceToDevice, s), "D2D loss");
  }
  return rc;
}

} // extern "C"

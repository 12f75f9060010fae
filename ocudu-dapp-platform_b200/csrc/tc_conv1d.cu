// 1-D convolution (kernel 5, 'same' padding) on the 5th-generation tensor cores: the layers of the
// learned channel estimator, forward and backward, as implicit GEMMs with tcgen05.mma (BF16
// operands from shared memory, FP32 accumulators in tensor memory).
//
// Activation layout: [C/8][R][8] bf16 - channel chunks of 8, each a column of R 16-byte rows
// (one row per resource element position of a batch of concatenated samples, with zero rows
// between samples). In this layout a row is a core-matrix row of the tensor cores' K-major
// no-swizzle operand format with 8-row groups 128 bytes apart, so row r of a chunk sits at
// r * 16 bytes. The five taps of the convolution are therefore the same shared-memory tile seen
// from five start addresses 16 bytes apart: no im2col copy.
//
//   forward:  Y[r][co] = sum_{t, ci} X[r + t - 2][ci] * W[co][ci][t]      (M = rows, N = co, K = 5 x ci)
//   input gradient: the same kernel with W'[ci][co][t] = W[co][ci][4 - t], plus a residual gradient and
//                   the ReLU mask of the forward activation in the epilogue
//   weight gradient: dW[t][ci][co] = sum_r X[r + t - 2][ci] * dY[r][co]   (M = (tap, ci), N = co, K = rows;
//                    both operands MN-major in the activation layout, the taps as row-shifted copies of
//                    the input tile)
//
// Every wait on an mbarrier has an iteration limit; on expiry the kernel records an error code,
// skips its epilogue, frees its tensor memory and returns.
#include "pg_internal.h"
#include "tc_common.cuh"

#include <cuda_bf16.h>

namespace {

using namespace pg::tc;

constexpr int kTapCount    = 5;
constexpr int kTileRows    = 128;
constexpr int kHaloRows    = kTileRows + kTapCount - 1; // 132
constexpr int kConvThreads = 128;

// True for the bf16 values of the 8 lanes of v that are > 0 (ReLU outputs: +0 or positive).
__device__ __forceinline__ void positive_mask(const uint4 v, bool* m)
{
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t lo = w[j] & 0xffffu, hi = w[j] >> 16;
    m[2 * j]     = lo - 1u < 0x7fffu;
    m[2 * j + 1] = hi - 1u < 0x7fffu;
  }
}

// Forward convolution over row tiles of 128 (persistent CTAs). CIN, COUT in {16, 64}.
// Epilogue: + bias (if bias != null), + residual (if res != null), ReLU (if relu), zero where the
// ReLU output `mask` (same layout as y) is not positive (if mask != null), stored as bf16 on valid
// rows.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv1d_fwd_kernel(const uint4* __restrict__ x, const uint4* __restrict__ w,
                                                                  const float* __restrict__ bias,
                                                                  const uint4* __restrict__ res,
                                                                  const uint4* __restrict__ mask, uint4* __restrict__ y,
                                                                  const uint8_t* __restrict__ row_valid, int R,
                                                                  int relu, int* __restrict__ err)
{
  constexpr int      kInChunks  = CIN / 8;
  constexpr uint32_t kXChunkB   = kHaloRows * 16;        // bytes per input chunk column in smem
  constexpr uint32_t kWTapB     = kInChunks * COUT * 16; // bytes per tap of packed weights
  constexpr uint32_t kCols      = tmem_cols<COUT>();
  extern __shared__ __align__(128) unsigned char smem[];
  uint4*              xs      = reinterpret_cast<uint4*>(smem);                          // [kInChunks][132]
  uint4*              ws      = reinterpret_cast<uint4*>(smem + kInChunks * kXChunkB);   // [5][kInChunks][COUT]
  uint64_t*           mbar    = reinterpret_cast<uint64_t*>(smem + kInChunks * kXChunkB + kTapCount * kWTapB);
  uint32_t*           tmem_sm = reinterpret_cast<uint32_t*>(mbar + 1);
  uint32_t*           ok_sm   = tmem_sm + 1;
  const int           tid     = threadIdx.x;
  const int           warp    = tid >> 5;

  // Weights once per CTA.
  for (int i = tid; i < kTapCount * kInChunks * COUT; i += kConvThreads) {
    ws[i] = w[i];
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_sm), kCols);
  }
  if (tid == 0) {
    mbar_init(smem_u32(mbar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem   = *tmem_sm;
  const uint32_t idesc  = make_idesc(kTileRows, COUT, false, false);
  const int      ntiles = (R + kTileRows - 1) / kTileRows;
  uint32_t       phase  = 0;
  bool           ok     = true;

  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int m0 = tile * kTileRows;
    // Input rows m0 - 2 .. m0 + 129 of every chunk (zero outside [0, R)).
    for (int i = tid; i < kInChunks * kHaloRows; i += kConvThreads) {
      const int c  = i / kHaloRows;
      const int rr = i - c * kHaloRows;
      const int gr = m0 + rr - 2;
      xs[i]        = (gr >= 0 && gr < R) ? x[(size_t)c * R + gr] : make_uint4(0, 0, 0, 0);
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t xb = smem_u32(xs);
      const uint32_t wb = smem_u32(ws);
      uint32_t       acc = 0;
#pragma unroll
      for (int t = 0; t < kTapCount; ++t) {
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
          const uint64_t ad = make_desc(xb + (uint32_t)(2 * kc) * kXChunkB + (uint32_t)t * 16u, kXChunkB, 128);
          const uint64_t bd = make_desc(wb + (uint32_t)t * kWTapB + (uint32_t)(2 * kc) * (COUT * 16), COUT * 16, 128);
          mma_bf16(tmem, ad, bd, idesc, acc);
          acc = 1;
        }
      }
      mma_commit(smem_u32(mbar));
    }
    // One thread waits (bounded) and publishes the outcome, so that every thread takes the same
    // path.
    if (tid == 0) {
      const bool done = mbar_wait_bounded(smem_u32(mbar), phase);
      *ok_sm          = done ? 1u : 0u;
      if (!done) {
        atomicExch(err, 1);
      }
    }
    phase ^= 1u;
    __syncthreads();
    tc_fence_after();
    ok = *ok_sm != 0;
    if (!ok) {
      break;
    }
    // Epilogue: thread = row (warp w holds TMEM lanes 32w .. 32w + 31).
    const int      r   = warp * 32 + (tid & 31);
    const int      gr  = m0 + r;
    const bool     st  = gr < R && row_valid[gr] != 0;
    const uint32_t tad = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int cc = 0; cc < COUT / 16; ++cc) {
      float v[16];
      tmem_ld16(tad + (uint32_t)(cc * 16), v);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int oc = 2 * cc + h; // output chunk of 8 channels
        float     o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          o[j] = v[8 * h + j] + (bias != nullptr ? bias[8 * oc + j] : 0.f);
        }
        if (st && res != nullptr) {
          const uint4          rv = res[(size_t)oc * R + gr];
          const __nv_bfloat16* rb = reinterpret_cast<const __nv_bfloat16*>(&rv);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            o[j] += __bfloat162float(rb[j]);
          }
        }
        if (relu) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            o[j] = fmaxf(o[j], 0.f);
          }
        }
        if (st && mask != nullptr) {
          bool m[8];
          positive_mask(mask[(size_t)oc * R + gr], m);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            o[j] = m[j] ? o[j] : 0.f;
          }
        }
        if (gr < R) {
          // Rows outside samples are written as zeros, so that a buffer reused with another row
          // layout keeps zero rows between its samples.
          uint4           pk = make_uint4(0, 0, 0, 0);
          __nv_bfloat162* pb = reinterpret_cast<__nv_bfloat162*>(&pk);
          if (st) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              pb[j] = __floats2bfloat162_rn(o[2 * j], o[2 * j + 1]);
            }
          }
          y[(size_t)oc * R + gr] = pk;
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  __syncthreads();
  if (warp == 0) {
    tmem_dealloc(tmem, kCols);
  }
}

// ---------------------------------------------------------------------------------------------
// Weight gradient. D[m][co] = sum_r A[m][r] * dY[r][co] over the K tiles (128 rows) of this CTA's
// row range, with m = (tap, ci): the input tile is staged as kCopies row-shifted copies
// (copy k holds X[r0 - 2 + k + j]), so that the 16 eight-channel groups of one M tile of 128 sit at
// a uniform stride; M tile j adds j * kCopies rows to the start address. CIN = 64: 2 copies, 3 M
// tiles (taps 0-1, 2-3, 4 and a discarded 5th); CIN = 16: 8 copies, 1 M tile (taps 0-4 and three
// discarded). Both operands are MN-major without swizzle (SBO = stride of the 8-element MN groups,
// LBO = stride of the 8-row K groups). Two smem stages: the loads of tile i + 1 overlap the MMAs of
// tile i. Epilogue: FP32 partial sums added to dw[t][ci][co] with vector atomics.
constexpr int kWgTile     = 128;
constexpr int kWgCopyRows = kWgTile + 8;

template <int CIN, int COUT>
struct wg_cfg {
  static constexpr int      kInChunks   = CIN / 8;
  static constexpr int      kCopies     = 16 / kInChunks;
  static constexpr int      kMTiles     = (kTapCount + kCopies - 1) / kCopies;
  static constexpr uint32_t kABytes     = 16u * kWgCopyRows * 16u;
  static constexpr uint32_t kBBytes     = (uint32_t)(COUT / 8) * kWgTile * 16u;
  static constexpr uint32_t kStageBytes = kABytes + kBBytes;
  static constexpr uint32_t kCols       = tmem_cols<kMTiles * COUT>();
  static constexpr size_t   kSmem       = 2 * (size_t)kStageBytes + 32;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv1d_wgrad_kernel(const uint4* __restrict__ x,
                                                                    const uint4* __restrict__ dy, int R,
                                                                    int tiles_per_cta, float* __restrict__ dw,
                                                                    int* __restrict__ err)
{
  using C = wg_cfg<CIN, COUT>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t*  mbar    = reinterpret_cast<uint64_t*>(smem + 2 * C::kStageBytes);
  uint32_t*  tmem_sm = reinterpret_cast<uint32_t*>(mbar + 2);
  uint32_t*  ok_sm   = tmem_sm + 1;
  const int  tid     = threadIdx.x;
  const int  warp    = tid >> 5;
  const int  ntiles  = (R + kWgTile - 1) / kWgTile;
  const int  t0      = blockIdx.x * tiles_per_cta;
  const int  nt      = min(ntiles, t0 + tiles_per_cta) - t0;
  if (nt <= 0) {
    return;
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_sm), C::kCols);
  }
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem  = *tmem_sm;
  const uint32_t idesc = make_idesc(kTileRows, COUT, true, true);
  const uint4    zero  = make_uint4(0, 0, 0, 0);
  bool           ok    = true;

  for (int i = 0; i < nt; ++i) {
    const int      st = i & 1;
    unsigned char* A  = smem + st * C::kStageBytes;
    unsigned char* B  = A + C::kABytes;
    if (i >= 2) {
      // The stage is free once the MMAs of tile i - 2 (commit number (i - 2) / 2 on its barrier)
      // have completed.
      if (tid == 0) {
        const bool done = mbar_wait_bounded(smem_u32(&mbar[st]), (uint32_t)((i - 2) >> 1) & 1u);
        *ok_sm          = done ? 1u : 0u;
        if (!done) {
          atomicExch(err, 1);
        }
      }
      __syncthreads();
      ok = *ok_sm != 0;
      if (!ok) {
        break;
      }
    }
    const int r0 = (t0 + i) * kWgTile;
    uint4*    As = reinterpret_cast<uint4*>(A);
    for (int q = tid; q < 16 * kWgCopyRows; q += kConvThreads) {
      const int g  = q / kWgCopyRows;
      const int j  = q - g * kWgCopyRows;
      const int k  = g / C::kInChunks;
      const int c  = g - k * C::kInChunks;
      const int gr = r0 - 2 + k + j;
      As[q]        = (gr >= 0 && gr < R) ? x[(size_t)c * R + gr] : zero;
    }
    uint4* Bs = reinterpret_cast<uint4*>(B);
    for (int q = tid; q < (COUT / 8) * kWgTile; q += kConvThreads) {
      const int c  = q / kWgTile;
      const int j  = q - c * kWgTile;
      const int gr = r0 + j;
      Bs[q]        = gr < R ? dy[(size_t)c * R + gr] : zero;
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t ab = smem_u32(A);
      const uint32_t bb = smem_u32(B);
#pragma unroll
      for (int ks = 0; ks < kWgTile / 16; ++ks) {
        const uint64_t bd = make_desc(bb + (uint32_t)ks * 256u, 128, kWgTile * 16);
#pragma unroll
        for (int j = 0; j < C::kMTiles; ++j) {
          const uint64_t ad =
              make_desc(ab + (uint32_t)(j * C::kCopies) * 16u + (uint32_t)ks * 256u, 128, kWgCopyRows * 16);
          mma_bf16(tmem + (uint32_t)(j * COUT), ad, bd, idesc, (i > 0 || ks > 0) ? 1u : 0u);
        }
      }
      mma_commit(smem_u32(&mbar[st]));
    }
  }
  if (ok) {
    const int last = nt - 1;
    if (tid == 0) {
      const bool done = mbar_wait_bounded(smem_u32(&mbar[last & 1]), (uint32_t)(last >> 1) & 1u);
      *ok_sm          = done ? 1u : 0u;
      if (!done) {
        atomicExch(err, 1);
      }
    }
    __syncthreads();
    tc_fence_after();
    ok = *ok_sm != 0;
  }
  if (ok) {
    // Thread = TMEM lane m of every M tile: group g = m / 8 (copy k, chunk c), lane e = m % 8.
    const int      m   = warp * 32 + (tid & 31);
    const int      g   = m >> 3;
    const int      k   = g / C::kInChunks;
    const int      ci  = 8 * (g - k * C::kInChunks) + (m & 7);
    const uint32_t tad = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int j = 0; j < C::kMTiles; ++j) {
      const int tap = j * C::kCopies + k;
#pragma unroll
      for (int cc = 0; cc < COUT / 16; ++cc) {
        float v[16];
        tmem_ld16(tad + (uint32_t)(j * COUT + cc * 16), v);
        if (tap < kTapCount) {
          float4* dst = reinterpret_cast<float4*>(dw + ((size_t)tap * CIN + ci) * COUT + cc * 16);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            atomicAdd(dst + q, make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tmem_dealloc(tmem, C::kCols);
  }
}

// Bias gradient db[co] += sum over rows of dY[r][co]: blockIdx.y = 8-channel chunk, grid-stride rows.
__global__ void conv1d_bias_grad_kernel(const uint4* __restrict__ dy, int R, float* __restrict__ db)
{
  __shared__ float part[8];
  const int c = blockIdx.y;
  if (threadIdx.x < 8) {
    part[threadIdx.x] = 0.f;
  }
  __syncthreads();
  float acc[8] = {};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const uint4           v = dy[(size_t)c * R + r];
    const __nv_bfloat16*  b = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j] += __bfloat162float(b[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float s = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&part[j], s);
    }
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    atomicAdd(&db[8 * c + threadIdx.x], part[threadIdx.x]);
  }
}

template <int CIN, int COUT>
size_t fwd_smem_bytes()
{
  return (size_t)(CIN / 8) * kHaloRows * 16 + (size_t)kTapCount * (CIN / 8) * COUT * 16 + 16;
}

template <int CIN, int COUT>
int fwd_setup()
{
  return cudaFuncSetAttribute(conv1d_fwd_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fwd_smem_bytes<CIN, COUT>()) == cudaSuccess
             ? PG_OK
             : PG_ERR_CUDA;
}

template <int CIN, int COUT>
int wg_setup()
{
  return cudaFuncSetAttribute(conv1d_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)wg_cfg<CIN, COUT>::kSmem) == cudaSuccess
             ? PG_OK
             : PG_ERR_CUDA;
}

template <int CIN, int COUT>
int fwd_launch(pg_context* ctx, const void* x, const void* w, const float* bias, const void* res, const void* mask,
               void* y, const uint8_t* row_valid, int R, int relu, int* err, cudaStream_t s)
{
  const int ntiles = (R + kTileRows - 1) / kTileRows;
  const int grid   = std::max(1, std::min(ntiles, ctx->sm_count * 2));
  conv1d_fwd_kernel<CIN, COUT><<<grid, kConvThreads, fwd_smem_bytes<CIN, COUT>(), s>>>(
      static_cast<const uint4*>(x), static_cast<const uint4*>(w), bias, static_cast<const uint4*>(res),
      static_cast<const uint4*>(mask), static_cast<uint4*>(y), row_valid, R, relu, err);
  return pg::check_cuda(ctx, cudaGetLastError(), "conv1d_fwd_kernel launch");
}

template <int CIN, int COUT>
int wg_launch(pg_context* ctx, const void* x, const void* dy, int R, float* dw, float* db, int* err, cudaStream_t s)
{
  const int ntiles = (R + kWgTile - 1) / kWgTile;
  // At least four K tiles per CTA (fewer partial sums to add), at most two CTAs per SM.
  const int per    = std::max(4, (ntiles + 2 * ctx->sm_count - 1) / (2 * ctx->sm_count));
  const int grid   = (ntiles + per - 1) / per;
  conv1d_wgrad_kernel<CIN, COUT><<<grid, kConvThreads, wg_cfg<CIN, COUT>::kSmem, s>>>(
      static_cast<const uint4*>(x), static_cast<const uint4*>(dy), R, per, dw, err);
  int rc = pg::check_cuda(ctx, cudaGetLastError(), "conv1d_wgrad_kernel launch");
  if (rc == PG_OK && db != nullptr) {
    const int bgrid = std::max(1, std::min((R + 255) / 256, ctx->sm_count));
    conv1d_bias_grad_kernel<<<dim3(bgrid, COUT / 8), 256, 0, s>>>(static_cast<const uint4*>(dy), R, db);
    rc = pg::check_cuda(ctx, cudaGetLastError(), "conv1d_bias_grad_kernel launch");
  }
  return rc;
}

} // namespace

namespace pg {

int conv_setup(pg_context* ctx)
{
  int rc = fwd_setup<16, 64>();
  if (rc == PG_OK) {
    rc = fwd_setup<64, 64>();
  }
  if (rc == PG_OK) {
    rc = fwd_setup<64, 16>();
  }
  if (rc == PG_OK) {
    rc = wg_setup<16, 64>();
  }
  if (rc == PG_OK) {
    rc = wg_setup<64, 64>();
  }
  if (rc == PG_OK) {
    rc = wg_setup<64, 16>();
  }
  if (rc != PG_OK) {
    (void)cudaGetLastError();
    return set_error(ctx, PG_ERR_CUDA, "cudaFuncSetAttribute(conv1d kernels)");
  }
  return PG_OK;
}

int conv_forward_launch(pg_context* ctx, int cin, int cout, const void* x, const void* w, const float* bias,
                        const void* res, const void* mask, void* y, const uint8_t* row_valid, int R, int relu,
                        int* err, cudaStream_t s)
{
  if (R <= 0) {
    return PG_OK;
  }
  if (cin == 16 && cout == 64) {
    return fwd_launch<16, 64>(ctx, x, w, bias, res, mask, y, row_valid, R, relu, err, s);
  }
  if (cin == 64 && cout == 64) {
    return fwd_launch<64, 64>(ctx, x, w, bias, res, mask, y, row_valid, R, relu, err, s);
  }
  if (cin == 64 && cout == 16) {
    return fwd_launch<64, 16>(ctx, x, w, bias, res, mask, y, row_valid, R, relu, err, s);
  }
  return set_error(ctx, PG_ERR_INVALID, "conv1d: channel counts must be (16,64), (64,64) or (64,16)");
}

int conv_wgrad_launch(pg_context* ctx, int cin, int cout, const void* x, const void* dy, int R, float* dw, float* db,
                      int* err, cudaStream_t s)
{
  if (R <= 0) {
    return PG_OK;
  }
  if (cin == 16 && cout == 64) {
    return wg_launch<16, 64>(ctx, x, dy, R, dw, db, err, s);
  }
  if (cin == 64 && cout == 64) {
    return wg_launch<64, 64>(ctx, x, dy, R, dw, db, err, s);
  }
  if (cin == 64 && cout == 16) {
    return wg_launch<64, 16>(ctx, x, dy, R, dw, db, err, s);
  }
  return set_error(ctx, PG_ERR_INVALID, "conv1d: channel counts must be (16,64), (64,64) or (64,16)");
}

} // namespace pg

extern "C" int pg_conv1d_forward_device(pg_context* ctx, int cin, int cout, const void* x, const void* w,
                                        const float* bias, const void* res, void* y, const uint8_t* row_valid, int rows,
                                        int relu, int* err, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (x == nullptr || w == nullptr || bias == nullptr || y == nullptr || row_valid == nullptr || err == nullptr ||
      rows < 0) {
    return pg::set_error(ctx, PG_ERR_INVALID, "conv1d: null buffer or negative row count");
  }
  return pg::conv_forward_launch(ctx, cin, cout, x, w, bias, res, nullptr, y, row_valid, rows, relu, err,
                                 static_cast<cudaStream_t>(stream));
}

extern "C" int pg_conv1d_backward_data_device(pg_context* ctx, int cin, int cout, const void* dy, const void* w_t,
                                              const void* res, const void* mask, void* dx, const uint8_t* row_valid,
                                              int rows, int* err, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (dy == nullptr || w_t == nullptr || dx == nullptr || row_valid == nullptr || err == nullptr || rows < 0) {
    return pg::set_error(ctx, PG_ERR_INVALID, "conv1d backward: null buffer or negative row count");
  }
  // The input gradient of a (cin -> cout) layer is a (cout -> cin) convolution.
  return pg::conv_forward_launch(ctx, cout, cin, dy, w_t, nullptr, res, mask, dx, row_valid, rows, 0, err,
                                 static_cast<cudaStream_t>(stream));
}

extern "C" int pg_conv1d_backward_weights_device(pg_context* ctx, int cin, int cout, const void* x, const void* dy,
                                                 int rows, float* dw, float* db, int* err, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (x == nullptr || dy == nullptr || dw == nullptr || err == nullptr || rows < 0) {
    return pg::set_error(ctx, PG_ERR_INVALID, "conv1d weight gradient: null buffer or negative row count");
  }
  return pg::conv_wgrad_launch(ctx, cin, cout, x, dy, rows, dw, db, err, static_cast<cudaStream_t>(stream));
}

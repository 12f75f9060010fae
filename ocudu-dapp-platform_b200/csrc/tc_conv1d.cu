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
//   input gradient: the same kernel with W'[ci][co][t] = W[co][ci][4 - t]
//   weight gradient: dW[co][ci][t] = sum_r dY[r][co] * X[r + t - 2][ci]   (M = co, N = ci, K = rows; both
//                    operands MN-major in the same activation layout)
//
// Every wait on an mbarrier has an iteration limit; on expiry the kernel records an error code,
// skips its epilogue, frees its tensor memory and returns.
#include "pg_internal.h"

#include <cuda_bf16.h>

namespace {

constexpr int      kTapCount     = 5;
constexpr int      kTileRows     = 128;
constexpr int      kHaloRows     = kTileRows + kTapCount - 1; // 132
constexpr int      kConvThreads  = 128;
constexpr uint32_t kWaitLimit    = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle (bits: start >> 4 [0,14), LBO >> 4 [16,30),
// SBO >> 4 [32,46), version 1 [46,48), layout type 0 [61,64)).
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3fffu);
  d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, majors, N >> 3 at bit 17, M >> 4 at 24.
__host__ __device__ constexpr uint32_t make_idesc(int m, int n, bool a_mn_major, bool b_mn_major)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: true when the phase completed, false when the limit expired.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity)
{
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    if (mbar_try_wait(mbar, parity)) {
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ void fence_async_shared()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = __uint_as_float(r[i]);
  }
}

template <int N>
__host__ __device__ constexpr uint32_t tmem_cols()
{
  return N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
}

// Forward convolution over row tiles of 128 (persistent CTAs). CIN, COUT in {16, 64}.
// Epilogue: + bias, + residual (if res != null), ReLU (if relu), stored as bf16 on valid rows.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv1d_fwd_kernel(const uint4* __restrict__ x, const uint4* __restrict__ w,
                                                                  const float* __restrict__ bias,
                                                                  const uint4* __restrict__ res, uint4* __restrict__ y,
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
          o[j] = v[8 * h + j] + bias[8 * oc + j];
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
        if (st) {
          uint4           pk;
          __nv_bfloat162* pb = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            pb[j] = __floats2bfloat162_rn(o[2 * j], o[2 * j + 1]);
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
int fwd_launch(pg_context* ctx, const void* x, const void* w, const float* bias, const void* res, void* y,
               const uint8_t* row_valid, int R, int relu, int* err, cudaStream_t s)
{
  const int ntiles = (R + kTileRows - 1) / kTileRows;
  const int grid   = std::max(1, std::min(ntiles, ctx->sm_count * 2));
  conv1d_fwd_kernel<CIN, COUT><<<grid, kConvThreads, fwd_smem_bytes<CIN, COUT>(), s>>>(
      static_cast<const uint4*>(x), static_cast<const uint4*>(w), bias, static_cast<const uint4*>(res),
      static_cast<uint4*>(y), row_valid, R, relu, err);
  return pg::check_cuda(ctx, cudaGetLastError(), "conv1d_fwd_kernel launch");
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
  if (rc != PG_OK) {
    (void)cudaGetLastError();
    return set_error(ctx, PG_ERR_CUDA, "cudaFuncSetAttribute(conv1d kernels)");
  }
  return PG_OK;
}

int conv_forward_launch(pg_context* ctx, int cin, int cout, const void* x, const void* w, const float* bias,
                        const void* res, void* y, const uint8_t* row_valid, int R, int relu, int* err, cudaStream_t s)
{
  if (R <= 0) {
    return PG_OK;
  }
  if (cin == 16 && cout == 64) {
    return fwd_launch<16, 64>(ctx, x, w, bias, res, y, row_valid, R, relu, err, s);
  }
  if (cin == 64 && cout == 64) {
    return fwd_launch<64, 64>(ctx, x, w, bias, res, y, row_valid, R, relu, err, s);
  }
  if (cin == 64 && cout == 16) {
    return fwd_launch<64, 16>(ctx, x, w, bias, res, y, row_valid, R, relu, err, s);
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
  return pg::conv_forward_launch(ctx, cin, cout, x, w, bias, res, y, row_valid, rows, relu, err,
                                 static_cast<cudaStream_t>(stream));
}

// Open Fronthaul block-floating-point (BFP) IQ decompression for sm_100a, writing the complex bf16
// resource grid the PUSCH path reads, so that the host hands over the compressed uplink U-plane
// payload (about 58 % of the grid's bytes at 9-bit width) instead of the grid.
//
// Format (O-RAN.WG4.CUS Annex A.1.2, as lib/ofh/compression/iq_compression_bfp_impl.cpp:89-141
// reads it): per PRB one exponent byte, then the 24 samples (I, Q of 12 subcarriers) of data_width
// bits each, packed big-endian. A sample is sign-extended from data_width bits and scaled by
// 2^exponent / (2^15 - 1); the value is rounded to bf16 (nearest, ties to even).
//
// Rounding of the scaling follows the reference's implementation for the width: for 9, 14 and 16
// bits its x86 vector decompressor (iq_compression_bfp_avx512.cpp:147-201) multiplies the sample by
// the float (2^e / 32767) - two roundings; for the other widths it falls back to the generic one,
// which divides the integer sample * 2^e by 32767 - one rounding. The kernel does the same per width.
//
// Mapping: one CTA per 128 PRBs (384 threads, four subcarriers each). The CTA's compressed bytes
// are a contiguous run of 128 * (1 + 3 * width) bytes, a multiple of 16, so they are staged into
// shared memory with 16-byte loads (byte loads when the buffer is not 16-byte aligned), all in
// flight before the barrier; each thread then reads its I and Q fields through a 32-bit big-endian
// window and writes complex bf16 words, coalesced across the CTA.
#include "pg_internal.h"

#include <cuda_bf16.h>

namespace {

constexpr int kBfpPrbs    = 128;
constexpr int kBfpThreads = 384; // each thread writes kBfpPrbs * 12 / 384 = 4 subcarriers
constexpr int kBfpMaxPrbBytes = 1 + 3 * 16;

__device__ __forceinline__ int bfp_field(const uint8_t* __restrict__ p, uint32_t bit, int w)
{
  const uint8_t* b      = p + (bit >> 3);
  const uint32_t window = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | (uint32_t)b[3];
  const uint32_t raw    = (window << (bit & 7u)) >> (32 - w);
  return (int)(raw << (32 - w)) >> (32 - w); // sign extension from w bits
}

__device__ __forceinline__ uint32_t bf16_bits(float v)
{
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v));
}

__global__ void __launch_bounds__(kBfpThreads) bfp_decompress_kernel(const uint8_t* __restrict__ in, uint32_t nof_prb,
                                                                   int w, int prb_bytes, int mul_path,
                                                                   uint32_t* __restrict__ out)
{
  __shared__ __align__(16) uint8_t s[kBfpPrbs * kBfpMaxPrbBytes + 16];
  const uint32_t p0 = blockIdx.x * kBfpPrbs;
  const uint32_t np = min((uint32_t)kBfpPrbs, nof_prb - p0);
  const uint8_t* src    = in + (size_t)p0 * prb_bytes;
  const uint32_t nbytes = np * (uint32_t)prb_bytes;
  const int      tid    = threadIdx.x;
  uint32_t       done   = 0;
  if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
    const uint32_t nv = nbytes / 16;
    for (uint32_t q = tid; q < nv; q += kBfpThreads) {
      reinterpret_cast<uint4*>(s)[q] = __ldg(reinterpret_cast<const uint4*>(src) + q);
    }
    done = nv * 16;
  }
  for (uint32_t q = done + tid; q < nbytes; q += kBfpThreads) {
    s[q] = __ldg(src + q);
  }
  if (tid < 16) {
    s[nbytes + tid] = 0; // the bytes a 32-bit window may read past the last field
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kBfpPrbs * 12 / kBfpThreads; ++j) {
    const uint32_t idx = (uint32_t)(tid + j * kBfpThreads);
    const uint32_t p = idx / 12u, k = idx - p * 12u;
    if (p >= np) {
      break;
    }
    const uint8_t* prb = s + p * (uint32_t)prb_bytes;
    const int      e   = prb[0] & 31;
    const int      re  = bfp_field(prb + 1, 2u * k * (uint32_t)w, w);
    const int      im  = bfp_field(prb + 1, (2u * k + 1u) * (uint32_t)w, w);
    float          fr, fi;
    if (mul_path) {
      const float scale = __fdiv_rn((float)(1 << e), 32767.0f);
      fr                = __fmul_rn((float)re, scale);
      fi                = __fmul_rn((float)im, scale);
    } else {
      const int scaler = (int)(int16_t)(1 << e); // the reference's int16_t scaling factor
      fr               = __fdiv_rn(__int2float_rn(re * scaler), 32767.0f);
      fi               = __fdiv_rn(__int2float_rn(im * scaler), 32767.0f);
    }
    out[(size_t)p0 * 12u + idx] = bf16_bits(fr) | (bf16_bits(fi) << 16);
  }
}

} // namespace

namespace pg {

int bfp_prb_bytes(int data_width)
{
  return 1 + 3 * data_width;
}

int bfp_decompress_launch(pg_context* ctx, const uint8_t* in, uint32_t nof_prb, int data_width, uint32_t* out,
                          cudaStream_t s)
{
  if (data_width < 1 || data_width > 16) {
    return set_error(ctx, PG_ERR_INVALID, "BFP data width must be 1 to 16 bits");
  }
  if (nof_prb == 0) {
    return PG_OK;
  }
  const int mul_path = (data_width == 9 || data_width == 14 || data_width == 16) ? 1 : 0;
  bfp_decompress_kernel<<<(nof_prb + kBfpPrbs - 1) / kBfpPrbs, kBfpThreads, 0, s>>>(
      in, nof_prb, data_width, bfp_prb_bytes(data_width), mul_path, out);
  return check_cuda(ctx, cudaGetLastError(), "bfp_decompress_kernel launch");
}

} // namespace pg

extern "C" {

int pg_bfp_prb_bytes(int data_width)
{
  return (data_width >= 1 && data_width <= 16) ? pg::bfp_prb_bytes(data_width) : -1;
}

int pg_bfp_decompress_device(pg_context* ctx, const uint8_t* compressed, uint32_t nof_prb, int data_width,
                             uint32_t* iq, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (nof_prb > 0 && (compressed == nullptr || iq == nullptr)) {
    return pg::set_error(ctx, PG_ERR_INVALID, "null device buffer");
  }
  cudaStream_t s         = static_cast<cudaStream_t>(stream);
  const unsigned int rec = pg::timing_record_flags(ctx, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, s, rec);
  }
  const int rc = pg::bfp_decompress_launch(ctx, compressed, nof_prb, data_width, iq, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, s, rec);
  }
  return rc;
}

} // extern "C"

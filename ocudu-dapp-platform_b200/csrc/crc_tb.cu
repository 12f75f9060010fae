// CRC over packed bit strings and transport-block assembly, bit-exact with the reference's
// crc_calculator::calculate (lib/phy/upper/channel_coding/crc_calculator_lut_impl.cpp:53-140,
// MSB first, zero initial value, no output XOR) and the TB join of pusch_decoder_impl
// (lib/phy/upper/channel_processors/pusch/pusch_decoder_impl.cpp:612-710: codeblock payloads
// concatenated, TB CRC checked over TBS + CRC bits).
//
// The CRC is linear, so the remainder of an L-bit message is the XOR over its 32-bit words of
// W(x) * x^e mod g(x), e = bits after the word plus the CRC order. Every thread folds one word:
// W mod g, times x^e mod g (from two tables: x^k and x^(1024k), k < 1024 / 2048) with a GF(2)
// multiply-and-reduce, then the CTA XOR-reduces. There is no sequential dependency on the
// message length.
#include "pg_internal.h"

namespace {

constexpr int kCrcThreads = 256;

__device__ __forceinline__ uint32_t gf2_reduce(uint64_t p, int top, uint32_t g, int order)
{
  // p has degree < top; returns p mod g (g includes the x^order term).
  for (int i = top - 1; i >= order; --i) {
    if ((p >> i) & 1ull) {
      p ^= (uint64_t)g << (i - order);
    }
  }
  return (uint32_t)p;
}

__device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b, uint32_t g, int order)
{
  uint64_t p = 0;
  for (int i = 0; i < order; ++i) {
    if ((b >> i) & 1u) {
      p ^= (uint64_t)a << i;
    }
  }
  return gf2_reduce(p, 2 * order - 1, g, order);
}

__device__ __forceinline__ uint32_t xpow(const uint32_t* tab, uint32_t e, uint32_t g, int order)
{
  const uint32_t* lo = tab;
  const uint32_t* hi = tab + 1024;
  return gf2_mulmod(__ldg(lo + (e & 1023u)), __ldg(hi + (e >> 10)), g, order);
}

// Up to 32 bits starting at bit `bit` of a packed MSB-first buffer, returned MSB aligned.
__device__ __forceinline__ uint32_t load_bits(const uint8_t* buf, uint32_t bit, int nbits)
{
  const uint8_t* p   = buf + (bit >> 3);
  const int      sh  = bit & 7;
  const int      nby = (sh + nbits + 7) >> 3;
  uint64_t       v   = 0;
  for (int b = 0; b < 5; ++b) {
    v = (v << 8) | (b < nby ? p[b] : 0u);
  }
  // v holds 40 bits; the wanted field starts at bit sh from the top.
  const uint32_t w = (uint32_t)(v >> (8 - sh));
  return nbits >= 32 ? w : (w & ~(0xffffffffu >> nbits));
}

__device__ __forceinline__ uint32_t word_contribution(uint32_t w, int valid, uint32_t e_lsb_full, const uint32_t* tab,
                                                      uint32_t g, int order)
{
  // valid bits at the top of w (1..32); their LSB sits at exponent e_lsb_full + (32 - valid).
  if (valid < 32) {
    w >>= (32 - valid);
  }
  const uint32_t e = e_lsb_full + (uint32_t)(32 - valid);
  if (w == 0) {
    return 0;
  }
  const uint32_t wm = gf2_reduce(w, 32, g, order);
  return gf2_mulmod(wm, xpow(tab, e, g, order), g, order);
}

__device__ __forceinline__ uint32_t block_xor(uint32_t v, uint32_t* red)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v ^= __shfl_xor_sync(0xffffffffu, v, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = v;
  }
  __syncthreads();
  uint32_t t = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      t ^= red[i];
    }
  }
  return t;
}

__global__ void __launch_bounds__(kCrcThreads) crc_kernel(const pg_crc_item* __restrict__ items,
                                                          const uint8_t* __restrict__ data,
                                                          uint32_t* __restrict__ out,
                                                          const uint32_t* __restrict__ tabs)
{
  __shared__ uint32_t red[kCrcThreads / 32];
  const pg_crc_item   it = items[blockIdx.x];
  uint32_t            g;
  int                 order;
  pg::crc_poly_params(it.poly, &g, &order);
  const uint32_t* tab = tabs + (size_t)it.poly * (1024 + 2048);
  const uint32_t  L   = it.nof_bits;
  uint32_t        acc = 0;
  for (uint32_t w = threadIdx.x; 32u * w < L; w += kCrcThreads) {
    const int      valid = (int)min(32u, L - 32u * w);
    const uint32_t bits  = load_bits(data, it.bit_offset + 32u * w, valid);
    // Exponent of bit 31 (LSB) of a full word at this position.
    const uint32_t e_lsb = L - 32u * w - (uint32_t)valid + (uint32_t)order - (uint32_t)(32 - valid);
    acc ^= word_contribution(bits, valid, e_lsb, tab, g, order);
  }
  const uint32_t crc = block_xor(acc, red);
  if (threadIdx.x == 0) {
    out[blockIdx.x] = crc;
  }
}

// Transport-block assembly and TB CRC, split into chunks of kTbChunkWords 32-bit words so that a
// large TB is spread over many CTAs (grid.x = TB, grid.y strides over its chunks). Each thread
// gathers kTbWordsPerThread words of the TB from the codeblock payloads, stores them, and folds
// its bytes with a byte-wise table (Sarwate) into the remainder of its piece alone; the piece's
// contribution to the TB remainder is that value times x^(bits after the piece) mod g, and the
// contributions meet by XOR (the CRC is linear) in tb_crc, which starts at zero.
constexpr int kTbWordsPerThread = 4;
constexpr int kTbChunkWords     = kCrcThreads * kTbWordsPerThread;
constexpr int kTbGridY          = 16; // CTAs per TB: up to 16 chunks (512 Kbit) run in parallel

__global__ void __launch_bounds__(kCrcThreads) tb_assemble_kernel(const pg_tb_desc* __restrict__ tbs,
                                                                  const uint8_t* __restrict__ cb_bits,
                                                                  const uint32_t* __restrict__ cb_bit_offsets,
                                                                  uint8_t* __restrict__ tb_out,
                                                                  uint32_t* __restrict__ tb_crc,
                                                                  const uint32_t* __restrict__ tabs,
                                                                  const uint32_t* __restrict__ chunks)
{
  __shared__ uint32_t byte_tab[256];
  __shared__ uint32_t red[kCrcThreads / 32];
  // The TB and the chunks of this CTA: one chunk of a chunk list (TB | chunk << 16), or chunks
  // blockIdx.y, blockIdx.y + gridDim.y, ... of TB blockIdx.x.
  const uint32_t   item        = chunks != nullptr ? chunks[blockIdx.x] : 0u;
  const uint32_t   tb          = chunks != nullptr ? (item & 0xffffu) : blockIdx.x;
  const uint32_t   chunk_first = chunks != nullptr ? (item >> 16) : blockIdx.y;
  const uint32_t   chunk_step  = chunks != nullptr ? 0xffffu : gridDim.y;
  const pg_tb_desc d           = tbs[tb];
  if (chunk_first * (uint64_t)kTbChunkWords * 32u >= (uint64_t)d.cb_payload_bits * d.nof_cbs) {
    return; // no chunk of this TB for this CTA (the whole CTA leaves: no barrier is pending)
  }
  uint32_t            g;
  int                 order;
  pg::crc_poly_params(d.crc_poly, &g, &order);
  const uint32_t mask = (1u << order) - 1u;
  {
    // Remainder register after one byte i entered an all-zero register (MSB first).
    uint32_t c = (uint32_t)threadIdx.x << (order - 8);
    for (int k = 0; k < 8; ++k) {
      c = ((c >> (order - 1)) & 1u) ? (((c << 1) ^ g) & mask) : ((c << 1) & mask);
    }
    byte_tab[threadIdx.x] = c;
  }
  __syncthreads();
  const uint32_t* tab      = tabs + (size_t)d.crc_poly * (1024 + 2048);
  const uint32_t  P        = d.cb_payload_bits;
  const uint32_t  L        = P * d.nof_cbs; // TBS + TB CRC bits, a multiple of 8
  const uint32_t  words    = (L + 31) / 32;
  uint8_t*        out      = tb_out + d.tb_out_offset;
  const uint32_t  tb_bytes = d.tbs_bits / 8;
  for (uint32_t chunk = chunk_first; chunk * kTbChunkWords < words; chunk += chunk_step) {
    const uint32_t w0  = chunk * kTbChunkWords + threadIdx.x * kTbWordsPerThread;
    uint32_t       rem = 0;
    uint32_t       end_bit = 0;
#pragma unroll
    for (int k = 0; k < kTbWordsPerThread; ++k) {
      const uint32_t w = w0 + (uint32_t)k;
      if (w >= words) {
        break;
      }
      const uint32_t i0    = 32u * w;
      const int      valid = (int)min(32u, L - i0);
      // Gather the word from at most two codeblock payloads.
      const uint32_t c0   = i0 / P;
      const uint32_t o0   = i0 - c0 * P;
      const int      n0   = (int)min((uint32_t)valid, P - o0);
      uint32_t       bits = load_bits(cb_bits, cb_bit_offsets[d.cb_first + c0] + o0, n0);
      if (n0 < valid) {
        const uint32_t rest = load_bits(cb_bits, cb_bit_offsets[d.cb_first + c0 + 1], valid - n0);
        bits |= rest >> n0;
      }
      for (int b = 0; b < valid / 8; ++b) {
        const uint32_t byte = 4u * w + (uint32_t)b;
        const uint32_t v    = (bits >> (24 - 8 * b)) & 0xffu;
        if (byte < tb_bytes) {
          out[byte] = (uint8_t)v;
        }
        rem = ((rem << 8) & mask) ^ byte_tab[((rem >> (order - 8)) ^ v) & 0xffu];
      }
      end_bit = i0 + (uint32_t)valid;
    }
    uint32_t contrib = 0;
    if (end_bit != 0 && rem != 0) {
      contrib = gf2_mulmod(rem, xpow(tab, L - end_bit, g, order), g, order);
    }
    const uint32_t part = block_xor(contrib, red);
    if (threadIdx.x == 0 && part != 0) {
      atomicXor(tb_crc + tb, part);
    }
    __syncthreads();
  }
}

} // namespace

namespace pg {

void crc_tables_host(uint32_t* tab /* 3 * 3072 */)
{
  for (int p = 0; p < 3; ++p) {
    uint32_t g;
    int      order;
    crc_poly_params(p, &g, &order);
    const uint32_t mask = (1u << order) - 1u;
    uint32_t*      lo   = tab + (size_t)p * 3072;
    uint32_t*      hi   = lo + 1024;
    uint32_t       x    = 1;
    // x^k for k < 1024 and x^(1024k) for k < 2048.
    uint32_t step = 0;
    for (int k = 0; k < 1024; ++k) {
      lo[k] = x;
      const uint32_t top = (x >> (order - 1)) & 1u;
      x                  = (x << 1) & mask;
      if (top) {
        x ^= g & mask;
      }
    }
    step = x; // x^1024 mod g
    auto mulmod = [&](uint32_t a, uint32_t b) {
      uint64_t pr = 0;
      for (int i = 0; i < order; ++i) {
        if ((b >> i) & 1u) {
          pr ^= (uint64_t)a << i;
        }
      }
      for (int i = 2 * order - 2; i >= order; --i) {
        if ((pr >> i) & 1ull) {
          pr ^= (uint64_t)g << (i - order);
        }
      }
      return (uint32_t)pr;
    };
    uint32_t acc = 1;
    for (int k = 0; k < 2048; ++k) {
      hi[k] = acc;
      acc   = mulmod(acc, step);
    }
  }
}

int crc_launch(pg_context* ctx, const pg_crc_item* items_dev, int n, const uint8_t* data, uint32_t* out,
               cudaStream_t stream)
{
  if (n == 0) {
    return PG_OK;
  }
  crc_kernel<<<n, kCrcThreads, 0, stream>>>(items_dev, data, out, ctx->dev.crc_tabs);
  return check_cuda(ctx, cudaGetLastError(), "crc_kernel launch");
}

int tb_assemble_launch(pg_context* ctx, const pg_tb_desc* tbs_dev, int n, const uint8_t* cb_bits,
                       const uint32_t* cb_bit_offsets, uint8_t* tb_out, uint32_t* tb_crc, cudaStream_t stream,
                       const uint32_t* chunks_dev, int nof_chunks)
{
  if (n == 0) {
    return PG_OK;
  }
  if (int rc = check_cuda(ctx, cudaMemsetAsync(tb_crc, 0, (size_t)n * sizeof(uint32_t), stream),
                          "cudaMemsetAsync(tb crc)")) {
    return rc;
  }
  if (chunks_dev != nullptr) {
    if (nof_chunks > 0) {
      tb_assemble_kernel<<<nof_chunks, kCrcThreads, 0, stream>>>(tbs_dev, cb_bits, cb_bit_offsets, tb_out, tb_crc,
                                                                 ctx->dev.crc_tabs, chunks_dev);
    }
  } else {
    tb_assemble_kernel<<<dim3(n, kTbGridY), kCrcThreads, 0, stream>>>(tbs_dev, cb_bits, cb_bit_offsets, tb_out, tb_crc,
                                                                       ctx->dev.crc_tabs, nullptr);
  }
  return check_cuda(ctx, cudaGetLastError(), "tb_assemble_kernel launch");
}

void tb_chunk_list(const pg_tb_desc* tbs, int n, std::vector<uint32_t>& out)
{
  out.clear();
  for (int t = 0; t < n; ++t) {
    const uint64_t bits   = (uint64_t)tbs[t].cb_payload_bits * tbs[t].nof_cbs;
    const uint64_t words  = (bits + 31) / 32;
    const uint64_t nchunk = (words + kTbChunkWords - 1) / kTbChunkWords;
    for (uint64_t c = 0; c < nchunk; ++c) {
      out.push_back((uint32_t)t | ((uint32_t)c << 16));
    }
  }
}

} // namespace pg

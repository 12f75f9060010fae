// Batched LDPC rate dematching (TS 38.212 Section 5.4.2), bit-exact with the reference's
// ldpc_rate_dematcher (lib/phy/upper/channel_coding/ldpc/ldpc_rate_dematcher_impl.cpp:29-250) on
// finite LLRs.
//
// The reference walks the E received LLRs sequentially through the circular buffer: bit
// de-interleaving (out[K*j + i] = in[i*Qm + j]), then placement from k0 onward, skipping the
// filler positions, wrapping at N_cb and combining wrapped values with the saturating LLR sum.
// Here every output position is computed independently: the valid (non-filler) positions form a
// cycle of length V = N_cb - F; position p with valid index v receives the de-interleaved inputs
// t = (v - v0) mod V, t + V, t + 2V, ... < E, summed in that order onto 0 (new data) or onto the
// previous buffer content (soft combining). Filler positions hold +127; positions at or beyond N_cb
// are zeroed on new data and untouched otherwise. kRmGridY CTAs per codeblock. Without repetition
// (E <= V, the usual case) the kernel reads the input in coalesced tiles and transposes them through
// shared memory; with repetition every output position is computed independently.
#include "pg_internal.h"

#include <algorithm>

namespace {

constexpr int kRmThreads = 256;
constexpr int kRmGridY   = 8;

__device__ __forceinline__ int llr_sum(int a, int b)
{
  // log_likelihood_ratio::operator+ (lib/phy/upper/log_likelihood_ratio.cpp:21-53).
  if (a == -b) {
    return 0;
  }
  if (a == 127 || a == -127) {
    return a;
  }
  if (b == 127 || b == -127) {
    return b;
  }
  return max(-120, min(120, a + b));
}

// Rows of the de-interleaver matrix per tile of the transposing path: a tile reads rows*Qm <= 2 KB
// of input.
constexpr int kRmTileRows = 256;
constexpr int kRmRepBatch = 4; // repetitions whose loads a thread issues together

__global__ void __launch_bounds__(kRmThreads) rate_dematch_kernel(const pg_rm_cb* __restrict__ cbs,
                                                                  const int8_t* __restrict__ in_all,
                                                                  int8_t* __restrict__ out_all,
                                                                  const uint32_t* __restrict__ list)
{
  __shared__ int8_t tile[kRmTileRows * 8];
  const pg_rm_cb d   = cbs[list != nullptr ? list[blockIdx.x] : blockIdx.x];
  const int      bg  = d.base_graph;
  const int      Z   = d.lifting_size;
  const int      Kb  = bg == 1 ? 22 : 10;
  const int      N   = (bg == 1 ? 66 : 50) * Z;
  const int      Ncb = (d.nref > 0 && (int)d.nref < N) ? (int)d.nref : N;
  const int      F   = d.nof_filler_bits;
  const int      sys = (Kb - 2) * Z;
  const int      inf = sys - F;
  const int      E   = (int)d.rm_length;
  const int      Qm  = d.modulation_order;
  const int      Kq  = E / Qm;
  const int      sh  = bg == 1 ? (d.rv == 0 ? 0 : d.rv == 1 ? 17 : d.rv == 2 ? 33 : 56)
                               : (d.rv == 0 ? 0 : d.rv == 1 ? 13 : d.rv == 2 ? 25 : 43);
  const int      k0  = (int)(((long long)sh * Ncb) / N) * Z;
  const int      V   = Ncb - F;
  const int      v0  = k0 < inf ? k0 : (k0 < sys ? inf : k0 - F);
  const int8_t*  in  = in_all + d.in_offset;
  int8_t*        out = out_all + d.out_offset;
  const bool     nd  = d.new_data != 0;

  if (E <= V) {
    // No repetition: each buffer position receives at most one input. The input, row i holding
    // the Qm LLRs of de-interleaver column i, is read a tile of rows at a time (coalesced) and
    // transposed through shared memory; bit plane j of rows i0.. lands on consecutive buffer
    // positions (t = j Kq + i, valid index (v0 + t) mod V, past the fillers), so the stores are
    // coalesced too. Positions no input reaches are written by the per-position loop below.
    const int ntiles = (Kq + kRmTileRows - 1) / kRmTileRows;
    for (int tl = blockIdx.y; tl < ntiles; tl += gridDim.y) {
      const int i0   = tl * kRmTileRows;
      const int rows = min(kRmTileRows, Kq - i0);
      __syncthreads();
      for (int k = threadIdx.x; k < rows * Qm; k += kRmThreads) {
        tile[k] = in[i0 * Qm + k];
      }
      __syncthreads();
      for (int k = threadIdx.x; k < rows * Qm; k += kRmThreads) {
        const int j = k / rows;
        const int i = k - j * rows;
        const int t = j * Kq + i0 + i;
        int       v = v0 + t;
        v           = v >= V ? v - V : v;
        const int p = v < inf ? v : v + F;
        const int x = tile[i * Qm + j];
        out[p]      = (int8_t)llr_sum(nd ? 0 : (int)out[p], x);
      }
    }
    for (int p = blockIdx.y * kRmThreads + threadIdx.x; p < N; p += gridDim.y * kRmThreads) {
      if (p >= inf && p < sys) {
        out[p] = 127;
        continue;
      }
      if (p >= Ncb) {
        if (nd) {
          out[p] = 0;
        }
        continue;
      }
      const int v = p < inf ? p : p - F;
      int       t = v - v0;
      t           = t < 0 ? t + V : t;
      if (t >= E && nd) {
        out[p] = 0;
      }
    }
    return;
  }

  // Repetition (E > V): position p receives t, t + V, ... in that order. De-interleaver index
  // src = (t mod Kq) * Qm + t div Kq with the quotient from a float reciprocal, corrected to the
  // exact value (t < 2^24).
  const float inv_kq = 1.0f / (float)(Kq > 0 ? Kq : 1);
  for (int p = blockIdx.y * kRmThreads + threadIdx.x; p < N; p += gridDim.y * kRmThreads) {
    if (p >= inf && p < sys) {
      out[p] = 127;
      continue;
    }
    if (p >= Ncb) {
      if (nd) {
        out[p] = 0;
      }
      continue;
    }
    const int v   = p < inf ? p : p - F;
    int       t   = v - v0;
    t             = t < 0 ? t + V : t;
    int       acc = nd ? 0 : (int)out[p];
    // Four repetitions per step: their loads are issued together, the sums taken in order.
    for (; t < E; t += kRmRepBatch * V) {
      int x[kRmRepBatch];
#pragma unroll
      for (int u = 0; u < kRmRepBatch; ++u) {
        const int tu = t + u * V;
        int       src = tu;
        if (Qm > 1) {
          int q = __float2int_rz((float)tu * inv_kq);
          int r = tu - q * Kq;
          if (r < 0) {
            --q;
            r += Kq;
          } else if (r >= Kq) {
            ++q;
            r -= Kq;
          }
          src = r * Qm + q;
        }
        x[u] = tu < E ? (int)in[src] : 0;
      }
#pragma unroll
      for (int u = 0; u < kRmRepBatch; ++u) {
        if (t + u * V < E) {
          acc = llr_sum(acc, x[u]);
        }
      }
    }
    out[p] = (int8_t)acc;
  }
}

// The circular buffers of the codeblocks whose LLRs the demodulator stores in place (placed[c]
// = 1: new data, E <= V), before it does: +127 at the filler positions [inf, (Kb - 2) Z) and 0
// everywhere else, which is what rate dematching leaves at every position that no LLR reaches.
// 16-byte stores; the first and last bytes of a buffer that does not start or end on a 16-byte
// boundary are stored one by one.
__global__ void __launch_bounds__(kRmThreads) rm_prefill_kernel(const pg_rm_cb* __restrict__ cbs,
                                                                const uint8_t* __restrict__ placed,
                                                                int8_t* __restrict__ out_all)
{
  if (placed[blockIdx.x] == 0) {
    return;
  }
  const pg_rm_cb d    = cbs[blockIdx.x];
  const int      Z    = d.lifting_size;
  const int      N    = (d.base_graph == 1 ? 66 : 50) * Z;
  const int      sys  = ((d.base_graph == 1 ? 22 : 10) - 2) * Z;
  const int      inf  = sys - (int)d.nof_filler_bits;
  int8_t*        out  = out_all + d.out_offset;
  const int      head = min(N, (int)((16u - (unsigned)(reinterpret_cast<uintptr_t>(out) & 15u)) & 15u));
  const int      nch  = (N - head) / 16;
  const int      tail = head + 16 * nch;
  const int      tid  = blockIdx.y * kRmThreads + threadIdx.x;
  const int      nthr = gridDim.y * kRmThreads;
  auto value = [&](int p) { return (int8_t)((p >= inf && p < sys) ? 127 : 0); };
  if (tid < head) {
    out[tid] = value(tid);
  }
  if (tail + tid < N) {
    out[tail + tid] = value(tail + tid);
  }
  for (int q = tid; q < nch; q += nthr) {
    const int c   = head + 16 * q;
    const int fil = max(0, min(c + 16, sys) - max(c, inf));
    uint4     w   = make_uint4(0u, 0u, 0u, 0u);
    if (fil == 16) {
      w = make_uint4(0x7f7f7f7fu, 0x7f7f7f7fu, 0x7f7f7f7fu, 0x7f7f7f7fu);
    } else if (fil > 0) {
      int8_t* b = reinterpret_cast<int8_t*>(&w);
      for (int i = 0; i < 16; ++i) {
        b[i] = value(c + i);
      }
    }
    *reinterpret_cast<uint4*>(out + c) = w;
  }
}

} // namespace

namespace pg {

int validate_rm_descs(pg_context* ctx, const pg_rm_cb* cbs, int n, size_t in_total, size_t out_total)
{
  if (n < 0 || (n > 0 && cbs == nullptr)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid codeblock list");
  }
  if (n > ctx->max_codeblocks) {
    return set_error(ctx, PG_ERR_CAPACITY, "rate-dematch batch exceeds max_codeblocks");
  }
  for (int i = 0; i < n; ++i) {
    const pg_rm_cb& d = cbs[i];
    char            buf[160];
    const int       qm = d.modulation_order;
    if ((d.base_graph != 1 && d.base_graph != 2) || lifting_set_index(d.lifting_size) < 0 || d.rv > 3 ||
        !(qm == 1 || qm == 2 || qm == 4 || qm == 6 || qm == 8)) {
      snprintf(buf, sizeof(buf), "codeblock %d: invalid base graph, lifting size, rv or modulation", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    const int Z   = d.lifting_size;
    const int N   = nshort_of(d.base_graph) * Z;
    const int sys = (kb_of(d.base_graph) - 2) * Z;
    const int Ncb = (d.nref > 0 && (int)d.nref < N) ? (int)d.nref : N;
    if ((int)d.nof_filler_bits >= sys || Ncb <= sys) {
      snprintf(buf, sizeof(buf), "codeblock %d: filler bits or N_ref out of range", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (d.rm_length % qm != 0) {
      snprintf(buf, sizeof(buf), "codeblock %d: E=%u not a multiple of Qm=%d", i, d.rm_length, qm);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (in_total != 0 && (size_t)d.in_offset + d.rm_length > in_total) {
      snprintf(buf, sizeof(buf), "codeblock %d: input beyond the buffer", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (out_total != 0 && (size_t)d.out_offset + (size_t)N > out_total) {
      snprintf(buf, sizeof(buf), "codeblock %d: output beyond the buffer", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
  }
  return PG_OK;
}

int rate_dematch_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const int8_t* in, int8_t* out,
                        cudaStream_t stream)
{
  return rate_dematch_launch(ctx, descs_dev, n, in, out, stream, kRmGridY);
}

int rate_dematch_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const int8_t* in, int8_t* out,
                        cudaStream_t stream, int ctas_per_cb, const uint32_t* list)
{
  if (n == 0) {
    return PG_OK;
  }
  // Each codeblock's N <= 25,344 output positions spread over ctas_per_cb CTAs.
  ctas_per_cb = std::max(1, std::min(32, ctas_per_cb));
  rate_dematch_kernel<<<dim3(n, ctas_per_cb), kRmThreads, 0, stream>>>(descs_dev, in, out, list);
  return check_cuda(ctx, cudaGetLastError(), "rate_dematch_kernel launch");
}

int rm_prefill_launch(pg_context* ctx, const pg_rm_cb* descs_dev, int n, const uint8_t* placed, int8_t* out,
                      cudaStream_t stream)
{
  if (n == 0) {
    return PG_OK;
  }
  // N <= 25,344 bytes = 1,584 chunks: two CTAs of 256 threads per codeblock, about three stores each.
  rm_prefill_kernel<<<dim3(n, 2), kRmThreads, 0, stream>>>(descs_dev, placed, out);
  return check_cuda(ctx, cudaGetLastError(), "rm_prefill_kernel launch");
}

} // namespace pg

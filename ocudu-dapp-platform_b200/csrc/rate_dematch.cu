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

__global__ void __launch_bounds__(kRmThreads) rate_dematch_kernel(const pg_rm_cb* __restrict__ cbs,
                                                                  const int8_t* __restrict__ in_all,
                                                                  int8_t* __restrict__ out_all,
                                                                  const uint8_t* __restrict__ fill_only)
{
  __shared__ int8_t tile[kRmTileRows * 8];
  const pg_rm_cb d   = cbs[blockIdx.x];
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

  if (E <= V && fill_only != nullptr && fill_only[blockIdx.x] != 0) {
    // One CTA per codeblock suffices for this fill (at most N / 16 chunks); the others leave.
    if (blockIdx.y != 0) {
      return;
    }
    // The demodulator placed this codeblock's LLRs itself (new data, E <= V): they occupy the valid
    // indices [v0, v0 + E) mod V, up to four position intervals past the fillers. Every other
    // position is a filler (+127) or unreached / beyond N_cb (0). The buffer is written in 16-byte
    // chunks: chunks of placed LLRs only are skipped, chunks without any are stored whole, and the
    // few chunks that mix them are merged byte by byte.
    int       ka[4], kb[4], nk = 0;
    const int e_end = v0 + E;
    auto add_v = [&](int a, int b) {
      const int b1 = min(b, inf);
      if (a < b1) {
        ka[nk] = a;
        kb[nk] = b1;
        ++nk;
      }
      const int a2 = max(a, inf);
      if (a2 < b) {
        ka[nk] = a2 + F;
        kb[nk] = b + F;
        ++nk;
      }
    };
    if (e_end <= V) {
      add_v(v0, e_end);
    } else {
      add_v(v0, V);
      add_v(0, e_end - V);
    }
    auto placed_at = [&](int p) {
      bool k = false;
      for (int i = 0; i < nk; ++i) {
        k |= p >= ka[i] && p < kb[i];
      }
      return k;
    };
    auto fill_value = [&](int p) { return (int8_t)((p >= inf && p < sys) ? 127 : 0); };
    const int head  = (int)((16u - (unsigned)(reinterpret_cast<uintptr_t>(out) & 15u)) & 15u);
    const int first = min(head, N);
    const int nch   = (N - first) / 16;
    const int tail  = first + 16 * nch;
    for (int p = threadIdx.x; p < first; p += kRmThreads) {
      if (!placed_at(p)) {
        out[p] = fill_value(p);
      }
    }
    for (int p = tail + threadIdx.x; p < N; p += kRmThreads) {
      if (!placed_at(p)) {
        out[p] = fill_value(p);
      }
    }
    for (int q = threadIdx.x; q < nch; q += kRmThreads) {
      const int c = first + 16 * q;
      int       kept = 0;
      for (int i = 0; i < nk; ++i) {
        kept += max(0, min(c + 16, kb[i]) - max(c, ka[i]));
      }
      if (kept == 16) {
        continue;
      }
      const int fil = max(0, min(c + 16, sys) - max(c, inf));
      uint4*    dst = reinterpret_cast<uint4*>(out + c);
      if (kept == 0 && fil == 0) {
        *dst = make_uint4(0u, 0u, 0u, 0u);
      } else if (kept == 0 && fil == 16) {
        *dst = make_uint4(0x7f7f7f7fu, 0x7f7f7f7fu, 0x7f7f7f7fu, 0x7f7f7f7fu);
      } else {
        uint4   w = *dst;
        int8_t* b = reinterpret_cast<int8_t*>(&w);
        for (int i = 0; i < 16; ++i) {
          if (!placed_at(c + i)) {
            b[i] = fill_value(c + i);
          }
        }
        *dst = w;
      }
    }
    return;
  }
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
    for (; t < E; t += V) {
      int src = t;
      if (Qm > 1) {
        int q = __float2int_rz((float)t * inv_kq);
        int r = t - q * Kq;
        if (r < 0) {
          --q;
          r += Kq;
        } else if (r >= Kq) {
          ++q;
          r -= Kq;
        }
        src = r * Qm + q;
      }
      acc = llr_sum(acc, in[src]);
    }
    out[p] = (int8_t)acc;
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
                        cudaStream_t stream, int ctas_per_cb, const uint8_t* fill_only)
{
  if (n == 0) {
    return PG_OK;
  }
  // Each codeblock's N <= 25,344 output positions spread over ctas_per_cb CTAs.
  ctas_per_cb = std::max(1, std::min(32, ctas_per_cb));
  rate_dematch_kernel<<<dim3(n, ctas_per_cb), kRmThreads, 0, stream>>>(descs_dev, in, out, fill_only);
  return check_cuda(ctx, cudaGetLastError(), "rate_dematch_kernel launch");
}

} // namespace pg

// Batched LDPC decoder for sm_100a: layered normalised min-sum on int8 messages, bit-exact with
// the reference's ldpc_decoder_avx512 / ldpc_decoder_avx2
// (lib/phy/upper/channel_coding/ldpc/ldpc_decoder_impl.cpp:41-306,
//  lib/phy/upper/channel_coding/ldpc/ldpc_decoder_avx512.cpp:69-253).
//
// Mapping: one CTA per codeblock, one thread per lifted check lane j (0 <= j < Z). For base-graph
// row r, edge e (variable node v_e, lifted shift s_e), lane j reads soft bit (v_e, (j+s_e) mod Z):
// the rows of a layer touch every lifted variable lane exactly once, so the Z lanes of a row are
// independent and one __syncthreads separates consecutive rows (the layer schedule). Soft bits
// live in shared memory; check-to-variable messages live in a per-codeblock global scratch slab
// (edge-major, lane-minor: coalesced, L2 resident), indexed by (edge, check lane) rather than
// the reference's rotated-back (variable slot, variable lane): the stored values are identical.
//
// Arithmetic, per lane and edge (all exactly as the reference's AVX-512 kernels):
//   v2c = soft == +-127 ? soft : clamp(soft - c2v, -120, 120)
//   min1/min2 over |v2c| starting at 120 (first minimum wins), sign = xor of v2c signs
//   scale: m -> (m * 52428) >> 16     (floor(0.8 * 2^16) = 52428; m <= 120 always)
//   c2v  = (sign xor sign(v2c)) ? -mag : mag,  mag = |v2c| == min1 ? scale(min2) : scale(min1)
//          (equivalent to the reference's index test: a tie at min1 implies min1 == min2)
//   soft = |v2c| == 127 ? v2c : promote(c2v + v2c) with |sum| > 120 -> +-127
// After each iteration: hard bits (soft <= 0), fail if any soft bit is 0, else CRC over the
// K*Z - F significant bits; CRC == 0 stops with iterations = it + 1.
#include "pg_internal.h"

#include <cuda_fp16.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace pg {
#include "ldpc_base_graphs.inc"
} // namespace pg

namespace {

constexpr int kThreads = 384;

__constant__ uint8_t  c_edge_col[2][pg::kBg1Edges];
__constant__ uint16_t c_edge_v[2][pg::kBg1Edges][8];
__constant__ uint8_t  c_row_deg[2][pg::kBg1Rows];
// Layer steps: runs of consecutive base-graph rows whose columns are pairwise disjoint. The rows of
// a step touch disjoint soft bits, so running them between the same two barriers gives exactly
// the results of the reference's one-row-at-a-time order (BG1: 46 rows in 32 steps, BG2: 42 in 28).
__constant__ uint8_t  c_step_row0[2][pg::kBg1Rows]; // first row of each step
__constant__ uint8_t  c_step_nrows[2][pg::kBg1Rows];
__constant__ uint8_t  c_nsteps[2];
__constant__ uint16_t c_row_e0[2][pg::kBg1Rows + 1]; // first edge of each row (prefix sums of the degrees)

__device__ __forceinline__ int dev_set_index(int Z)
{
  const int a_tab[8] = {2, 3, 5, 7, 9, 11, 13, 15};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int t = Z;
    while ((t & 1) == 0 && t > a_tab[i]) {
      t >>= 1;
    }
    if (t == a_tab[i]) {
      return i;
    }
  }
  return -1;
}

// Steps of a codeblock that processes nof_layers rows: those whose first row is below nof_layers.
__device__ __forceinline__ int steps_for_layers(int g, int nof_layers)
{
  int n = 0;
  while (n < c_nsteps[g] && c_step_row0[g][n] < nof_layers) {
    ++n;
  }
  return n;
}

// Pulls the check-to-variable messages of step st (rows up to nof_layers) into L1 ahead of their
// use: one prefetch per 128-byte line, thread `tid` taking line tid. Message rows are
// row_bytes apart (one per edge) starting at base.
__device__ __forceinline__ void prefetch_step(const int g, const int st, const int nof_layers, const int tid,
                                              const char* base, const int row_bytes)
{
  const int r0    = c_step_row0[g][st];
  const int r1    = min(r0 + (int)c_step_nrows[g][st], nof_layers);
  const int ea    = c_row_e0[g][r0];
  const int lpe   = (row_bytes + 127) >> 7;
  const int lines = (c_row_e0[g][r1] - ea) * lpe;
  if (tid < lines) {
    const int e = tid / lpe;
    const char* p = base + (size_t)(ea + e) * row_bytes + ((tid - e * lpe) << 7);
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
  }
}

__device__ __forceinline__ int scale_mag(int m)
{
  return (m * 52428) >> 16;
}

__device__ __forceinline__ int warp_max(int v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

__device__ __forceinline__ uint32_t warp_xor(uint32_t v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v ^= __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// One layer (base-graph row) for check lane tid, specialised on the row degree so that the edge
// loops unroll without predication. FIRST selects the first iteration, where every row's
// check-to-variable messages are still zero (the reference copies the soft bits into the v2c
// messages then: ldpc_decoder_impl.cpp:208-212).
template <int DEG, bool FIRST, int ZT>
__device__ __forceinline__ void row_update(const int tid, const int Zr, int8_t* __restrict__ soft,
                                           const uint32_t* __restrict__ edge, int8_t* __restrict__ c2v_row)
{
  const int Z = ZT > 0 ? ZT : Zr;
  int       m[DEG];
  unsigned  pos[DEG];
  int       min1 = 120, min2 = 120, sgn = 0;
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    const uint32_t ed = edge[e];
    const unsigned p0 = (unsigned)tid + (ed & 0xffffu);
    const unsigned p  = min(p0, p0 - (unsigned)Z) + (ed >> 16);
    pos[e]            = p;
    const int x       = soft[p];
    int       v       = x;
    if (!FIRST) {
      const int c = c2v_row[e * Z];
      v           = max(-120, min(120, x - c));
      v           = (x == 127 || x == -127) ? x : v;
    }
    m[e]        = v;
    const int a = abs(v);
    min2        = min(min2, max(min1, a));
    min1        = min(min1, a);
    sgn ^= v;
  }
  const int s1 = scale_mag(min1);
  const int s2 = scale_mag(min2);
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    const int v    = m[e];
    const int a    = abs(v);
    const int mag  = (a == min1) ? s2 : s1;
    const int c    = ((v ^ sgn) < 0) ? -mag : mag;
    c2v_row[e * Z] = (int8_t)c;
    int t          = c + v;
    t              = (t > 120) ? 127 : ((t < -120) ? -127 : t);
    t              = (a == 127) ? v : t;
    soft[pos[e]]   = (int8_t)t;
  }
}

// Degree-19 rows (BG1 rows 0-3): the same update as a rolled loop with the v2c messages staged in
// shared memory (one byte per edge and lane), so the wide rows do not raise the register budget
// of the whole kernel; the soft-bit addresses are recomputed in the second pass.
template <bool FIRST, int ZT, int NT>
__device__ __forceinline__ void row_update_wide(const int deg, const int tid, const int Zr, int8_t* __restrict__ soft,
                                                const uint32_t* __restrict__ edge, int8_t* __restrict__ c2v_row,
                                                int8_t* __restrict__ mbuf)
{
  const int Z    = ZT > 0 ? ZT : Zr;
  int       min1 = 120, min2 = 120, sgn = 0;
#pragma unroll 2
  for (int e = 0; e < deg; ++e) {
    const uint32_t ed = edge[e];
    const unsigned p0 = (unsigned)tid + (ed & 0xffffu);
    const unsigned p  = min(p0, p0 - (unsigned)Z) + (ed >> 16);
    const int      x  = soft[p];
    int            v  = x;
    if (!FIRST) {
      const int c = c2v_row[e * Z];
      v           = max(-120, min(120, x - c));
      v           = (x == 127 || x == -127) ? x : v;
    }
    mbuf[e * NT + tid] = (int8_t)v;
    const int a              = abs(v);
    min2                     = min(min2, max(min1, a));
    min1                     = min(min1, a);
    sgn ^= v;
  }
  const int s1 = scale_mag(min1);
  const int s2 = scale_mag(min2);
#pragma unroll 2
  for (int e = 0; e < deg; ++e) {
    const uint32_t ed  = edge[e];
    const unsigned p0  = (unsigned)tid + (ed & 0xffffu);
    const unsigned p   = min(p0, p0 - (unsigned)Z) + (ed >> 16);
    const int      v   = mbuf[e * NT + tid];
    const int      a   = abs(v);
    const int      mag = (a == min1) ? s2 : s1;
    const int      c   = ((v ^ sgn) < 0) ? -mag : mag;
    c2v_row[e * Z]     = (int8_t)c;
    int t              = c + v;
    t                  = (t > 120) ? 127 : ((t < -120) ? -127 : t);
    t                  = (a == 127) ? v : t;
    soft[p]            = (int8_t)t;
  }
}

// Base-graph row degrees: BG1 {3..10, 19}, BG2 {3..10}.
template <bool FIRST, int ZT, int NT>
__device__ __forceinline__ void row_dispatch(int deg, int tid, int Z, int8_t* soft, const uint32_t* edge, int8_t* c2v_row,
                                             int8_t* mbuf)
{
  switch (deg) {
    case 3: row_update<3, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 4: row_update<4, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 5: row_update<5, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 6: row_update<6, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 7: row_update<7, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 8: row_update<8, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 9: row_update<9, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    case 10: row_update<10, FIRST, ZT>(tid, Z, soft, edge, c2v_row); break;
    default: row_update_wide<FIRST, ZT, NT>(deg, tid, Z, soft, edge, c2v_row, mbuf); break;
  }
}

// Shared memory of the one-lane decoder: NT threads, lifting sizes up to MAXZ (22 * MAXZ / 32 <= NT,
// so that one thread per 32-bit hard-decision word covers the message).
template <int NT, int MAXZ>
struct smem_scalar_t {
  __align__(16) int8_t soft[pg::kMaxNodes * MAXZ];
  uint32_t             edge[pg::kBg1Edges];
  uint32_t             hard[(22 * MAXZ) / 32];
  uint32_t             red[NT / 32];
  int8_t               mbuf[pg::kMaxRowDegree * NT]; // v2c staging of the degree-19 rows
  int                  s_last;
  int                  s_done;
};
using smem_t = smem_scalar_t<kThreads, pg::kMaxZ>;

// Decodes codeblock cb with check-to-variable slab `slab`, one lane per thread (NT threads, Z <=
// MAXZ); ZT > 0 specialises the lifting size at compile time.
template <int ZT, int NT, int MAXZ>
__device__ __forceinline__ void decode_codeblock(const pg_ldpc_cb& d, smem_scalar_t<NT, MAXZ>& sm,
                                                 const int8_t* __restrict__ llrs,
                                                 uint8_t* __restrict__ bits, int32_t* __restrict__ iterations,
                                                 int8_t* __restrict__ c2v_all, const uint32_t* __restrict__ crc_pow,
                                                 const int cb, const int slab)
{
  int8_t*   soft   = sm.soft;
  uint32_t* edge   = sm.edge;
  uint32_t* hard   = sm.hard;
  uint32_t* red    = sm.red;
  int&      s_last = sm.s_last;
  int&      s_done = sm.s_done;
  const int        tid = threadIdx.x;
  const int        bg  = d.base_graph;
  const int        Z   = ZT > 0 ? ZT : (int)d.lifting_size;
  const int        set = (Z >= 2 && Z <= MAXZ) ? dev_set_index(Z) : -1;
  if ((bg != 1 && bg != 2) || set < 0) {
    if (tid == 0) {
      iterations[cb] = -1;
    }
    return;
  }
  const int     g        = bg - 1;
  const int     Kb       = bg == 1 ? 22 : 10;
  const int     nrows    = bg == 1 ? pg::kBg1Rows : pg::kBg2Rows;
  const int     nedges   = bg == 1 ? pg::kBg1Edges : pg::kBg2Edges;
  const int     nfull    = bg == 1 ? 68 : 52;
  const int     msg_len  = Kb * Z;
  const int     n        = (int)d.nof_llrs;
  const int8_t* in       = llrs + d.llr_offset;
  int8_t*       c2v      = c2v_all + (size_t)slab * pg::kC2vStride;
  const int     nbytes   = (msg_len + 7) / 8;
  uint8_t*      out      = bits + d.out_offset;
  const int     crc_poly = d.crc_poly;
  const int     nwords   = (msg_len + 31) / 32;

  // Edge table of this lifting size: node offset (col * Z) and shift (V mod Z).
  for (int e = tid; e < nedges; e += NT) {
    const int col = c_edge_col[g][e];
    const int s   = c_edge_v[g][e][set] % Z;
    edge[e]       = ((uint32_t)(col * Z) << 16) | (uint32_t)s;
  }
  if (tid == 0) {
    s_last = 0;
    s_done = 0;
  }
  __syncthreads();

  // One pass over the input: soft bits (2Z punctured zeros, whole nodes clamped to +-64, a ragged
  // tail as is, ldpc_decoder_impl.cpp:147-188) and the last non-zero LLR (the trailing-zero trim,
  // ldpc_decoder_impl.cpp:66-71), four LLRs per thread step.
  const int nof_full = (n / Z) * Z;
  const int soft_len = nfull * Z;
  for (int i = tid; i < 2 * Z; i += NT) {
    soft[i] = 0;
  }
  for (int i = 2 * Z + n + tid; i < soft_len; i += NT) {
    soft[i] = 0;
  }
  int        last    = 0;
  const bool aligned = (reinterpret_cast<uintptr_t>(in) & 3u) == 0;
  for (int k0 = 4 * tid; k0 < n; k0 += 4 * NT) {
    int v[4];
    if (aligned && k0 + 3 < n) {
      const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(in + k0));
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        v[j] = (int)(int8_t)(w >> (8 * j));
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        v[j] = k0 + j < n ? (int)in[k0 + j] : 0;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + j;
      if (k < n && 2 * Z + k < soft_len) {
        last = v[j] != 0 ? k + 1 : last;
        soft[2 * Z + k] = (int8_t)(k < nof_full ? max(-64, min(64, v[j])) : v[j]);
      }
    }
  }
  last = warp_max(last);
  if ((tid & 31) == 0 && last > 0) {
    atomicMax(&s_last, last);
  }
  __syncthreads();

  const int input_size = s_last;
  if (input_size < msg_len) {
    for (int b = tid; b < nbytes; b += NT) {
      out[b] = 0xff;
    }
    if (tid == 0) {
      iterations[cb] = 0;
    }
    return;
  }
  int cb_len = max(input_size + 2 * Z, (Kb + 4) * Z);
  cb_len     = ((cb_len + Z - 1) / Z) * Z;
  const int nof_layers = min(cb_len / Z - Kb, nrows);

  uint32_t g_poly = 0;
  int      order  = 24;
  if (crc_poly == PG_CRC16) {
    order = 16;
  }
  const uint32_t* pow_tab = crc_pow + (size_t)(crc_poly <= PG_CRC24B ? crc_poly : 0) * pg::kCrcPowLen;
  (void)g_poly;
  const int crc_len = msg_len - (int)d.nof_filler_bits;

  int result = 0;
  const int max_it = d.max_iterations;
  const int nsteps = steps_for_layers(g, nof_layers);
  for (int it = 0; it < max_it; ++it) {
    for (int st = 0; st < nsteps; ++st) {
      // Messages are read from the second iteration on: prefetch the next step's.
      if (it > 0 || st + 1 == nsteps) {
        prefetch_step(g, st + 1 < nsteps ? st + 1 : 0, nof_layers, tid, reinterpret_cast<const char*>(c2v), Z);
      }
      const int r0 = c_step_row0[g][st];
      const int r1 = min(r0 + (int)c_step_nrows[g][st], nof_layers);
      if (tid < Z) {
        for (int r = r0; r < r1; ++r) {
          const int deg     = c_row_deg[g][r];
          const int e0      = c_row_e0[g][r];
          int8_t*   c2v_row = c2v + (size_t)e0 * Z + tid;
          if (it == 0) {
            row_dispatch<true, ZT, NT>(deg, tid, Z, soft, edge + e0, c2v_row, sm.mbuf);
          } else {
            row_dispatch<false, ZT, NT>(deg, tid, Z, soft, edge + e0, c2v_row, sm.mbuf);
          }
        }
      }
      __syncthreads();
    }

    // Hard decisions, zero check and CRC over the significant bits.
    int      zero = 0;
    uint32_t crc  = 0;
    if (tid < nwords) {
      const int4* p = reinterpret_cast<const int4*>(soft + 32 * tid);
      const int4  a = p[0];
      const int4  b = p[1];
      const int   wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      uint32_t    w     = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int idx = 32 * tid + 4 * k + j;
          const int x   = (int)(int8_t)((uint32_t)wv[k] >> (8 * j));
          if (idx < msg_len) {
            w |= (uint32_t)(x <= 0) << (31 - (4 * k + j));
            zero |= (x == 0);
          }
        }
      }
      hard[tid] = w;
      if (crc_poly != PG_CRC_NONE) {
        const int valid = crc_len - 32 * tid;
        uint32_t  wc    = w;
        if (valid <= 0) {
          wc = 0;
        } else if (valid < 32) {
          wc &= ~((1u << (32 - valid)) - 1u);
        }
        const int e_w = crc_len - 32 * tid - 32 + order;
        while (wc != 0) {
          const int q = __ffs(wc) - 1;
          crc ^= __ldg(pow_tab + e_w + q);
          wc &= wc - 1;
        }
      }
    }
    zero = __syncthreads_or(zero);
    crc  = warp_xor(crc);
    if ((tid & 31) == 0) {
      red[tid >> 5] = crc;
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t t = 0;
      for (int w = 0; w < NT / 32; ++w) {
        t ^= red[w];
      }
      s_done = (crc_poly != PG_CRC_NONE && !zero && t == 0) ? 1 : 0;
    }
    __syncthreads();
    if (s_done) {
      result = it + 1;
      break;
    }
  }

  if (crc_poly == PG_CRC_NONE) {
    // Syndrome check over the processed rows (ldpc_decoder_impl.cpp:329-387).
    int bad = 0;
    if (tid < Z) {
      int e0 = 0;
      for (int r = 0; r < nof_layers; ++r) {
        const int deg    = c_row_deg[g][r];
        int       parity = 0;
        for (int e = 0; e < deg; ++e) {
          const uint32_t ed = edge[e0 + e];
          int            p  = tid + (int)(ed & 0xffffu);
          p                 = (p >= Z) ? p - Z : p;
          const int x       = soft[p + (int)(ed >> 16)];
          bad |= (x == 0);
          parity ^= (x <= 0);
        }
        bad |= parity;
        e0 += deg;
      }
    }
    bad = __syncthreads_or(bad);
    // The hard words of the last iteration are in hard[]; a zero soft bit also fails.
    int zero = 0;
    if (tid < nwords) {
      for (int k = 0; k < 32; ++k) {
        const int idx = 32 * tid + k;
        if (idx < msg_len && soft[idx] == 0) {
          zero = 1;
        }
      }
    }
    zero   = __syncthreads_or(zero);
    result = (!bad && !zero) ? max_it : 0;
  }

  for (int b = tid; b < nbytes; b += NT) {
    out[b] = (uint8_t)(hard[b >> 2] >> (24 - 8 * (b & 3)));
  }
  if (tid == 0) {
    iterations[cb] = result;
  }
}


// counter == nullptr: one CTA per codeblock (blockIdx.x), slab blockIdx.x. Otherwise a persistent
// grid: each CTA takes the next work index from *counter (zeroed before the launch), decodes
// codeblock order[w] (or w) with its own slab blockIdx.x, and stops when the n codeblocks are
// taken. Codeblocks are independent, so the order of work changes no result.
__global__ void __launch_bounds__(kThreads, 2) ldpc_decode_kernel(const pg_ldpc_cb* __restrict__ descs,
                                                              const int8_t* __restrict__ llrs,
                                                              uint8_t* __restrict__ bits,
                                                              int32_t* __restrict__ iterations,
                                                              int8_t* __restrict__ c2v_all,
                                                              const uint32_t* __restrict__ crc_pow,
                                                              const uint32_t* __restrict__ order, int n,
                                                              int* __restrict__ counter, int skip_z)
{
  __shared__ smem_t sm;
  __shared__ int    s_work;
  if (counter == nullptr) {
    const pg_ldpc_cb d = descs[blockIdx.x];
    if (d.lifting_size == 384) {
      decode_codeblock<384, kThreads, pg::kMaxZ>(d, sm, llrs, bits, iterations, c2v_all, crc_pow, blockIdx.x, blockIdx.x);
    } else {
      decode_codeblock<0, kThreads, pg::kMaxZ>(d, sm, llrs, bits, iterations, c2v_all, crc_pow, blockIdx.x, blockIdx.x);
    }
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) {
      s_work = atomicAdd(counter, 1);
    }
    __syncthreads();
    const int w = s_work;
    __syncthreads();
    if (w >= n) {
      break;
    }
    const int        cb = order != nullptr ? (int)order[w] : w;
    const pg_ldpc_cb d  = descs[cb];
    if (d.lifting_size == skip_z) {
      continue; // left to ldpc_decode_x2_kernel
    }
    if (d.lifting_size == 384) {
      decode_codeblock<384, kThreads, pg::kMaxZ>(d, sm, llrs, bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
    } else {
      decode_codeblock<0, kThreads, pg::kMaxZ>(d, sm, llrs, bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Two-lanes-per-thread decoder: one 192-thread CTA per codeblock, every lifting size.
//
// Pair mode (even Z > 192, H = Z / 2): thread j (0 <= j < H) carries check lanes j and j + H as
// the two halves of one f16x2 register. For an edge of shift s the two variable lanes it reads,
// (j + s) mod Z and (j + H + s) mod Z, differ by H, so soft bits live twice in shared memory and
// the shifted pair is one 16-bit word: D[col][w] = (soft[col][w], soft[col][(w + H) mod Z]).
// The reference's int8 rules become exact f16x2 identities:
//   v2c      = x == +-127 ? x : clamp(x - c, -120, 120)       (reference)
//   v        = min(max(clamp(x - c, -120, 120), 104x - 12984), 104x + 12984)  (fused
//              multiply-adds; for |x| <= 120 the bounds lie outside [-120, 120], for x = +-127
//              they are +-224; in the first iteration c = 0 and x is not clamped, and the bounds
//              keep every |x| <= 126 as it is)
//              so v = v2c, except that a saturated soft bit gives +-224 instead of +-127. Both
//              exceed every magnitude the minimum search starts from (120) and keep the sign, so
//              the row's minima, sign and messages are the same; and +-224 plus any message
//              (|c2v| <= 96) stays above 120 in magnitude, so the soft update below gives +-127
//              back without the reference's separate test of |v2c| == 127.
//   min1/min2/sign: min.xorsign.abs keeps min(|.|) and accumulates the sign product in min1's sign
//   c2v      = sign(product of the others) * (|v2c| == min1 ? s2 : s1),
//              magnitude = s2 + (s1 - s2) * (|v| != min1), the comparison as f16 1.0 / 0.0, sign by
//              XOR of sign bits
//   soft     = |v2c| == 127 ? v2c : promote(c2v + v2c) = promote(c2v + v),
//              promote(t) = clamp(8t - 7 clamp(t, +-120), +-127)
//   scale    s = (m * 52428) >> 16 from a table indexed by the f16 bit pattern of m over 16.
// Every value used is an integer of magnitude at most 2,560 (even above 2,048), so f16 arithmetic
// (11-bit significand) on it is exact; the bounds are exact where they decide (x = +-127).
// Storage is int8 in offset binary (byte = value + 128): f16 bits 0x6400 | byte are 1024 + byte, so
// one byte permute and one f16x2 subtraction of 1152 give the values, and an addition of 1152 and a
// byte permute give the bytes back, exactly. Check-to-variable messages are byte pairs per (edge,
// thread) in the global slab.
//
// Scalar mode (Z <= 192): the one-lane arithmetic of ldpc_decode_kernel with 192 threads.
constexpr int kX2Threads  = 192; // = kMaxZ / 2
constexpr int kScaleTab   = 1408;
constexpr int kX2MaxPerSm = 4;   // resident CTAs per SM (registers)

template <int NT>
struct __align__(16) smem_pair_nt_t {
  uint16_t D[pg::kMaxNodes * pg::kMaxZ]; // soft-bit pairs, column stride Z
  uint32_t edge[pg::kBg1Edges];          // col*Z << 16 | s
  uint32_t hard[(22 * pg::kMaxZ) / 32];
  uint32_t red[NT / 32];
  int      s_last;
  int      s_done;
};
using smem_pair_t      = smem_pair_nt_t<kX2Threads>;
using smem_x2_scalar_t = smem_scalar_t<kX2Threads, kX2Threads>;
constexpr size_t kX2Smem = sizeof(smem_pair_t) > sizeof(smem_x2_scalar_t) ? sizeof(smem_pair_t)
                                                                           : sizeof(smem_x2_scalar_t);

// Split decoder: 384 threads per codeblock. Pair mode (even Z > 192) runs two threads per lane
// pair, each taking every second edge of a row; other lifting sizes run the one-lane arithmetic
// with one thread per lane.
constexpr int kSplitThreads  = 384;
constexpr int kSplitMaxPerSm = 2;
using smem_split_pair_t      = smem_pair_nt_t<kSplitThreads>;
using smem_split_scalar_t    = smem_scalar_t<kSplitThreads, pg::kMaxZ>;
constexpr size_t kSplitSmem  = sizeof(smem_split_pair_t) > sizeof(smem_split_scalar_t) ? sizeof(smem_split_pair_t)
                                                                                        : sizeof(smem_split_scalar_t);

__device__ __forceinline__ uint32_t h2_sub(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_add(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("add.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_fma(uint32_t a, uint32_t b, uint32_t c)
{
  uint32_t r;
  asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t h2_mul(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_min(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("min.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_max(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_min_xs(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("min.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t h2_max_xs(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("max.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}

// f16x2 constants (both halves equal).
constexpr uint32_t kH120    = 0x57805780u; // 120
constexpr uint32_t kHm120   = 0xd780d780u; // -120
constexpr uint32_t kH127    = 0x57f057f0u; // 127
constexpr uint32_t kHm127   = 0xd7f0d7f0u; // -127
constexpr uint32_t kH104    = 0x56805680u; // 104
constexpr uint32_t kHm12984 = 0xf257f257u; // -12984
constexpr uint32_t kH12984  = 0x72577257u; // 12984
constexpr uint32_t kH8      = 0x48004800u; // 8
constexpr uint32_t kHm7     = 0xc700c700u; // -7
constexpr uint32_t kH1152   = 0x64806480u; // 1152 = 1024 + 128
constexpr uint32_t kAbs     = 0x7fff7fffu;
constexpr uint32_t kSign    = 0x80008000u;

// Offset-binary byte pair -> f16x2 integers (low byte first).
__device__ __forceinline__ uint32_t bytes_to_h2(uint32_t b)
{
  return h2_sub(__byte_perm(b, 0x6464u, 0x5140u), kH1152);
}
__device__ __forceinline__ uint32_t h2_to_bytes_biased(uint32_t c)
{
  return h2_add(c, kH1152); // bytes 0 and 2 are the offset-binary values
}

__device__ __forceinline__ uint32_t x2_scale(const uint16_t* __restrict__ tab, uint32_t m)
{
  return (uint32_t)__ldg(tab + ((m & 0xffffu) >> 4)) | ((uint32_t)__ldg(tab + (m >> 20)) << 16);
}

__device__ __forceinline__ uint32_t h2_ne(uint32_t a, uint32_t b)
{
  uint32_t r;
  asm("set.ne.f16x2.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}

// v2c of one edge (saturated soft bits as +-224) from its soft-bit pair x and its stored
// check-to-variable pair.
template <bool FIRST>
__device__ __forceinline__ uint32_t pair_v2c(const uint32_t x, const uint16_t* __restrict__ c2v)
{
  uint32_t d = x;
  if (!FIRST) {
    d = h2_min(h2_max(h2_sub(x, bytes_to_h2(*c2v)), kHm120), kH120);
  }
  return h2_min(h2_max(d, h2_fma(x, kH104, kHm12984)), h2_fma(x, kH104, kH12984));
}

// One layer for thread j. Rows of degree up to 10 keep each edge's v2c, soft-bit position and
// partner position from the first pass; the degree-19 rows keep the v2c of their first ten edges
// and recompute the rest (the soft bits and messages they read are not yet overwritten), so that
// they stay within the register budget of four CTAs per SM.
template <int DEG, bool FIRST>
__device__ __forceinline__ void row_update_pair(const unsigned j, const unsigned Z, const unsigned H,
                                                uint16_t* __restrict__ D, const uint32_t* __restrict__ edge,
                                                uint16_t* __restrict__ c2v_row, const uint16_t* __restrict__ tab)
{
  constexpr bool KEEP = DEG <= 10;
  constexpr int  NV   = KEEP ? DEG : 10;
  uint32_t       v[NV];
  unsigned       pos[KEEP ? DEG : 1], par[KEEP ? DEG : 1];
  uint32_t       min1 = kH120, min2 = kH120;
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    const uint32_t ed = edge[e];
    const unsigned p0 = j + (ed & 0xffffu);
    const unsigned w  = min(p0, p0 - Z); // (j + s) mod Z
    const unsigned p  = w + (ed >> 16);
    if constexpr (KEEP) {
      pos[e] = p;
      par[e] = w < H ? p + H : p - H;
    }
    const uint32_t vv = pair_v2c<FIRST>(bytes_to_h2(D[p]), c2v_row + e * kX2Threads);
    if (e < NV) {
      v[e < NV ? e : 0] = vv;
    }
    const uint32_t t = h2_max_xs(min1, vv);
    min2             = h2_min_xs(min2, t);
    min1             = h2_min_xs(min1, vv);
  }
  const uint32_t m1  = min1 & kAbs;
  const uint32_t s1  = x2_scale(tab, m1);
  const uint32_t s2  = x2_scale(tab, min2 & kAbs);
  const uint32_t nds = h2_sub(s1, s2);
  const uint32_t sgn = min1 & kSign;  // sign product of every v2c of the row
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    unsigned p, q;
    if constexpr (KEEP) {
      p = pos[e];
      q = par[e];
    } else {
      const uint32_t ed = edge[e];
      const unsigned p0 = j + (ed & 0xffffu);
      const unsigned w  = min(p0, p0 - Z);
      p                 = w + (ed >> 16);
      q                 = w < H ? p + H : p - H;
    }
    const uint32_t vv  = e < NV ? v[e < NV ? e : 0] : pair_v2c<FIRST>(bytes_to_h2(D[p]), c2v_row + e * kX2Threads);
    const uint32_t mag = h2_fma(nds, h2_ne(vv & kAbs, m1), s2);
    const uint32_t c   = mag ^ ((sgn ^ vv) & kSign);
    c2v_row[e * kX2Threads] = (uint16_t)__byte_perm(h2_to_bytes_biased(c), 0, 0x0020);
    const uint32_t t   = h2_add(c, vv);
    const uint32_t cl  = h2_min(h2_max(t, kHm120), kH120);
    uint32_t       u   = h2_fma(cl, kHm7, h2_mul(t, kH8));
    u                  = h2_min(h2_max(u, kHm127), kH127);
    const uint32_t ub  = h2_to_bytes_biased(u);
    D[p] = (uint16_t)__byte_perm(ub, 0, 0x0020);
    D[q] = (uint16_t)__byte_perm(ub, 0, 0x0002);
  }
}

// One layer for lane pair j split over two threads: thread t (0 or 1) takes edges t, t + 2, ... of
// the row (a thread with an odd-degree row's missing last edge contributes +120, which changes no
// minimum and no sign), the two partial (min1, min2, sign) meet through one shuffle, and each
// thread updates its own edges. With at most ten edges per thread every row keeps its v2c, soft-bit
// positions and partner positions in registers. Threads past the last lane pair (j >= H) run the
// row without loads or stores, so that every shuffle has its whole warp.
template <int DEG, bool FIRST>
__device__ __forceinline__ void row_update_split(const unsigned j, const unsigned t, const unsigned Z, const unsigned H,
                                                 uint16_t* __restrict__ D, const uint32_t* __restrict__ edge,
                                                 uint16_t* __restrict__ c2v_row, const uint16_t* __restrict__ tab)
{
  constexpr int NE     = (DEG + 1) / 2;
  const bool    active = j < H;
  uint32_t      v[NE];
  unsigned      pos[NE], par[NE];
  uint32_t      min1 = kH120, min2 = kH120;
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const unsigned e     = 2 * k + t;
    const bool     valid = active && ((DEG % 2) == 0 || k + 1 < NE || e < DEG);
    const uint32_t ed    = edge[valid ? e : 0];
    const unsigned p0    = j + (ed & 0xffffu);
    const unsigned w     = min(p0, p0 - Z); // (j + s) mod Z
    const unsigned p     = w + (ed >> 16);
    pos[k]               = p;
    par[k]               = w < H ? p + H : p - H;
    uint32_t vv          = kH120;
    if (valid) {
      vv = pair_v2c<FIRST>(bytes_to_h2(D[p]), c2v_row + e * kX2Threads);
    }
    v[k]             = vv;
    const uint32_t x = h2_max_xs(min1, vv);
    min2             = h2_min_xs(min2, x);
    min1             = h2_min_xs(min1, vv);
  }
  const uint32_t o1 = __shfl_xor_sync(0xffffffffu, min1, 1);
  const uint32_t o2 = __shfl_xor_sync(0xffffffffu, min2, 1);
  min2              = h2_min_xs(h2_min_xs(min2, o2), h2_max_xs(min1, o1));
  min1              = h2_min_xs(min1, o1);
  const uint32_t m1  = min1 & kAbs;
  const uint32_t s1  = x2_scale(tab, m1);
  const uint32_t s2  = x2_scale(tab, min2 & kAbs);
  const uint32_t nds = h2_sub(s1, s2);
  const uint32_t sgn = min1 & kSign; // sign product of every v2c of the row
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const unsigned e     = 2 * k + t;
    const bool     valid = active && ((DEG % 2) == 0 || k + 1 < NE || e < DEG);
    if (valid) {
      const uint32_t vv  = v[k];
      const uint32_t mag = h2_fma(nds, h2_ne(vv & kAbs, m1), s2);
      const uint32_t c   = mag ^ ((sgn ^ vv) & kSign);
      c2v_row[e * kX2Threads] = (uint16_t)__byte_perm(h2_to_bytes_biased(c), 0, 0x0020);
      const uint32_t tt  = h2_add(c, vv);
      const uint32_t cl  = h2_min(h2_max(tt, kHm120), kH120);
      uint32_t       u   = h2_fma(cl, kHm7, h2_mul(tt, kH8));
      u                  = h2_min(h2_max(u, kHm127), kH127);
      const uint32_t ub  = h2_to_bytes_biased(u);
      D[pos[k]]          = (uint16_t)__byte_perm(ub, 0, 0x0020);
      D[par[k]]          = (uint16_t)__byte_perm(ub, 0, 0x0002);
    }
  }
}

template <bool FIRST>
__device__ __forceinline__ void row_dispatch_split(int deg, unsigned j, unsigned t, unsigned Z, unsigned H,
                                                   uint16_t* D, const uint32_t* edge, uint16_t* c2v_row,
                                                   const uint16_t* tab)
{
  switch (deg) {
    case 3: row_update_split<3, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 4: row_update_split<4, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 5: row_update_split<5, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 6: row_update_split<6, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 7: row_update_split<7, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 8: row_update_split<8, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 9: row_update_split<9, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    case 10: row_update_split<10, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
    default: row_update_split<19, FIRST>(j, t, Z, H, D, edge, c2v_row, tab); break;
  }
}

template <bool FIRST>
__device__ __forceinline__ void row_dispatch_pair(int deg, unsigned j, unsigned Z, unsigned H, uint16_t* D,
                                                  const uint32_t* edge, uint16_t* c2v_row, const uint16_t* tab)
{
  switch (deg) {
    case 3: row_update_pair<3, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 4: row_update_pair<4, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 5: row_update_pair<5, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 6: row_update_pair<6, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 7: row_update_pair<7, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 8: row_update_pair<8, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 9: row_update_pair<9, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    case 10: row_update_pair<10, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
    default: row_update_pair<19, FIRST>(j, Z, H, D, edge, c2v_row, tab); break;
  }
}

// Eight input LLRs from index k (any k; outside [0, n) they are zero) as soft bits in offset
// binary, four per word: whole nodes (index < nof_full) clamped to +-64, a ragged tail as is
// (ldpc_decoder_impl.cpp:147-188). last: one past the last non-zero LLR seen (the trailing-zero trim,
// ldpc_decoder_impl.cpp:66-71).
__device__ __forceinline__ void fetch8(const int8_t* __restrict__ in, int k, int n, int nof_full, bool aligned,
                                       int& last, uint32_t& w0, uint32_t& w1)
{
  int v[8];
  if (aligned && k >= 0 && k + 8 <= n) {
    const uint2 q = __ldg(reinterpret_cast<const uint2*>(in + k));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v[i]     = (int)(int8_t)(q.x >> (8 * i));
      v[i + 4] = (int)(int8_t)(q.y >> (8 * i));
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[i] = (k + i >= 0 && k + i < n) ? (int)__ldg(in + k + i) : 0;
    }
  }
  w0 = 0;
  w1 = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int kk = k + i;
    last         = v[i] != 0 ? kk + 1 : last;
    const int x  = kk < nof_full ? max(-64, min(64, v[i])) : v[i];
    const uint32_t b = (uint32_t)(x + 128);
    if (i < 4) {
      w0 |= b << (8 * i);
    } else {
      w1 |= b << (8 * (i - 4));
    }
  }
}

// Decodes codeblock cb (even Z > 192) with check-to-variable slab `slab`: NT threads, T threads per
// lane pair (NT = 192 * T).
template <int NT, int T>
__device__ void decode_codeblock_pair(const pg_ldpc_cb& d, smem_pair_nt_t<NT>& sm, const int8_t* __restrict__ llrs,
                                      uint8_t* __restrict__ bits, int32_t* __restrict__ iterations,
                                      int8_t* __restrict__ c2v_all, const uint32_t* __restrict__ crc_pow,
                                      const uint16_t* __restrict__ scale_tab, const int cb, const int slab)
{
  static_assert(NT == kX2Threads * T && (T == 1 || T == 2), "one or two threads per lane pair");
  const int tid = threadIdx.x;
  const int bg  = d.base_graph;
  const int Z   = (int)d.lifting_size;
  const int H   = Z >> 1;
  const int set = (Z <= pg::kMaxZ) ? dev_set_index(Z) : -1;
  if ((bg != 1 && bg != 2) || set < 0 || (Z & 15) != 0) {
    if (tid == 0) {
      iterations[cb] = -1;
    }
    return;
  }
  const int     g        = bg - 1;
  const int     Kb       = bg == 1 ? 22 : 10;
  const int     nrows    = bg == 1 ? pg::kBg1Rows : pg::kBg2Rows;
  const int     nedges   = bg == 1 ? pg::kBg1Edges : pg::kBg2Edges;
  const int     nfull    = bg == 1 ? 68 : 52;
  const int     msg_len  = Kb * Z;
  const int     n        = (int)d.nof_llrs;
  const int8_t* in       = llrs + d.llr_offset;
  uint16_t*     c2v      = reinterpret_cast<uint16_t*>(c2v_all + (size_t)slab * pg::kC2vStride);
  const int     nbytes   = (msg_len + 7) / 8;
  uint8_t*      out      = bits + d.out_offset;
  const int     crc_poly = d.crc_poly;
  const int     nwords   = (msg_len + 31) / 32;
  uint16_t*     D        = sm.D;

  for (int e = tid; e < nedges; e += NT) {
    const int col = c_edge_col[g][e];
    const int s   = c_edge_v[g][e][set] % Z;
    sm.edge[e]    = ((uint32_t)(col * Z) << 16) | (uint32_t)s;
  }
  if (tid == 0) {
    sm.s_last = 0;
    sm.s_done = 0;
  }
  __syncthreads();

  // Soft bits, eight lanes of each half of a column per thread step (2Z punctured zeros, then the
  // input), both copies: D[col][w0 + i] = (soft[w0 + i], soft[w0 + H + i]) and the swapped pair at
  // w0 + H + i.
  {
    const int  per_col  = H / 8;
    const int  nchunks  = nfull * per_col;
    const int  nof_full = (n / Z) * Z;
    const bool aligned  = (reinterpret_cast<uintptr_t>(in) & 7u) == 0;
    int        last     = 0;
#pragma unroll 4
    for (int q = tid; q < nchunks; q += NT) {
      const int col = q / per_col;
      const int w0  = (q - col * per_col) * 8;
      const int k   = (col - 2) * Z + w0;
      uint32_t  l0, l1, h0, h1;
      fetch8(in, k, n, nof_full, aligned, last, l0, l1);
      fetch8(in, k + H, n, nof_full, aligned, last, h0, h1);
      uint4 lo, hi;
      lo.x = __byte_perm(l0, h0, 0x5140);
      lo.y = __byte_perm(l0, h0, 0x7362);
      lo.z = __byte_perm(l1, h1, 0x5140);
      lo.w = __byte_perm(l1, h1, 0x7362);
      hi.x = __byte_perm(h0, l0, 0x5140);
      hi.y = __byte_perm(h0, l0, 0x7362);
      hi.z = __byte_perm(h1, l1, 0x5140);
      hi.w = __byte_perm(h1, l1, 0x7362);
      *reinterpret_cast<uint4*>(D + col * Z + w0)     = lo;
      *reinterpret_cast<uint4*>(D + col * Z + w0 + H) = hi;
    }
    last = warp_max(last);
    if ((tid & 31) == 0 && last > 0) {
      atomicMax(&sm.s_last, last);
    }
  }
  __syncthreads();

  const int input_size = sm.s_last;
  if (input_size < msg_len) {
    for (int b = tid; b < nbytes; b += NT) {
      out[b] = 0xff;
    }
    if (tid == 0) {
      iterations[cb] = 0;
    }
    __syncthreads();
    return;
  }
  int cb_len = max(input_size + 2 * Z, (Kb + 4) * Z);
  cb_len     = ((cb_len + Z - 1) / Z) * Z;
  const int nof_layers = min(cb_len / Z - Kb, nrows);

  int order = 24;
  if (crc_poly == PG_CRC16) {
    order = 16;
  }
  const uint32_t* pow_tab = crc_pow + (size_t)(crc_poly <= PG_CRC24B ? crc_poly : 0) * pg::kCrcPowLen;
  const int       crc_len = msg_len - (int)d.nof_filler_bits;

  int            result = 0;
  const int      max_it = d.max_iterations;
  const int      lane   = tid & 31;
  const unsigned j      = (unsigned)tid;
  const int nsteps = steps_for_layers(g, nof_layers);
  for (int it = 0; it < max_it; ++it) {
    for (int st = 0; st < nsteps; ++st) {
      // Messages are read from the second iteration on: prefetch the next step's.
      if (it > 0 || st + 1 == nsteps) {
        prefetch_step(g, st + 1 < nsteps ? st + 1 : 0, nof_layers, tid, reinterpret_cast<const char*>(c2v),
                      kX2Threads * 2);
      }
      const int r0 = c_step_row0[g][st];
      const int r1 = min(r0 + (int)c_step_nrows[g][st], nof_layers);
      if (T == 1 && tid < H) {
        for (int r = r0; r < r1; ++r) {
          const int deg     = c_row_deg[g][r];
          const int e0      = c_row_e0[g][r];
          uint16_t* c2v_row = c2v + (size_t)e0 * kX2Threads + tid;
          if (it == 0) {
            row_dispatch_pair<true>(deg, j, (unsigned)Z, (unsigned)H, D, sm.edge + e0, c2v_row, scale_tab);
          } else {
            row_dispatch_pair<false>(deg, j, (unsigned)Z, (unsigned)H, D, sm.edge + e0, c2v_row, scale_tab);
          }
        }
      } else if (T == 2 && tid < ((2 * H + 31) & ~31)) {
        const unsigned jp = (unsigned)tid >> 1, tp = (unsigned)tid & 1u;
        for (int r = r0; r < r1; ++r) {
          const int deg     = c_row_deg[g][r];
          const int e0      = c_row_e0[g][r];
          uint16_t* c2v_row = c2v + (size_t)e0 * kX2Threads + jp;
          if (it == 0) {
            row_dispatch_split<true>(deg, jp, tp, (unsigned)Z, (unsigned)H, D, sm.edge + e0, c2v_row, scale_tab);
          } else {
            row_dispatch_split<false>(deg, jp, tp, (unsigned)Z, (unsigned)H, D, sm.edge + e0, c2v_row, scale_tab);
          }
        }
      }
      __syncthreads();
    }

    // Hard decisions (soft <= 0: offset byte <= 128; the low byte of D[i] is soft bit i), zero
    // check and CRC: one 32-bit word per warp step, lane k holding bit k of the word (MSB first
    // after the reversal); each set bit within the CRC length adds x^e mod g.
    int      zero = 0;
    uint32_t crc  = 0;
    for (int wi = tid >> 5; wi < nwords; wi += NT / 32) {
      const int      idx = 32 * wi + lane;
      const uint32_t b   = idx < msg_len ? (D[idx] & 0xffu) : 0xffu;
      const bool     bit = b <= 128u;
      zero |= b == 128u;
      const uint32_t w = __brev(__ballot_sync(0xffffffffu, bit));
      if (lane == 0) {
        sm.hard[wi] = w;
      }
      if (crc_poly != PG_CRC_NONE && bit && idx < crc_len) {
        crc ^= __ldg(pow_tab + (crc_len - 1 - idx + order));
      }
    }
    zero = __syncthreads_or(zero);
    crc  = warp_xor(crc);
    if (lane == 0) {
      sm.red[tid >> 5] = crc;
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t t = 0;
      for (int w = 0; w < NT / 32; ++w) {
        t ^= sm.red[w];
      }
      sm.s_done = (crc_poly != PG_CRC_NONE && !zero && t == 0) ? 1 : 0;
    }
    __syncthreads();
    if (sm.s_done) {
      result = it + 1;
      break;
    }
  }

  if (crc_poly == PG_CRC_NONE) {
    // Syndrome check over the processed rows (ldpc_decoder_impl.cpp:329-387), both lanes.
    int bad = 0;
    if (tid < H) {
      int e0 = 0;
      for (int r = 0; r < nof_layers; ++r) {
        const int deg    = c_row_deg[g][r];
        uint32_t  parity = 0;
        for (int e = 0; e < deg; ++e) {
          const uint32_t ed = sm.edge[e0 + e];
          const unsigned p0 = j + (ed & 0xffffu);
          const uint32_t x  = D[min(p0, p0 - (unsigned)Z) + (ed >> 16)];
          const uint32_t lo = x & 0xffu, hi = x >> 8;
          bad |= (lo == 128u) | (hi == 128u);
          parity ^= (uint32_t)(lo <= 128u) | ((uint32_t)(hi <= 128u) << 1);
        }
        bad |= parity != 0;
        e0 += deg;
      }
    }
    bad      = __syncthreads_or(bad);
    int zero = 0;
    for (int i = tid; i < msg_len; i += NT) {
      zero |= (D[i] & 0xffu) == 128u;
    }
    zero   = __syncthreads_or(zero);
    result = (!bad && !zero) ? max_it : 0;
  }

  for (int b = tid; b < nbytes; b += NT) {
    out[b] = (uint8_t)(sm.hard[b >> 2] >> (24 - 8 * (b & 3)));
  }
  if (tid == 0) {
    iterations[cb] = result;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Lifting size 384 (every large transport block): the two-lanes-per-thread arithmetic above with
// everything that depends on Z fixed at compile time and the soft bits stored once, as f16.
//
// Thread j (0 <= j < 192) carries check lanes j and j + 192. Soft bits: E[col][k] = (soft[col][k],
// soft[col][k + 192]) as one f16x2 word, 0 <= k < 192 (52 KB for BG1, so four CTAs share an SM).
// For an edge of shift s, lane j reads variable lane (j + s) mod 384 and lane j + 192 reads
// (j + 192 + s) mod 384: both are halves of the same word k = (j + s') mod 192 with s' = s mod 192,
// swapped when (j + s' >= 192) differs from (s >= 192). Per edge the constant tables give 4 s', the
// column's byte offset and the byte-permute selector of the wrapped case (c_z_*, set for Z = 384
// at table upload); the selector of the unwrapped case differs from it by 0x2222.
// The 0.8 scaling, floor(m * 52428 / 2^16) for integer 0 <= m <= 120, is
// max(fma(m, f16(0.8), 1023.5) - 1024, 0) in f16: the fused multiply-add rounds once, to an integer
// (the spacing of f16 in [1024, 2048)), and f16(0.8) = 0.7998046875 errs by at most 0.024 at
// m = 120, inside the 0.1 margin of every rounding decision (checked for every m).
// Check-to-variable messages are offset-binary byte pairs per (edge, thread) in the L2 slab, as in
// the two-lanes-per-thread decoder.
// Saturation: the soft update keeps 8t - 7 clamp(t, +-120) without the final clamp to +-127, so a
// soft bit the reference saturates to +-127 is here any magnitude of at least 128 (or f16
// infinity). Such a value acts as +-127 everywhere it is used: its bounds 104x -+ 12984 are at least
// 328 in magnitude, so its v2c stays at least 328 (no minimum, no message-magnitude tie, the sign
// kept) and its next soft update is again at least 128 in magnitude; the hard decision reads only
// the sign. The message magnitudes are at most 96 and finite, so no infinity meets its negative.
constexpr int kZ384      = 384;
constexpr int kZH        = 192;
constexpr int kZThreads  = 192;
constexpr int kZMaxPerSm = 4;   // register budget of the launch bounds (80 registers a thread)
constexpr int kZResidentPerSm = 3; // resident CTAs per SM: shared memory (soft bits + edge tables)
constexpr int kZ19Keep   = 8;  // v2c kept in registers by rows above kZKeepDeg edges
constexpr int kZKeepDeg  = 10; // rows of up to this many edges keep v2c, address and selector

__constant__ uint32_t c_z_sp4[2][pg::kBg1Edges]; // 4 (s mod 192)
__constant__ uint32_t c_z_col[2][pg::kBg1Edges]; // byte offset of the edge's column in E
__constant__ uint32_t c_z_sel[2][pg::kBg1Edges]; // selector when j + s' >= 192

template <int NT>
struct __align__(16) smem_z_nt_t {
  uint32_t E[pg::kMaxNodes * kZH];
  uint32_t hard[(22 * kZ384) / 32];
  uint32_t red[NT / 32];
  int      s_last;
  int      s_done;
};
using smem_z_t = smem_z_nt_t<kZThreads>;

constexpr uint32_t kH0p8     = 0x3a663a66u; // f16(0.8) = 0.7998046875
constexpr uint32_t kH1023p5  = 0x63ff63ffu; // 1023.5
constexpr uint32_t kHm1024   = 0xe400e400u; // -1024

__device__ __forceinline__ uint32_t z_scale(uint32_t m)
{
  return h2_max(h2_add(h2_fma(m, kH0p8, kH1023p5), kHm1024), 0u);
}

__device__ __forceinline__ uint32_t lds_u32(const unsigned char* base, uint32_t off)
{
  return *reinterpret_cast<const uint32_t*>(base + off);
}
__device__ __forceinline__ void sts_u32(unsigned char* base, uint32_t off, uint32_t v)
{
  *reinterpret_cast<uint32_t*>(base + off) = v;
}

// Byte offset in E and byte-permute selector of edge e (global edge index) for thread j (j4 = 4 j),
// from the CTA's copy of the edge table: {4 (s mod 192), column byte offset, selector when
// j + s' >= 192, selector otherwise}.
__device__ __forceinline__ void z_edge(const uint4* __restrict__ zt, const int e, const uint32_t j4, uint32_t& adr,
                                       uint32_t& sel)
{
  const uint4    c  = zt[e];
  const uint32_t t4 = j4 + c.x;
  const uint32_t k4 = __viaddmin_u32(t4, 0u - 4u * kZH, t4); // (j + s') mod 192, times 4
  sel               = k4 == t4 ? c.w : c.z;
  adr               = k4 + c.y;
}

// The edge tables of both base graphs in shared memory (one copy per CTA, filled once per launch).
__device__ __forceinline__ void z_load_edge_tables(uint4* zt)
{
  for (int i = threadIdx.x; i < 2 * pg::kBg1Edges; i += blockDim.x) {
    const int      g = i / pg::kBg1Edges, e = i - g * pg::kBg1Edges;
    const uint32_t sw = c_z_sel[g][e];
    zt[i]             = make_uint4(c_z_sp4[g][e], c_z_col[g][e], sw, sw ^ 0x2222u);
  }
  __syncthreads();
}

// One layer (base-graph row of degree DEG, first edge e0) for thread j. Rows of up to kZKeepDeg
// edges keep each edge's v2c, address and selector from the first pass; the degree-19 rows keep
// the v2c of their first kZ19Keep edges and recompute the rest (the soft bits and messages they
// read are not yet overwritten), so that four CTAs fit an SM without spills.
template <int DEG, bool FIRST>
__device__ __forceinline__ void row_update_z(const uint4* __restrict__ zt, const int e0, const uint32_t j4, unsigned char* E,
                                             uint16_t* __restrict__ c2v_row)
{
  constexpr bool KEEP = DEG <= kZKeepDeg;
  constexpr int  NV   = KEEP ? DEG : kZ19Keep;
  uint32_t       v[NV];
  uint32_t       adr[KEEP ? DEG : 1], sel[KEEP ? DEG : 1];
  uint32_t       min1 = kH120, min2 = kH120;
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    uint32_t a, s;
    z_edge(zt, e0 + e, j4, a, s);
    if constexpr (KEEP) {
      adr[e] = a;
      sel[e] = s;
    }
    const uint32_t vv = pair_v2c<FIRST>(__byte_perm(lds_u32(E, a), 0, s), c2v_row + e * kZH);
    if (e < NV) {
      v[e < NV ? e : 0] = vv;
    }
    const uint32_t t  = h2_max_xs(min1, vv);
    min2              = h2_min_xs(min2, t);
    min1              = h2_min_xs(min1, vv);
  }
  const uint32_t m1  = min1 & kAbs;
  const uint32_t s1  = z_scale(m1);
  const uint32_t s2  = z_scale(min2 & kAbs);
  const uint32_t nds = h2_sub(s1, s2);
  const uint32_t sgn = min1 & kSign; // sign product of every v2c of the row
#pragma unroll
  for (int e = 0; e < DEG; ++e) {
    uint32_t a, s;
    if constexpr (KEEP) {
      a = adr[e];
      s = sel[e];
    } else {
      z_edge(zt, e0 + e, j4, a, s);
    }
    const uint32_t vv  = e < NV ? v[e < NV ? e : 0]
                                : pair_v2c<FIRST>(__byte_perm(lds_u32(E, a), 0, s), c2v_row + e * kZH);
    const uint32_t mag = h2_fma(nds, h2_ne(vv & kAbs, m1), s2);
    const uint32_t c   = mag ^ ((sgn ^ vv) & kSign);
    c2v_row[e * kZH] = (uint16_t)__byte_perm(h2_to_bytes_biased(c), 0, 0x0020);
    const uint32_t tt  = h2_add(c, vv);
    const uint32_t cl  = h2_min(h2_max(tt, kHm120), kH120);
    const uint32_t u   = h2_fma(cl, kHm7, h2_mul(tt, kH8));
    sts_u32(E, a, __byte_perm(u, 0, s));
  }
}

// The same layer split over the two threads of lane pair j (t = 0, 1): thread t takes edges t,
// t + 2, ... (a missing last edge of an odd-degree row contributes +120, which changes no minimum
// and no sign), the two partial (min1, min2, sign) meet through one shuffle, and each thread updates
// its own edges.
template <int DEG, bool FIRST>
__device__ __forceinline__ void row_update_z_split(const uint4* __restrict__ zt, const int e0, const uint32_t j4, const int t,
                                                   unsigned char* E, uint16_t* __restrict__ c2v_row)
{
  constexpr int  NE   = (DEG + 1) / 2;
  constexpr bool KEEP = NE <= 3; // wider rows recompute address and selector (register budget)
  uint32_t       v[NE], adr[KEEP ? NE : 1], sel[KEEP ? NE : 1];
  uint32_t       min1 = kH120, min2 = kH120;
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const int  e     = 2 * k + t;
    const bool valid = (DEG % 2) == 0 || k + 1 < NE || e < DEG;
    uint32_t   vv    = kH120;
    if (valid) {
      uint32_t a, s;
      z_edge(zt, e0 + e, j4, a, s);
      if constexpr (KEEP) {
        adr[k] = a;
        sel[k] = s;
      }
      vv = pair_v2c<FIRST>(__byte_perm(lds_u32(E, a), 0, s), c2v_row + e * kZH);
    }
    v[k]             = vv;
    const uint32_t x = h2_max_xs(min1, vv);
    min2             = h2_min_xs(min2, x);
    min1             = h2_min_xs(min1, vv);
  }
  const uint32_t o1 = __shfl_xor_sync(0xffffffffu, min1, 1);
  const uint32_t o2 = __shfl_xor_sync(0xffffffffu, min2, 1);
  min2              = h2_min_xs(h2_min_xs(min2, o2), h2_max_xs(min1, o1));
  min1              = h2_min_xs(min1, o1);
  const uint32_t m1  = min1 & kAbs;
  const uint32_t s1  = z_scale(m1);
  const uint32_t s2  = z_scale(min2 & kAbs);
  const uint32_t nds = h2_sub(s1, s2);
  const uint32_t sgn = min1 & kSign; // sign product of every v2c of the row
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const int  e     = 2 * k + t;
    const bool valid = (DEG % 2) == 0 || k + 1 < NE || e < DEG;
    if (valid) {
      uint32_t a, s;
      if constexpr (KEEP) {
        a = adr[k];
        s = sel[k];
      } else {
        z_edge(zt, e0 + e, j4, a, s);
      }
      const uint32_t vv  = v[k];
      const uint32_t mag = h2_fma(nds, h2_ne(vv & kAbs, m1), s2);
      const uint32_t c   = mag ^ ((sgn ^ vv) & kSign);
      c2v_row[e * kZH]   = (uint16_t)__byte_perm(h2_to_bytes_biased(c), 0, 0x0020);
      const uint32_t tt  = h2_add(c, vv);
      const uint32_t cl  = h2_min(h2_max(tt, kHm120), kH120);
      const uint32_t u   = h2_fma(cl, kHm7, h2_mul(tt, kH8));
      sts_u32(E, a, __byte_perm(u, 0, s));
    }
  }
}

template <bool FIRST>
__device__ __forceinline__ void row_dispatch_z_split(int deg, const uint4* zt, int e0, uint32_t j4, int t, unsigned char* E,
                                                     uint16_t* c2v_row)
{
  switch (deg) {
    case 3: row_update_z_split<3, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 4: row_update_z_split<4, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 5: row_update_z_split<5, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 6: row_update_z_split<6, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 7: row_update_z_split<7, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 8: row_update_z_split<8, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 9: row_update_z_split<9, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    case 10: row_update_z_split<10, FIRST>(zt, e0, j4, t, E, c2v_row); break;
    default: row_update_z_split<19, FIRST>(zt, e0, j4, t, E, c2v_row); break;
  }
}

template <bool FIRST>
__device__ __forceinline__ void row_dispatch_z(int deg, const uint4* zt, int e0, uint32_t j4, unsigned char* E, uint16_t* c2v_row)
{
  switch (deg) {
    case 3: row_update_z<3, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 4: row_update_z<4, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 5: row_update_z<5, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 6: row_update_z<6, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 7: row_update_z<7, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 8: row_update_z<8, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 9: row_update_z<9, FIRST>(zt, e0, j4, E, c2v_row); break;
    case 10: row_update_z<10, FIRST>(zt, e0, j4, E, c2v_row); break;
    default: row_update_z<19, FIRST>(zt, e0, j4, E, c2v_row); break;
  }
}

// f16 soft bit -> hard bit: soft <= 0 (either zero counts as 0).
__device__ __forceinline__ bool z_hard(uint32_t h)
{
  return (h & 0x8000u) != 0 || (h & 0x7fffu) == 0;
}

// Decodes codeblock cb (Z = 384) with check-to-variable slab `slab`: NT threads, T = NT / 192 per
// lane pair (T = 2: each row's edges split between the pair's two threads).
template <int NT>
__device__ void decode_codeblock_z384(const pg_ldpc_cb& d, smem_z_nt_t<NT>& sm, const uint4* __restrict__ ztab,
                                      const int8_t* __restrict__ llrs,
                                      uint8_t* __restrict__ bits, int32_t* __restrict__ iterations,
                                      int8_t* __restrict__ c2v_all, const uint32_t* __restrict__ crc_pow, const int cb,
                                      const int slab)
{
  constexpr int T = NT / kZH;
  static_assert(NT == kZH || NT == 2 * kZH, "one or two threads per lane pair");
  const int tid = threadIdx.x;
  const int bg  = d.base_graph;
  if (bg != 1 && bg != 2) {
    if (tid == 0) {
      iterations[cb] = -1;
    }
    return;
  }
  const int      g        = bg - 1;
  const uint4*   zt       = ztab + g * pg::kBg1Edges;
  const int      Kb       = bg == 1 ? 22 : 10;
  const int      nrows    = bg == 1 ? pg::kBg1Rows : pg::kBg2Rows;
  const int      nfull    = bg == 1 ? 68 : 52;
  const int      msg_len  = Kb * kZ384;
  const int      n        = (int)d.nof_llrs;
  const int8_t*  in       = llrs + d.llr_offset;
  uint16_t*      c2v      = reinterpret_cast<uint16_t*>(c2v_all + (size_t)slab * pg::kC2vStride);
  const int      nbytes   = msg_len / 8;
  uint8_t*       out      = bits + d.out_offset;
  const int      crc_poly = d.crc_poly;
  const int      nwords   = msg_len / 32;
  unsigned char* E        = reinterpret_cast<unsigned char*>(sm.E);
  const int      jp       = T == 1 ? tid : tid >> 1; // lane pair
  const int      tp       = T == 1 ? 0 : tid & 1;
  const uint32_t j4       = 4u * (uint32_t)jp;

  if (tid == 0) {
    sm.s_last = 0;
    sm.s_done = 0;
  }
  __syncthreads();

  // Soft bits as f16 pairs, eight pairs per thread step (2Z punctured zeros, then the input).
  {
    constexpr int per_col  = kZH / 8;
    const int     nchunks  = nfull * per_col;
    const int     nof_full = (n / kZ384) * kZ384;
    const bool    aligned  = (reinterpret_cast<uintptr_t>(in) & 7u) == 0;
    int           last     = 0;
#pragma unroll 2
    for (int q = tid; q < nchunks; q += NT) {
      const int col = q / per_col;
      const int w0  = (q - col * per_col) * 8;
      const int k   = (col - 2) * kZ384 + w0;
      uint32_t  l0, l1, h0, h1;
      fetch8(in, k, n, nof_full, aligned, last, l0, l1);
      fetch8(in, k + kZH, n, nof_full, aligned, last, h0, h1);
      const uint32_t p0 = __byte_perm(l0, h0, 0x5140), p1 = __byte_perm(l0, h0, 0x7362);
      const uint32_t p2 = __byte_perm(l1, h1, 0x5140), p3 = __byte_perm(l1, h1, 0x7362);
      uint4          a, b;
      a.x = bytes_to_h2(p0);
      a.y = bytes_to_h2(p0 >> 16);
      a.z = bytes_to_h2(p1);
      a.w = bytes_to_h2(p1 >> 16);
      b.x = bytes_to_h2(p2);
      b.y = bytes_to_h2(p2 >> 16);
      b.z = bytes_to_h2(p3);
      b.w = bytes_to_h2(p3 >> 16);
      *reinterpret_cast<uint4*>(sm.E + col * kZH + w0)     = a;
      *reinterpret_cast<uint4*>(sm.E + col * kZH + w0 + 4) = b;
    }
    last = warp_max(last);
    if ((tid & 31) == 0 && last > 0) {
      atomicMax(&sm.s_last, last);
    }
  }
  __syncthreads();

  const int input_size = sm.s_last;
  if (input_size < msg_len) {
    for (int b = tid; b < nbytes; b += NT) {
      out[b] = 0xff;
    }
    if (tid == 0) {
      iterations[cb] = 0;
    }
    __syncthreads();
    return;
  }
  int cb_len = max(input_size + 2 * kZ384, (Kb + 4) * kZ384);
  cb_len     = ((cb_len + kZ384 - 1) / kZ384) * kZ384;
  const int nof_layers = min(cb_len / kZ384 - Kb, nrows);

  int order = 24;
  if (crc_poly == PG_CRC16) {
    order = 16;
  }
  const uint32_t* pow_tab = crc_pow + (size_t)(crc_poly <= PG_CRC24B ? crc_poly : 0) * pg::kCrcPowLen;
  const int       crc_len = msg_len - (int)d.nof_filler_bits;

  int       result = 0;
  const int max_it = d.max_iterations;
  const int lane   = tid & 31;
  const int nsteps = steps_for_layers(g, nof_layers);
  for (int it = 0; it < max_it; ++it) {
    for (int st = 0; st < nsteps; ++st) {
      if (it > 0 || st + 1 == nsteps) {
        prefetch_step(g, st + 1 < nsteps ? st + 1 : 0, nof_layers, tid, reinterpret_cast<const char*>(c2v),
                      kZH * 2);
      }
      const int r0 = c_step_row0[g][st];
      const int r1 = min(r0 + (int)c_step_nrows[g][st], nof_layers);
      for (int r = r0; r < r1; ++r) {
        const int deg     = c_row_deg[g][r];
        const int e0      = c_row_e0[g][r];
        uint16_t* c2v_row = c2v + (size_t)e0 * kZH + jp;
        if (T == 1) {
          if (it == 0) {
            row_dispatch_z<true>(deg, zt, e0, j4, E, c2v_row);
          } else {
            row_dispatch_z<false>(deg, zt, e0, j4, E, c2v_row);
          }
        } else {
          if (it == 0) {
            row_dispatch_z_split<true>(deg, zt, e0, j4, tp, E, c2v_row);
          } else {
            row_dispatch_z_split<false>(deg, zt, e0, j4, tp, E, c2v_row);
          }
        }
      }
      __syncthreads();
    }

    // Hard decisions (soft <= 0), zero check and CRC: one 32-bit word per warp step, lane k
    // holding bit 32 wi + k (MSB first after the reversal); message bit i of column c = i / 384,
    // lane w = i mod 384 is half (w >= 192) of E[c][w mod 192].
    int      zero = 0;
    uint32_t crc  = 0;
    for (int wi = tid >> 5; wi < nwords; wi += NT / 32) {
      const int      idx = 32 * wi + lane;
      const int      col = idx / kZ384;
      const int      w   = idx - col * kZ384;
      const uint32_t x   = sm.E[col * kZH + (w < kZH ? w : w - kZH)];
      const uint32_t h   = w < kZH ? (x & 0xffffu) : (x >> 16);
      const bool     bit = z_hard(h);
      zero |= (h & 0x7fffu) == 0;
      const uint32_t wd = __brev(__ballot_sync(0xffffffffu, bit));
      if (lane == 0) {
        sm.hard[wi] = wd;
      }
      if (crc_poly != PG_CRC_NONE && bit && idx < crc_len) {
        crc ^= __ldg(pow_tab + (crc_len - 1 - idx + order));
      }
    }
    zero = __syncthreads_or(zero);
    crc  = warp_xor(crc);
    if (lane == 0) {
      sm.red[tid >> 5] = crc;
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t t = 0;
      for (int w = 0; w < NT / 32; ++w) {
        t ^= sm.red[w];
      }
      sm.s_done = (crc_poly != PG_CRC_NONE && !zero && t == 0) ? 1 : 0;
    }
    __syncthreads();
    if (sm.s_done) {
      result = it + 1;
      break;
    }
  }

  if (crc_poly == PG_CRC_NONE) {
    // Syndrome check over the processed rows (ldpc_decoder_impl.cpp:329-387), both lanes.
    int bad = 0;
    int e0  = 0;
    for (int r = 0; r < nof_layers && tid < kZH; ++r) {
      const int deg    = c_row_deg[g][r];
      uint32_t  parity = 0;
      for (int e = 0; e < deg; ++e) {
        uint32_t a, s;
        z_edge(zt, e0 + e, 4u * (uint32_t)tid, a, s);
        const uint32_t x  = __byte_perm(lds_u32(E, a), 0, s);
        const uint32_t lo = x & 0xffffu, hi = x >> 16;
        bad |= ((lo & 0x7fffu) == 0) | ((hi & 0x7fffu) == 0);
        parity ^= (uint32_t)z_hard(lo) | ((uint32_t)z_hard(hi) << 1);
      }
      bad |= parity != 0;
      e0 += deg;
    }
    bad      = __syncthreads_or(bad);
    int zero = 0;
    for (int i = tid; i < msg_len; i += NT) {
      const int      col = i / kZ384;
      const int      w   = i - col * kZ384;
      const uint32_t x   = sm.E[col * kZH + (w < kZH ? w : w - kZH)];
      zero |= (((w < kZH ? x : x >> 16) & 0x7fffu) == 0);
    }
    zero   = __syncthreads_or(zero);
    result = (!bad && !zero) ? max_it : 0;
  }

  for (int b = tid; b < nbytes; b += NT) {
    out[b] = (uint8_t)(sm.hard[b >> 2] >> (24 - 8 * (b & 3)));
  }
  if (tid == 0) {
    iterations[cb] = result;
  }
  __syncthreads();
}

constexpr size_t kZSmem = sizeof(smem_z_t) > kX2Smem ? sizeof(smem_z_t) : kX2Smem;

// Persistent decoder of a work list, every lifting size: Z = 384 through decode_codeblock_z384,
// other even Z > 192 in pair mode, Z <= 192 with the one-lane arithmetic (192 threads, four CTAs
// per SM).
__global__ void __launch_bounds__(kZThreads, kZMaxPerSm) ldpc_decode_z_kernel(const pg_ldpc_cb* __restrict__ descs,
                                                                      const int8_t* __restrict__ llrs,
                                                                      uint8_t* __restrict__ bits,
                                                                      int32_t* __restrict__ iterations,
                                                                      int8_t* __restrict__ c2v_all,
                                                                      const uint32_t* __restrict__ crc_pow,
                                                                      const uint16_t* __restrict__ scale_tab,
                                                                      const uint32_t* __restrict__ order, int n,
                                                                      int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_z_raw[];
  __shared__ int   s_work;
  __shared__ uint4 s_ztab[2 * pg::kBg1Edges];
  z_load_edge_tables(s_ztab);
  for (;;) {
    if (threadIdx.x == 0) {
      s_work = atomicAdd(counter, 1);
    }
    __syncthreads();
    const int w = s_work;
    __syncthreads();
    if (w >= n) {
      break;
    }
    const int        cb = order != nullptr ? (int)order[w] : w;
    const pg_ldpc_cb d  = descs[cb];
    if (d.lifting_size == kZ384) {
      decode_codeblock_z384<kZThreads>(d, *reinterpret_cast<smem_z_t*>(smem_z_raw), s_ztab, llrs, bits, iterations,
                                       c2v_all, crc_pow, cb, blockIdx.x);
    } else if (d.lifting_size > kX2Threads) {
      decode_codeblock_pair<kX2Threads, 1>(d, *reinterpret_cast<smem_pair_t*>(smem_z_raw), llrs, bits, iterations,
                                           c2v_all, crc_pow, scale_tab, cb, blockIdx.x);
    } else {
      decode_codeblock<0, kX2Threads, kX2Threads>(d, *reinterpret_cast<smem_x2_scalar_t*>(smem_z_raw), llrs, bits,
                                                  iterations, c2v_all, crc_pow, cb, blockIdx.x);
      __syncthreads();
    }
  }
}

// The Z = 384 decoder with two threads per lane pair (384 threads, two CTAs per SM): each row's
// edges are split between the pair, which halves the latency of a layer, for batches whose time is
// set by their slowest codeblocks. Other lifting sizes as ldpc_decode_split_kernel.
constexpr int    kZsThreads  = 2 * kZH;
constexpr int    kZsMaxPerSm = 2;
constexpr size_t kZsSmem     = std::max(sizeof(smem_z_nt_t<kZsThreads>), kSplitSmem);

__global__ void __launch_bounds__(kZsThreads, kZsMaxPerSm) ldpc_decode_zs_kernel(
    const pg_ldpc_cb* __restrict__ descs, const int8_t* __restrict__ llrs, uint8_t* __restrict__ bits,
    int32_t* __restrict__ iterations, int8_t* __restrict__ c2v_all, const uint32_t* __restrict__ crc_pow,
    const uint16_t* __restrict__ scale_tab, const uint32_t* __restrict__ order, int n, int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_zs_raw[];
  __shared__ int   s_work;
  __shared__ uint4 s_ztab[2 * pg::kBg1Edges];
  z_load_edge_tables(s_ztab);
  for (;;) {
    if (threadIdx.x == 0) {
      s_work = atomicAdd(counter, 1);
    }
    __syncthreads();
    const int w = s_work;
    __syncthreads();
    if (w >= n) {
      break;
    }
    const int        cb = order != nullptr ? (int)order[w] : w;
    const pg_ldpc_cb d  = descs[cb];
    if (d.lifting_size == kZ384) {
      decode_codeblock_z384<kZsThreads>(d, *reinterpret_cast<smem_z_nt_t<kZsThreads>*>(smem_zs_raw), s_ztab, llrs,
                                        bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
    } else if (d.lifting_size > kX2Threads && (d.lifting_size & 1) == 0) {
      decode_codeblock_pair<kSplitThreads, 2>(d, *reinterpret_cast<smem_split_pair_t*>(smem_zs_raw), llrs, bits,
                                              iterations, c2v_all, crc_pow, scale_tab, cb, blockIdx.x);
    } else {
      decode_codeblock<0, kSplitThreads, pg::kMaxZ>(d, *reinterpret_cast<smem_split_scalar_t*>(smem_zs_raw), llrs,
                                                    bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
      __syncthreads();
    }
  }
}

// Persistent decoder of a work list, every lifting size: each CTA takes the next work index from
// *counter, decodes codeblock order[w] (or w) in pair mode (even Z > 192) or scalar mode (Z <= 192)
// with slab blockIdx.x, and stops when the n codeblocks are taken.
__global__ void __launch_bounds__(kX2Threads, kX2MaxPerSm) ldpc_decode_x2_kernel(const pg_ldpc_cb* __restrict__ descs,
                                                                        const int8_t* __restrict__ llrs,
                                                                        uint8_t* __restrict__ bits,
                                                                        int32_t* __restrict__ iterations,
                                                                        int8_t* __restrict__ c2v_all,
                                                                        const uint32_t* __restrict__ crc_pow,
                                                                        const uint16_t* __restrict__ scale_tab,
                                                                        const uint32_t* __restrict__ order, int n,
                                                                        int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_x2_raw[];
  __shared__ int s_work;
  for (;;) {
    if (threadIdx.x == 0) {
      s_work = atomicAdd(counter, 1);
    }
    __syncthreads();
    const int w = s_work;
    __syncthreads();
    if (w >= n) {
      break;
    }
    const int        cb = order != nullptr ? (int)order[w] : w;
    const pg_ldpc_cb d  = descs[cb];
    if (d.lifting_size > kX2Threads) {
      decode_codeblock_pair<kX2Threads, 1>(d, *reinterpret_cast<smem_pair_t*>(smem_x2_raw), llrs, bits, iterations,
                                           c2v_all, crc_pow, scale_tab, cb, blockIdx.x);
    } else {
      decode_codeblock<0, kX2Threads, kX2Threads>(d, *reinterpret_cast<smem_x2_scalar_t*>(smem_x2_raw), llrs, bits,
                                                  iterations, c2v_all, crc_pow, cb, blockIdx.x);
      __syncthreads();
    }
  }
}

// Persistent split decoder of a work list, every lifting size: 384 threads per codeblock, pair mode
// with two threads per lane pair for even Z > 192, the one-lane arithmetic otherwise.
__global__ void __launch_bounds__(kSplitThreads, kSplitMaxPerSm) ldpc_decode_split_kernel(
    const pg_ldpc_cb* __restrict__ descs, const int8_t* __restrict__ llrs, uint8_t* __restrict__ bits,
    int32_t* __restrict__ iterations, int8_t* __restrict__ c2v_all, const uint32_t* __restrict__ crc_pow,
    const uint16_t* __restrict__ scale_tab, const uint32_t* __restrict__ order, int n, int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_split_raw[];
  __shared__ int s_work;
  for (;;) {
    if (threadIdx.x == 0) {
      s_work = atomicAdd(counter, 1);
    }
    __syncthreads();
    const int w = s_work;
    __syncthreads();
    if (w >= n) {
      break;
    }
    const int        cb = order != nullptr ? (int)order[w] : w;
    const pg_ldpc_cb d  = descs[cb];
    if (d.lifting_size > kX2Threads && (d.lifting_size & 1) == 0) {
      decode_codeblock_pair<kSplitThreads, 2>(d, *reinterpret_cast<smem_split_pair_t*>(smem_split_raw), llrs, bits,
                                              iterations, c2v_all, crc_pow, scale_tab, cb, blockIdx.x);
    } else if (d.lifting_size == 384) {
      decode_codeblock<384, kSplitThreads, pg::kMaxZ>(d, *reinterpret_cast<smem_split_scalar_t*>(smem_split_raw), llrs,
                                                      bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
      __syncthreads();
    } else {
      decode_codeblock<0, kSplitThreads, pg::kMaxZ>(d, *reinterpret_cast<smem_split_scalar_t*>(smem_split_raw), llrs,
                                                    bits, iterations, c2v_all, crc_pow, cb, blockIdx.x);
      __syncthreads();
    }
  }
}


// Longest-first work order of a batch for the persistent decoders. A codeblock's expected decoding
// time is its work per iteration (the edges of the check rows its input reaches, as the decoder
// counts them from the last non-zero LLR, times Z) times the iterations it needs, which fall as its
// information per message bit rises: the sum of its LLR magnitudes over its K = Kb Z message bits
// (the mean LLR magnitude over the code rate; on the 512-codeblock BG1/BG2 batch the iterations
// correlate with it at -0.9 within each graph). Cost = edges Z K / sum |LLR|; the key is
// 255 - 16 log2(1 + cost), clamped to 0..255 (no non-zero LLR: 255), and the order lists the
// codeblocks by ascending key, so that the long decodes start first and the short ones fill the
// tail. The order only schedules: every codeblock's result is independent of it. One CTA per
// codeblock reads its whole input, 16 bytes per load in the aligned body.
constexpr int kScoreThreads = 128;

__device__ __forceinline__ void score_word(uint32_t w, int idx, uint32_t& sum, uint32_t& cnt, int& last)
{
  const uint32_t a  = __vabsss4(w);                    // |x| per byte (saturating, -128 -> 127)
  const uint32_t nz = __vcmpne4(w, 0u) & 0x01010101u;  // 1 per non-zero byte
  sum               = __dp4a(a, 0x01010101u, sum);
  cnt               = __dp4a(nz, 0x01010101u, cnt);
  if (w != 0) {
    last = max(last, idx + 4 - (__clz(w) >> 3));     // one past the highest non-zero byte
  }
}

__global__ void __launch_bounds__(kScoreThreads) ldpc_score_kernel(const pg_ldpc_cb* __restrict__ descs, int n,
                                                                  const int8_t* __restrict__ llrs,
                                                                  uint8_t* __restrict__ keys)
{
  __shared__ uint32_t s_red[3][kScoreThreads / 32];
  const pg_ldpc_cb d    = descs[blockIdx.x];
  const int8_t*    in   = llrs + d.llr_offset;
  const int        len  = (int)d.nof_llrs;
  const int        head = min(len, (int)((16u - (unsigned)(reinterpret_cast<uintptr_t>(in) & 15u)) & 15u));
  const int        nvec = (len - head) / 16;
  uint32_t         sum = 0, cnt = 0;
  int              last = 0;
  for (int k = threadIdx.x; k < head; k += kScoreThreads) {
    score_word((uint32_t)(uint8_t)__ldg(in + k), k, sum, cnt, last);
  }
  const uint4* body = reinterpret_cast<const uint4*>(in + head);
  for (int q = threadIdx.x; q < nvec; q += kScoreThreads) {
    const uint4 v  = __ldg(body + q);
    const int   k0 = head + 16 * q;
    score_word(v.x, k0, sum, cnt, last);
    score_word(v.y, k0 + 4, sum, cnt, last);
    score_word(v.z, k0 + 8, sum, cnt, last);
    score_word(v.w, k0 + 12, sum, cnt, last);
  }
  for (int k = head + 16 * nvec + threadIdx.x; k < len; k += kScoreThreads) {
    score_word((uint32_t)(uint8_t)__ldg(in + k), k, sum, cnt, last);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_red[0][threadIdx.x >> 5] = sum;
    s_red[1][threadIdx.x >> 5] = cnt;
    s_red[2][threadIdx.x >> 5] = (uint32_t)last;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ts = 0, tc = 0;
    int      tl = 0;
    for (int w = 0; w < kScoreThreads / 32; ++w) {
      ts += s_red[0][w];
      tc += s_red[1][w];
      tl = max(tl, (int)s_red[2][w]);
    }
    uint32_t key = 255u;
    if (tc > 0) {
      const int   Z    = max(1, (int)d.lifting_size);
      const int   Kb   = d.base_graph == 1 ? 22 : 10;
      const int   nr   = d.base_graph == 1 ? pg::kBg1Rows : pg::kBg2Rows;
      const int   rows  = min(max((tl + 2 * Z) / Z, Kb + 4) - Kb, nr);
      const int   edges = c_row_e0[d.base_graph == 2 ? 1 : 0][rows];
      const float cost  = (float)edges * (float)Z * (float)(Kb * Z) / (float)max(ts, 1u);
      key               = 255u - (uint32_t)min(255.f, 16.f * log2f(1.f + cost));
    }
    keys[blockIdx.x] = (uint8_t)key;
  }
  (void)n;
}

// Counting sort of the keys in one CTA: order[0..n) = codeblocks by ascending key.
__global__ void __launch_bounds__(1024) ldpc_sort_kernel(const uint8_t* __restrict__ keys, int n,
                                                         uint32_t* __restrict__ order)
{
  __shared__ uint32_t bin[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    bin[i] = 0;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    atomicAdd(&bin[keys[k]], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // Exclusive prefix sum of the 256 bins: eight per lane, then across the warp.
    uint32_t v[8], t = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[i] = bin[8 * threadIdx.x + i];
      t += v[i];
    }
    uint32_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      inc += threadIdx.x >= (unsigned)o ? y : 0u;
    }
    uint32_t run = inc - t;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      bin[8 * threadIdx.x + i] = run;
      run += v[i];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    order[atomicAdd(&bin[keys[k]], 1u)] = (uint32_t)k;
  }
}

} // namespace

// Check-to-variable scratch of pg_ldpc_decode_batch_static_scratch (described with that entry).
static __device__ __align__(256) int8_t g_static_c2v[(size_t)PG_STATIC_SCRATCH_MAX_CODEBLOCKS * pg::kC2vStride];

namespace pg {

int lifting_set_index(int Z)
{
  static const int a_tab[8] = {2, 3, 5, 7, 9, 11, 13, 15};
  if (Z < 2 || Z > kMaxZ) {
    return -1;
  }
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

int ldpc_upload_tables(pg_context* ctx)
{
  uint8_t  col[2][kBg1Edges] = {};
  uint16_t v[2][kBg1Edges][8] = {};
  uint8_t  deg[2][kBg1Rows]   = {};
  for (int e = 0; e < PG_BG1_EDGES; ++e) {
    col[0][e] = PG_BG1_EDGE_COL[e];
    for (int s = 0; s < 8; ++s) {
      v[0][e][s] = PG_BG1_EDGE_V[e][s];
    }
  }
  for (int e = 0; e < PG_BG2_EDGES; ++e) {
    col[1][e] = PG_BG2_EDGE_COL[e];
    for (int s = 0; s < 8; ++s) {
      v[1][e][s] = PG_BG2_EDGE_V[e][s];
    }
  }
  for (int r = 0; r < PG_BG1_ROWS; ++r) {
    deg[0][r] = PG_BG1_ROW_DEG[r];
  }
  for (int r = 0; r < PG_BG2_ROWS; ++r) {
    deg[1][r] = PG_BG2_ROW_DEG[r];
  }
  // Scale table of the two-lanes-per-thread decoder: f16 bits of (m * 52428) >> 16 at (f16 bits of
  // m) >> 4, m = 0 .. 127.
  uint16_t scale[kScaleTab] = {};
  for (int m = 0; m <= 127; ++m) {
    const uint16_t key = __half_as_ushort(__float2half_rn((float)m)) >> 4;
    scale[key]         = __half_as_ushort(__float2half_rn((float)((m * 52428) >> 16)));
  }
  // Edge tables of the Z = 384 decoder (lifting set index 1): 4 (s mod 192), the column's byte
  // offset in the f16-pair soft bits and the byte-permute selector of the wrapped case (halves
  // swapped unless s >= 192).
  uint32_t z_sp4[2][kBg1Edges] = {}, z_col[2][kBg1Edges] = {}, z_sel[2][kBg1Edges] = {};
  for (int gi = 0; gi < 2; ++gi) {
    const int ne = gi == 0 ? PG_BG1_EDGES : PG_BG2_EDGES;
    for (int e = 0; e < ne; ++e) {
      const uint32_t s = (uint32_t)v[gi][e][1] % (uint32_t)kZ384;
      z_sp4[gi][e]     = 4u * (s % (uint32_t)kZH);
      z_col[gi][e]     = 4u * (uint32_t)kZH * col[gi][e];
      z_sel[gi][e]     = s >= (uint32_t)kZH ? 0x3210u : 0x1032u;
    }
  }
  int rc = check_cuda(ctx, cudaMemcpyToSymbol(c_edge_col, col, sizeof(col)), "cudaMemcpyToSymbol(edge_col)");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_z_sp4, z_sp4, sizeof(z_sp4)), "cudaMemcpyToSymbol(z_sp4)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_z_col, z_col, sizeof(z_col)), "cudaMemcpyToSymbol(z_col)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_z_sel, z_sel, sizeof(z_sel)), "cudaMemcpyToSymbol(z_sel)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaFuncSetAttribute(ldpc_decode_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kZSmem),
                    "cudaFuncSetAttribute(ldpc_decode_z_kernel)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaFuncSetAttribute(ldpc_decode_zs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kZsSmem),
                    "cudaFuncSetAttribute(ldpc_decode_zs_kernel)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.ldpc_scale, sizeof(scale)), "cudaMalloc(scale table)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpy(ctx->dev.ldpc_scale, scale, sizeof(scale), cudaMemcpyHostToDevice),
                    "cudaMemcpy(scale table)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaFuncSetAttribute(ldpc_decode_x2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kX2Smem),
                    "cudaFuncSetAttribute(ldpc_decode_x2_kernel)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaFuncSetAttribute(ldpc_decode_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSplitSmem),
                    "cudaFuncSetAttribute(ldpc_decode_split_kernel)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_edge_v, v, sizeof(v)), "cudaMemcpyToSymbol(edge_v)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_row_deg, deg, sizeof(deg)), "cudaMemcpyToSymbol(row_deg)");
  }
  // Layer steps: greedy runs of consecutive rows with pairwise disjoint columns.
  uint8_t  step_row0[2][kBg1Rows] = {}, step_nrows[2][kBg1Rows] = {}, nsteps[2] = {};
  uint16_t row_e0[2][kBg1Rows + 1] = {};
  for (int gi = 0; gi < 2; ++gi) {
    const int rows = gi == 0 ? PG_BG1_ROWS : PG_BG2_ROWS;
    for (int r = 0; r < rows; ++r) {
      row_e0[gi][r + 1] = (uint16_t)(row_e0[gi][r] + deg[gi][r]);
    }
    uint64_t used[2] = {0, 0}; // columns 0..67 of the current step
    int      ns      = 0;
    for (int r = 0; r < rows; ++r) {
      uint64_t cols[2] = {0, 0};
      for (int e = row_e0[gi][r]; e < row_e0[gi][r + 1]; ++e) {
        cols[col[gi][e] >> 6] |= 1ull << (col[gi][e] & 63);
      }
      if (r == 0 || (cols[0] & used[0]) != 0 || (cols[1] & used[1]) != 0) {
        step_row0[gi][ns]  = (uint8_t)r;
        step_nrows[gi][ns] = 1;
        ++ns;
        used[0] = cols[0];
        used[1] = cols[1];
      } else {
        ++step_nrows[gi][ns - 1];
        used[0] |= cols[0];
        used[1] |= cols[1];
      }
    }
    nsteps[gi] = (uint8_t)ns;
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_step_row0, step_row0, sizeof(step_row0)), "cudaMemcpyToSymbol(steps)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_step_nrows, step_nrows, sizeof(step_nrows)), "cudaMemcpyToSymbol(steps)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_nsteps, nsteps, sizeof(nsteps)), "cudaMemcpyToSymbol(steps)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyToSymbol(c_row_e0, row_e0, sizeof(row_e0)), "cudaMemcpyToSymbol(row_e0)");
  }
  if (rc == PG_OK) {
    // Device address of the static scratch on this context's device (current here), looked up
    // once so that the static-scratch entry makes no runtime call besides its launch.
    rc = check_cuda(ctx, cudaGetSymbolAddress((void**)&ctx->static_c2v, g_static_c2v),
                    "cudaGetSymbolAddress(static check-to-variable scratch)");
  }
  return rc;
}

int ldpc_launch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                int32_t* iterations, cudaStream_t stream)
{
  return ldpc_launch_scratch(ctx, descs_dev, n, llrs, bits, iterations, ctx->dev.c2v, stream);
}

int ldpc_launch_scratch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                        int32_t* iterations, int8_t* c2v, cudaStream_t stream)
{
  const uint32_t* order = nullptr;
  if (ctx->ldpc_order_mode == PG_LDPC_ORDER_LONGEST_FIRST && n > 1 && n <= ctx->max_codeblocks) {
    if (int rc = ldpc_order_launch(ctx, descs_dev, n, llrs, ctx->dev.ldpc_keys, ctx->dev.ldpc_order, stream)) {
      return rc;
    }
    order = ctx->dev.ldpc_order;
  }
  return ldpc_launch_persistent(ctx, descs_dev, n, llrs, bits, iterations, c2v, order, ctx->dev.ldpc_counter, stream);
}

int ldpc_order_launch(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* keys,
                      uint32_t* order, cudaStream_t stream)
{
  if (n <= 0) {
    return PG_OK;
  }
  ldpc_score_kernel<<<n, kScoreThreads, 0, stream>>>(descs_dev, n, llrs, keys);
  if (int rc = check_cuda(ctx, cudaGetLastError(), "ldpc_score_kernel launch")) {
    return rc;
  }
  ldpc_sort_kernel<<<1, 1024, 0, stream>>>(keys, n, order);
  return check_cuda(ctx, cudaGetLastError(), "ldpc_sort_kernel launch");
}

unsigned int timing_record_flags(pg_context* ctx, cudaStream_t s)
{
  // Under stream capture the timing events become event-record nodes of the graph (external
  // records); a plain record there would only mark a capture dependency.
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  if (ctx->timed && cudaStreamIsCapturing(s, &capturing) == cudaSuccess &&
      capturing == cudaStreamCaptureStatusActive) {
    return cudaEventRecordExternal;
  }
  return cudaEventRecordDefault;
}

int ldpc_resident_ctas(pg_context* ctx)
{
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ldpc_decode_kernel, kThreads, 0) != cudaSuccess ||
      per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  return per_sm * ctx->sm_count;
}

int ldpc_launch_persistent(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                           int32_t* iterations, int8_t* c2v, const uint32_t* order, int* counter,
                           cudaStream_t stream)
{
  const int per_sm = ctx->ldpc_ctas_per_sm > 0 ? ctx->ldpc_ctas_per_sm : kX2MaxPerSm;
  return ldpc_launch_persistent(ctx, descs_dev, n, llrs, bits, iterations, c2v, order, counter, stream,
                                per_sm * ctx->sm_count, PG_LDPC_KIND_ALL | ldpc_route(ctx->ldpc_kernel));
}

int ldpc_launch_persistent(pg_context* ctx, const pg_ldpc_cb* descs_dev, int n, const int8_t* llrs, uint8_t* bits,
                           int32_t* iterations, int8_t* c2v, const uint32_t* order, int* counter,
                           cudaStream_t stream, int max_ctas, int kinds)
{
  if (n == 0) {
    return PG_OK;
  }
  if (int rc = check_cuda(ctx, cudaMemsetAsync(counter, 0, 2 * sizeof(int), stream), "cudaMemsetAsync(ldpc counter)")) {
    return rc;
  }
  const unsigned int rec_flags = timing_record_flags(ctx, stream);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, stream, rec_flags);
  }
  // PG_LDPC_ROUTE_Z: the Z = 384 kernel (three per SM, pair mode and one-lane arithmetic for the
  // other lifting sizes);
  // PG_LDPC_ROUTE_SPLIT: the split kernel decodes every codeblock (two CTAs per SM);
  // PG_LDPC_ROUTE_X2: the two-lanes-per-thread kernel (four per SM); neither: ldpc_decode_kernel
  // (two per SM). The caller provides a slab per CTA (min(n, max_ctas) slabs, max_ctas <= four
  // per SM).
  int rc = PG_OK;
  if (kinds & PG_LDPC_ROUTE_ZS) {
    const int grid_zs = std::max(1, std::min(n, std::min(max_ctas, kZsMaxPerSm * ctx->sm_count)));
    ldpc_decode_zs_kernel<<<grid_zs, kZsThreads, kZsSmem, stream>>>(
        descs_dev, llrs, bits, iterations, c2v, ctx->dev.crc_pow, ctx->dev.ldpc_scale, order, n, counter + 1);
    rc = check_cuda(ctx, cudaGetLastError(), "ldpc_decode_zs_kernel launch");
  } else if (kinds & PG_LDPC_ROUTE_Z) {
    const int grid_z = std::max(1, std::min(n, std::min(max_ctas, kZResidentPerSm * ctx->sm_count)));
    ldpc_decode_z_kernel<<<grid_z, kZThreads, kZSmem, stream>>>(
        descs_dev, llrs, bits, iterations, c2v, ctx->dev.crc_pow, ctx->dev.ldpc_scale, order, n, counter + 1);
    rc = check_cuda(ctx, cudaGetLastError(), "ldpc_decode_z_kernel launch");
  } else if (kinds & PG_LDPC_ROUTE_SPLIT) {
    const int grid_s = std::max(1, std::min(n, std::min(max_ctas, kSplitMaxPerSm * ctx->sm_count)));
    ldpc_decode_split_kernel<<<grid_s, kSplitThreads, kSplitSmem, stream>>>(
        descs_dev, llrs, bits, iterations, c2v, ctx->dev.crc_pow, ctx->dev.ldpc_scale, order, n, counter + 1);
    rc = check_cuda(ctx, cudaGetLastError(), "ldpc_decode_split_kernel launch");
  } else if (kinds & PG_LDPC_ROUTE_X2) {
    const int grid_x2 = std::max(1, std::min(n, std::min(max_ctas, kX2MaxPerSm * ctx->sm_count)));
    ldpc_decode_x2_kernel<<<grid_x2, kX2Threads, kX2Smem, stream>>>(
        descs_dev, llrs, bits, iterations, c2v, ctx->dev.crc_pow, ctx->dev.ldpc_scale, order, n, counter + 1);
    rc = check_cuda(ctx, cudaGetLastError(), "ldpc_decode_x2_kernel launch");
  } else {
    const int grid = std::max(1, std::min(n, std::min(max_ctas, ctx->ldpc_ctas)));
    ldpc_decode_kernel<<<grid, kThreads, 0, stream>>>(descs_dev, llrs, bits, iterations, c2v, ctx->dev.crc_pow, order,
                                                      n, counter, 0);
    rc = check_cuda(ctx, cudaGetLastError(), "ldpc_decode_kernel launch");
  }
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, stream, rec_flags);
  }
  return rc;
}

} // namespace pg

// ---------------------------------------------------------------------------------------------
// Decoding with a module-static check-to-variable scratch (pg_ldpc_decode_batch_static_scratch).
//
// Some callers cannot allocate device memory while they decode: a PHY worker that has to finish
// each slot by its deadline (cudaMalloc / cudaFree take driver locks and may synchronise the whole
// device, so their latency has no useful bound), and a process that reserved its device memory
// when it started and must not run into out-of-memory in the middle of traffic. For them the
// scratch is a device array of this module, reserved by the driver when the module loads: room for
// PG_STATIC_SCRATCH_MAX_CODEBLOCKS codeblocks of the largest graph (BG1, Z = 384).
//
// Nothing in the array has to start at zero: the first layered iteration of each codeblock writes
// every check-to-variable message of the rows it processes before any later iteration reads one,
// so what an earlier call left behind is never read. Every call on a device uses the same array;
// kernels of two calls that run at the same time race on it. The array's device address is
// looked up once per context, in ldpc_upload_tables (called by pg_create).

extern "C" int pg_ldpc_decode_batch_static_scratch(pg_context* ctx, const pg_ldpc_cb* cbs_dev, int nof_cbs,
                                                   const int8_t* llrs, uint8_t* bits, int32_t* iterations,
                                                   void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (nof_cbs < 0) {
    return pg::set_error(ctx, PG_ERR_INVALID, "negative codeblock count");
  }
  if (nof_cbs > PG_STATIC_SCRATCH_MAX_CODEBLOCKS) {
    return pg::set_error(ctx, PG_ERR_CAPACITY,
                         "batch of " + std::to_string(nof_cbs) + " codeblocks exceeds the static scratch limit of " +
                             std::to_string(PG_STATIC_SCRATCH_MAX_CODEBLOCKS) + " codeblocks per call");
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  if (cbs_dev == nullptr || llrs == nullptr || bits == nullptr || iterations == nullptr) {
    return pg::set_error(ctx, PG_ERR_INVALID, "null device buffer");
  }
  int prev = -1;
  if (int rc = pg::check_cuda(ctx, cudaGetDevice(&prev), "cudaGetDevice")) {
    return rc;
  }
  if (prev != ctx->device) {
    if (int rc = pg::check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
      return rc;
    }
  }
  const cudaStream_t s          = static_cast<cudaStream_t>(stream);
  const unsigned int rec_flags  = pg::timing_record_flags(ctx, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, s, rec_flags);
  }
  ldpc_decode_kernel<<<nof_cbs, kThreads, 0, s>>>(cbs_dev, llrs, bits, iterations, ctx->static_c2v, ctx->dev.crc_pow,
                                                  nullptr, nof_cbs, nullptr, 0);
  int rc = pg::check_cuda(ctx, cudaGetLastError(), "ldpc_decode_kernel launch (static scratch)");
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, s, rec_flags);
  }
  if (prev != ctx->device) {
    cudaSetDevice(prev);
  }
  return rc;
}

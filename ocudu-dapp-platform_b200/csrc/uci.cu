// UCI on PUSCH for sm_100a: UL-SCH demultiplexing of HARQ-ACK and CSI Part 1 out of the
// descrambled codeword soft bits, and detection of short-block UCI messages (1 to 11 bits).
//
// Demultiplexing (lib/phy/upper/channel_processors/pusch/ulsch_demultiplex_impl.cpp:183-573,
// TS 38.212 Section 6.2.7): per OFDM symbol the reference selects, in this order, the reserved
// HARQ-ACK REs (every d-th of all REs), the HARQ-ACK REs of more than two bits (every d-th of the
// UCI REs), the CSI Part 1 REs (every d-th of the UCI REs that are neither), the HARQ-ACK REs of
// one or two bits (every d-th of the reserved REs), and leaves the rest to UL-SCH; the running
// counters that fix d and the counts carry from symbol to symbol. The host runs those counters once
// per codeword (ulsch_demux_layout) and hands each symbol's (d, count) pairs to the kernel. Every
// selection is "every d-th of a set, the first m", so a thread finds its RE's class and its rank
// in the output stream in closed form: the RE i of a symbol is the k-th selected one of a set
// that is all REs when i % d == 0 and k = i / d < m, and the number of selected REs below i is
// min(m, ceil(i / d)); CSI Part 1 ranks are the same over the REs that remain once the HARQ-ACK and
// reserved ones are taken out. One- and two-bit HARQ-ACK REs are zeroed in the UL-SCH stream
// (the reference punctures them) and, like one- and two-bit CSI Part 1, get their placeholder bits
// re-scrambled (ulsch_demultiplex_impl.cpp:86-181) from the codeword's scrambling sequence.
//
// Short blocks (lib/phy/upper/channel_coding/short/short_block_detector_impl.cpp:50-205): one warp
// per message. The soft bits are folded onto the block length with the reference's vector LLR
// sums (clipped to +-120); one bit is the sign of the first; two bits are the maximum correlation over the four
// simplex codewords; 3 to 11 bits are the maximum absolute correlation over the 2^(K-1) "even"
// Reed-Muller (32, K) codewords (the sign gives the first bit), spread over the lanes with the
// first maximum kept. Validity is the reference's generalized likelihood ratio test, computed in
// double precision on the same integers.
#include "pg_device.cuh"
#include "pg_internal.h"

#include <cmath>

#include <array>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

namespace {

#include "uci_rm_basis.inc"

__constant__ uint16_t c_rm_basis[32];

// Per-UE and per-symbol device descriptors.
struct demux_ue {
  uint32_t llr_offset, sch_offset, ack_offset, csi_offset;
  uint32_t c_init;
  uint16_t sym0, nsym; // symbols of this UE in the symbol table
  uint8_t  bpr, qm, ack_bits, csi_bits;
};
struct demux_sym {
  uint32_t in0, sch0, ack0, csi0; // soft-bit offsets at the symbol's first RE (codeword and streams)
  uint32_t ue;                    // index into the UE table
  uint16_t nre;                   // REs of the symbol that carry UL-SCH or UCI
  uint16_t rvd_d, rvd_m, ack_d, ack_m, csi_d, csi_m, ack2_d, ack2_m;
  uint16_t pad;
};

__device__ __forceinline__ uint32_t sel_below(uint32_t i, uint32_t d, uint32_t m)
{
  return m == 0 ? 0u : min(m, (i + d - 1) / d);
}
__device__ __forceinline__ bool sel_at(uint32_t i, uint32_t d, uint32_t m)
{
  return m != 0 && (i % d) == 0 && (i / d) < m;
}

// Copies the soft bits of one RE, re-scrambling the placeholder bits of a one- or two-bit UCI
// message (bits 1..2) and zeroing the source when the RE is punctured.
__device__ __forceinline__ void copy_re(const int8_t* __restrict__ src, int8_t* __restrict__ dst, int bpr, int qm,
                                        int uci_bits, uint32_t scr)
{
  for (int b = 0; b < bpr; ++b) {
    int       v = src[b];
    const int k = b % qm;
    if (uci_bits == 1 && qm > 1) {
      if (k == 1) {
        v = (((scr >> (b - 1)) ^ (scr >> b)) & 1u) ? -v : v;
      } else if (k >= 2) {
        v = ((scr >> b) & 1u) ? -v : v;
      }
    } else if (uci_bits == 2 && qm > 1 && k >= 2) {
      v = ((scr >> b) & 1u) ? -v : v;
    }
    dst[b] = (int8_t)v;
  }
}

// Copies n bytes from src to dst with the CTA: 32-bit destination words assembled from the two
// aligned source words that cover them (funnel shift), bytes at both ends. Every aligned source word
// read holds at least one byte of [src - 3, src + n).
__device__ __forceinline__ void copy_bytes_cta(int8_t* __restrict__ dst, const int8_t* __restrict__ src, uint32_t n)
{
  const uint32_t head = min(n, (4u - (uint32_t)(reinterpret_cast<uintptr_t>(dst) & 3u)) & 3u);
  if (threadIdx.x < head) {
    dst[threadIdx.x] = src[threadIdx.x];
  }
  dst += head;
  src += head;
  n -= head;
  const uint32_t  nw = n / 4;
  const uint32_t  sh = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 3u);
  const uint32_t* sw = reinterpret_cast<const uint32_t*>(src - sh);
  uint32_t*       dw = reinterpret_cast<uint32_t*>(dst);
  // The last word and the tail go byte by byte, so that no word beyond src + n is read.
  const uint32_t nfast = nw > 0 ? nw - 1 : 0;
  for (uint32_t w = threadIdx.x; w < nfast; w += blockDim.x) {
    const uint32_t lo = __ldg(sw + w);
    const uint32_t hi = sh ? __ldg(sw + w + 1) : 0u;
    dw[w]             = __funnelshift_r(lo, hi, 8u * sh);
  }
  for (uint32_t b = 4 * nfast + threadIdx.x; b < n; b += blockDim.x) {
    dst[b] = src[b];
  }
}

// One CTA per work item (symbol index, RE range [r0, r1) of at most kDemuxChunk REs), so that
// every thread handles at most one RE and the CTA issues its loads in one round.
constexpr uint32_t kDemuxChunk = 256;

__global__ void ulsch_demux_kernel(const demux_ue* __restrict__ ues, const demux_sym* __restrict__ syms,
                                   const uint2* __restrict__ items, const int8_t* __restrict__ llrs,
                                   int8_t* __restrict__ sch, int8_t* __restrict__ ack, int8_t* __restrict__ csi,
                                   const uint32_t* __restrict__ gold)
{
  const uint2     item = items[blockIdx.x];
  const demux_sym sd   = syms[item.x];
  const demux_ue  ud   = ues[sd.ue];
  const int       bpr  = ud.bpr;
  const uint32_t  r0 = item.y & 0xffffu, r1 = item.y >> 16;
  if (sd.rvd_m == 0 && sd.ack_m == 0 && sd.csi_m == 0) {
    // No UCI in this symbol: its soft bits go to UL-SCH unchanged.
    copy_bytes_cta(sch + ud.sch_offset + sd.sch0 + r0 * (uint32_t)bpr, llrs + ud.llr_offset + sd.in0 + r0 * (uint32_t)bpr,
                   (r1 - r0) * (uint32_t)bpr);
    return;
  }
  for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const bool     rvd   = sel_at(i, sd.rvd_d, sd.rvd_m);
    const bool     ack3  = sel_at(i, sd.ack_d, sd.ack_m);
    const uint32_t avail = i - sel_below(i, sd.ack_d, sd.ack_m) - sel_below(i, sd.rvd_d, sd.rvd_m);
    const bool     csi1  = !rvd && !ack3 && sel_at(avail, sd.csi_d, sd.csi_m);
    const uint32_t k_rvd = rvd ? i / sd.rvd_d : 0u;
    const bool     ack2  = rvd && sel_at(k_rvd, sd.ack2_d, sd.ack2_m);
    const uint32_t pos   = sd.in0 + i * (uint32_t)bpr; // codeword soft-bit index of the RE
    const int8_t*  src   = llrs + ud.llr_offset + pos;
    uint32_t       scr   = 0;
    if ((ack2 && ud.ack_bits <= 2) || (csi1 && ud.csi_bits <= 2)) {
      scr = pg::gold_word(gold, pg::kGoldWords, ud.c_init, pos);
    }
    if (ack3) {
      copy_re(src, ack + ud.ack_offset + sd.ack0 + (i / sd.ack_d) * bpr, bpr, ud.qm, 0, 0);
    } else if (csi1) {
      copy_re(src, csi + ud.csi_offset + sd.csi0 + (avail / sd.csi_d) * bpr, bpr, ud.qm,
              ud.csi_bits <= 2 ? ud.csi_bits : 0, scr);
    } else {
      if (ack2) {
        copy_re(src, ack + ud.ack_offset + sd.ack0 + (k_rvd / sd.ack2_d) * bpr, bpr, ud.qm, ud.ack_bits, scr);
      }
      const uint32_t rank = i - sel_below(i, sd.ack_d, sd.ack_m) - sel_below(avail, sd.csi_d, sd.csi_m);
      int8_t*        dst  = sch + ud.sch_offset + sd.sch0 + rank * bpr;
      for (int b = 0; b < bpr; ++b) {
        dst[b] = ack2 ? (int8_t)0 : src[b];
      }
    }
  }
}

// Sum of the reference's LLR vector addition (log_likelihood_ratio::sum,
// lib/phy/upper/log_likelihood_ratio.cpp:414-486, the x86 vector path of every block): saturated
// int8 addition clipped to +-120.
__device__ __forceinline__ int llr_sum(int a, int b)
{
  return max(-120, min(120, a + b));
}

struct short_item {
  uint32_t llr_offset, nof_llrs, out_offset;
  uint8_t  nof_bits, qm, pad[2];
};

// One warp per message.
__global__ void uci_short_block_kernel(const short_item* __restrict__ items, int n, const int8_t* __restrict__ llrs,
                                       uint8_t* __restrict__ bits, uint8_t* __restrict__ valid)
{
  const int w    = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n) {
    return;
  }
  const short_item it = items[w];
  const int        K  = it.nof_bits;
  const int        E  = (int)it.nof_llrs;
  const int        qm = it.qm;
  const int8_t*    in = llrs + it.llr_offset;
  uint8_t*         out = bits + it.out_offset;

  // Validity of the spans (short_block_detector_impl.cpp:42-64).
  int nz = 0;
  for (int i = lane; i < E; i += 32) {
    nz += in[i] != 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nz += __shfl_xor_sync(0xffffffffu, nz, o);
  }
  const int min_bits[11] = {2, 3, 9, 10, 11, 12, 13, 14, 14, 15, 17};
  const bool ok_spans = K >= 1 && K <= 11 && nz >= min_bits[max(1, min(K, 11)) - 1] && (K > 2 || E >= qm);
  if (!ok_spans) {
    for (int j = lane; j < K; j += 32) {
      out[j] = 1;
    }
    if (lane == 0) {
      valid[w] = 0;
    }
    return;
  }

  // Fold onto the block length L (rate dematching, short_block_detector_impl.cpp:131-158): lane
  // j < L sums positions j, j + L, j + 2L, ... in order.
  const int L   = K == 1 ? qm : (K == 2 ? 3 * qm : 32);
  int       acc = 0;
  if (lane < L) {
    acc = lane < E ? (int)in[lane] : 0;
    for (int i = lane + L; i < E; i += L) {
      acc = llr_sum(acc, in[i]);
    }
  }

  if (K == 1) {
    const int t0 = __shfl_sync(0xffffffffu, acc, 0);
    if (lane == 0) {
      out[0]   = t0 > 0 ? 0 : 1;
      valid[w] = 1; // the reference's metric 1 against threshold 0
    }
    return;
  }

  if (K == 2) {
    // detect_2 (short_block_detector_impl.cpp:66-108) on lane 0 from the folded block.
    int t[24];
#pragma unroll
    for (int j = 0; j < 24; ++j) {
      t[j] = __shfl_sync(0xffffffffu, acc, j);
    }
    if (lane == 0) {
      int l[3];
      if (L == 3) {
        l[0] = t[0];
        l[1] = t[1];
        l[2] = t[2];
      } else {
        const int step = L / 3 - 2;
        l[0]           = t[0] + t[step + 3];
        l[1]           = t[1] + t[2 * step + 4];
        l[2]           = t[step + 2] + t[2 * step + 5];
      }
      const int tab[4][3] = {{1, 1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, 1}};
      int       idx       = 0;
      double    best      = DBL_MIN;
      for (int c = 0; c < 4; ++c) {
        const int m = l[0] * tab[c][0] + l[1] * tab[c][1] + l[2] * tab[c][2];
        if ((double)m > best) {
          best = m;
          idx  = c;
        }
      }
      out[0]            = idx & 1;
      out[1]            = (idx >> 1) & 1;
      const double m2   = __dmul_rn(best, best);
      const int    norm = l[0] * l[0] + l[1] * l[1] + l[2] * l[2];
      const double met  = __ddiv_rn(__dmul_rn(2.0, m2), __dsub_rn(__dmul_rn(3.0, (double)norm), m2));
      valid[w]          = met > 0.0 ? 1 : 0;
    }
    return;
  }

  // 3..11 bits: correlations with the even codewords, lane-strided over the codeword index.
  const int ncw  = 1 << (K - 1);
  int       best = 0, best_idx = 0x7fffffff, best_sign = 0;
  const int tl   = acc; // folded soft bit of position `lane`
  for (int base = 0; base < ncw; base += 32) {
    const int idx = base + lane;
    // Every lane needs all 32 folded soft bits; they are shuffled in once per codeword.
    int metric = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int      x = __shfl_sync(0xffffffffu, tl, i);
      const uint32_t c = __popc(((uint32_t)idx << 1) & (uint32_t)c_rm_basis[i]) & 1u;
      metric += c ? -x : x;
    }
    if (idx < ncw) {
      const int a = abs(metric);
      if (a > best) {
        best      = a;
        best_idx  = idx;
        best_sign = metric < 0;
      }
    }
  }
  // First maximum over the lanes (largest |metric|, then smallest index).
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, best_idx, o);
    const int os = __shfl_xor_sync(0xffffffffu, best_sign, o);
    if (ob > best || (ob == best && oi < best_idx)) {
      best      = ob;
      best_idx  = oi;
      best_sign = os;
    }
  }
  int norm = tl * tl;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    norm += __shfl_xor_sync(0xffffffffu, norm, o);
  }
  if (best == 0) { // no positive correlation: the reference keeps index 0 and metric DBL_MIN
    best_idx  = 0;
    best_sign = 0;
  }
  const uint32_t msg = 2u * (uint32_t)best_idx + (uint32_t)best_sign;
  for (int j = lane; j < K; j += 32) {
    out[j] = (msg >> j) & 1u;
  }
  if (lane == 0) {
    const double bm  = best == 0 ? DBL_MIN : (double)best;
    const double m2  = __dmul_rn(bm, bm);
    const double met = __ddiv_rn(__dmul_rn(31.0, m2), __dsub_rn((double)(32u * (uint32_t)norm), m2));
    const double thr[11] = {0, 0, 12, 14, 16, 18, 20, 22, 24, 26, 29};
    valid[w]             = met > thr[K - 1] ? 1 : 0;
  }
}

} // namespace

namespace pg {

int uci_upload_tables(pg_context* ctx)
{
  return check_cuda(ctx, cudaMemcpyToSymbol(c_rm_basis, PG_UCI_RM_BASIS, sizeof(PG_UCI_RM_BASIS)),
                    "cudaMemcpyToSymbol(rm basis)");
}

} // namespace pg

namespace {

struct demux_layout {
  std::vector<demux_sym> syms;
  uint32_t               sizes[3] = {0, 0, 0}; // UL-SCH, HARQ-ACK, CSI Part 1 soft bits
};

// The reference's per-symbol counters (ulsch_demultiplex_impl.cpp:183-412) for one codeword.
// Returns an error text, empty when the configuration is consistent.
std::string ulsch_demux_layout(const pg_ulsch_demux_config& c, demux_layout& out)
{
  const unsigned qm = c.modulation_order;
  if (qm != 1 && qm != 2 && qm != 4 && qm != 6 && qm != 8) {
    return "modulation order must be 1, 2, 4, 6 or 8";
  }
  if (c.nof_layers < 1 || c.nof_layers > 4) {
    return "1 to 4 layers";
  }
  if (c.nof_prb < 1 || c.nof_prb > 275 || c.start_symbol_index + c.nof_symbols > 14 || c.nof_symbols < 1) {
    return "allocation outside the slot";
  }
  if (c.dmrs_type != 1 && c.dmrs_type != 2) {
    return "DM-RS type must be 1 or 2";
  }
  const unsigned max_cdm = c.dmrs_type == 1 ? 2u : 3u;
  if (c.nof_cdm_groups_without_data < 1 || c.nof_cdm_groups_without_data > max_cdm) {
    return "invalid number of CDM groups without data";
  }
  if ((c.dmrs_symbol_mask & 0x3fffu) == 0) {
    return "no DM-RS symbol";
  }
  if (c.nof_harq_ack_bits > 1706 || c.nof_csi_part1_bits > 1706) {
    return "UCI messages of more than 1706 bits";
  }
  if (c.nof_harq_ack_rvd != 0 && c.nof_harq_ack_bits > 2) {
    return "reserved HARQ-ACK bits apply to messages of at most two bits";
  }
  const unsigned bpr = qm * c.nof_layers;
  if (c.nof_harq_ack_rvd % bpr || c.nof_enc_harq_ack_bits % bpr || c.nof_enc_csi_part1_bits % bpr) {
    return "encoded UCI sizes must be multiples of the soft bits per RE";
  }
  if ((c.nof_harq_ack_bits == 0) != (c.nof_enc_harq_ack_bits == 0) ||
      (c.nof_csi_part1_bits == 0) != (c.nof_enc_csi_part1_bits == 0)) {
    return "UCI message and encoded sizes must be both zero or both non-zero";
  }
  // l1: first symbol without DM-RS after the first DM-RS symbol; l1_csi: first without DM-RS.
  const unsigned mask  = c.dmrs_symbol_mask & 0x3fffu;
  unsigned       first = 0;
  while (!((mask >> first) & 1u)) {
    ++first;
  }
  unsigned l1 = first;
  while (l1 < 14 && ((mask >> l1) & 1u)) {
    ++l1;
  }
  unsigned l1_csi = 0;
  while (l1_csi < 14 && ((mask >> l1_csi) & 1u)) {
    ++l1_csi;
  }
  const unsigned re_dmrs = (12u - c.nof_cdm_groups_without_data * (c.dmrs_type == 1 ? 6u : 4u)) * c.nof_prb;
  unsigned       m_rvd = 0, m_ack = 0, m_csi = 0;
  uint32_t       in = 0, sch = 0, ack = 0, csi = 0;
  for (unsigned sym = c.start_symbol_index; sym < c.start_symbol_index + c.nof_symbols; ++sym) {
    const bool     dm      = (mask >> sym) & 1u;
    const unsigned m_ulsch = dm ? re_dmrs : 12u * c.nof_prb;
    unsigned       m_uci   = dm ? 0u : m_ulsch;
    demux_sym      s{};
    s.in0 = in;
    s.sch0 = sch;
    s.ack0 = ack;
    s.csi0 = csi;
    s.nre  = (uint16_t)m_ulsch;
    s.rvd_d = s.ack_d = s.csi_d = s.ack2_d = 1;
    // Step 1: reserved REs.
    const unsigned rem_rvd = (c.nof_harq_ack_rvd - m_rvd) / bpr;
    if (sym >= l1 && m_uci > 0 && rem_rvd > 0) {
      unsigned d = 1, m = m_uci;
      if (rem_rvd < m_uci) {
        d = m_uci / rem_rvd;
        m = rem_rvd;
      }
      s.rvd_d = (uint16_t)d;
      s.rvd_m = (uint16_t)m;
      m_rvd += m * bpr;
    }
    // Step 2: HARQ-ACK of more than two bits.
    const unsigned rem_ack = (c.nof_enc_harq_ack_bits - m_ack) / bpr;
    if (sym >= l1 && m_uci > 0 && c.nof_harq_ack_bits > 2 && rem_ack > 0) {
      unsigned d = 1, m = m_uci;
      if (rem_ack < m_uci) {
        d = m_uci / rem_ack;
        m = rem_ack;
      }
      s.ack_d = (uint16_t)d;
      s.ack_m = (uint16_t)m;
      m_uci -= m;
      m_ack += m * bpr;
    }
    // Step 3: CSI Part 1 over the UCI REs that are not reserved.
    const unsigned rem_csi = (c.nof_enc_csi_part1_bits - m_csi) / bpr;
    const unsigned m_res   = s.rvd_m;
    if (sym >= l1_csi && m_uci > m_res && rem_csi > 0) {
      const unsigned avail = m_uci - m_res;
      unsigned       d = 1, m = avail;
      if (rem_csi < avail) {
        d = avail / rem_csi;
        m = rem_csi;
      }
      s.csi_d = (uint16_t)d;
      s.csi_m = (uint16_t)m;
      m_csi += m * bpr;
    }
    // Step 5: HARQ-ACK of at most two bits, from the reserved REs.
    if (m_res > 0 && c.nof_harq_ack_bits <= 2 && rem_ack > 0) {
      unsigned d = 1, m = m_res;
      if (rem_ack < m_res) {
        d = m_res / rem_ack;
        m = rem_ack;
      }
      s.ack2_d = (uint16_t)d;
      s.ack2_m = (uint16_t)m;
      m_ack += m * bpr;
    }
    in += m_ulsch * bpr;
    sch += (m_ulsch - s.ack_m - s.csi_m) * bpr;
    ack += (s.ack_m + s.ack2_m) * bpr;
    csi += s.csi_m * bpr;
    if (m_ulsch > 0) {
      out.syms.push_back(s);
    }
  }
  if (m_ack != c.nof_enc_harq_ack_bits || m_csi != c.nof_enc_csi_part1_bits || m_rvd != c.nof_harq_ack_rvd) {
    return "the encoded UCI does not fit the allocation";
  }
  if (in != c.nof_llrs) {
    return "nof_llrs is not the codeword size of the allocation (" + std::to_string(in) + ")";
  }
  if ((uint64_t)in + 64 > (uint64_t)(pg::kGoldWords - 2) * 32u) {
    return "codeword longer than the scrambling table";
  }
  out.sizes[0] = sch;
  out.sizes[1] = ack;
  out.sizes[2] = csi;
  return "";
}

} // namespace

using namespace pg;

namespace pg {

std::string uci_demux_blob(const pg_ulsch_demux_config* cfgs, int n, std::vector<uint8_t>& blob, uci_demux_work& w,
                           std::vector<std::array<uint32_t, 3>>* sizes)
{
  if (sizes != nullptr) {
    sizes->assign((size_t)n, std::array<uint32_t, 3>{0, 0, 0});
  }
  std::vector<demux_ue>  ues(n);
  std::vector<demux_sym> syms;
  for (int u = 0; u < n; ++u) {
    demux_layout      L;
    const std::string err = ulsch_demux_layout(cfgs[u], L);
    if (!err.empty()) {
      return "UE " + std::to_string(u) + ": " + err;
    }
    if (sizes != nullptr) {
      for (int k = 0; k < 3; ++k) {
        (*sizes)[u][k] = L.sizes[k];
      }
    }
    demux_ue& d  = ues[u];
    d.llr_offset = cfgs[u].llr_offset;
    d.sch_offset = cfgs[u].sch_offset;
    d.ack_offset = cfgs[u].harq_ack_offset;
    d.csi_offset = cfgs[u].csi_part1_offset;
    d.c_init     = cfgs[u].c_init;
    d.sym0       = (uint16_t)syms.size();
    d.nsym       = (uint16_t)L.syms.size();
    d.bpr        = (uint8_t)(cfgs[u].modulation_order * cfgs[u].nof_layers);
    d.qm         = cfgs[u].modulation_order;
    d.ack_bits   = (uint8_t)std::min<unsigned>(cfgs[u].nof_harq_ack_bits, 255u); // only <= 2 matters
    d.csi_bits   = (uint8_t)std::min<unsigned>(cfgs[u].nof_csi_part1_bits, 255u);
    for (demux_sym sy : L.syms) {
      sy.ue = (uint32_t)u;
      syms.push_back(sy);
    }
  }
  std::vector<uint2> items;
  for (size_t k = 0; k < syms.size(); ++k) {
    for (uint32_t r0 = 0; r0 < syms[k].nre; r0 += kDemuxChunk) {
      const uint32_t r1 = std::min<uint32_t>(syms[k].nre, r0 + kDemuxChunk);
      items.push_back(make_uint2((uint32_t)k, r0 | (r1 << 16)));
    }
  }
  // [UEs | symbols | items], the items (8-byte vectors) on a 16-byte boundary.
  const size_t b_ues = ues.size() * sizeof(demux_ue), b_syms = syms.size() * sizeof(demux_sym);
  w.o_syms           = b_ues;
  w.o_items          = (b_ues + b_syms + 15) & ~(size_t)15;
  w.nitems           = (int)items.size();
  blob.assign(w.o_items + items.size() * sizeof(uint2), 0);
  std::memcpy(blob.data(), ues.data(), b_ues);
  std::memcpy(blob.data() + b_ues, syms.data(), b_syms);
  std::memcpy(blob.data() + w.o_items, items.data(), items.size() * sizeof(uint2));
  return std::string();
}

int uci_demux_launch(pg_context* ctx, const void* blob_dev, const uci_demux_work& w, const int8_t* llrs, int8_t* sch,
                     int8_t* harq_ack, int8_t* csi_part1, cudaStream_t s)
{
  if (w.nitems == 0) {
    return PG_OK;
  }
  const uint8_t* b = static_cast<const uint8_t*>(blob_dev);
  ulsch_demux_kernel<<<(unsigned)w.nitems, kDemuxChunk, 0, s>>>(
      reinterpret_cast<const demux_ue*>(b), reinterpret_cast<const demux_sym*>(b + w.o_syms),
      reinterpret_cast<const uint2*>(b + w.o_items), llrs, sch, harq_ack, csi_part1, ctx->dev.gold);
  return check_cuda(ctx, cudaGetLastError(), "ulsch_demux_kernel launch");
}

std::string uci_short_blob(const pg_uci_short_block* items, int n, std::vector<uint8_t>& blob)
{
  std::vector<short_item> v(n);
  for (int i = 0; i < n; ++i) {
    const pg_uci_short_block& it = items[i];
    const unsigned            qm = it.modulation_order;
    if (it.nof_bits < 1 || it.nof_bits > 11) {
      return "message " + std::to_string(i) + ": 1 to 11 bits";
    }
    if (qm != 1 && qm != 2 && qm != 4 && qm != 6 && qm != 8) {
      return "message " + std::to_string(i) + ": invalid modulation order";
    }
    v[i] = short_item{it.llr_offset, it.nof_llrs, it.out_offset, it.nof_bits, (uint8_t)qm, {0, 0}};
  }
  blob.resize(v.size() * sizeof(short_item));
  std::memcpy(blob.data(), v.data(), blob.size());
  return std::string();
}

int uci_detect_launch(pg_context* ctx, const void* items_dev, int n, const int8_t* llrs, uint8_t* bits, uint8_t* valid,
                      cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  const unsigned warps_per_cta = 4;
  uci_short_block_kernel<<<(unsigned)((n + warps_per_cta - 1) / warps_per_cta), 32 * warps_per_cta, 0, s>>>(
      static_cast<const short_item*>(items_dev), n, llrs, bits, valid);
  return check_cuda(ctx, cudaGetLastError(), "uci_short_block_kernel launch");
}

} // namespace pg

namespace {

// CRC bits attached to a UCI payload of n bits (TS 38.212 Section 6.3.2.1 via 5.2.1): none up to 11
// bits, CRC6 up to 19, CRC11 above.
unsigned uci_crc_bits(unsigned n)
{
  return n < 12 ? 0u : (n < 20 ? 6u : 11u);
}

// Resource elements of one UCI field with UL-SCH (TS 38.212 Sections 6.3.2.4.1.1-3): the
// beta-offset share of the UCI-capable REs over the UL-SCH codeblock bits, capped. The single
// precision and the operation order are those of lib/ran/pusch/ulsch_info.cpp:12-135, so that a
// value on a rounding boundary gives the same count.
unsigned uci_re_with_sch(unsigned bits, float beta, unsigned re_uci, unsigned sum_cb)
{
  return (unsigned)std::ceil((float)(bits + uci_crc_bits(bits)) * beta * (float)re_uci / (float)sum_cb);
}

unsigned uci_re_without_sch(unsigned bits, float beta, float rate, unsigned qm)
{
  return (unsigned)std::ceil((float)(bits + uci_crc_bits(bits)) * beta / (rate * (float)qm));
}

} // namespace

extern "C" {

int pg_ulsch_information(const pg_ulsch_info_config* cfg, pg_ulsch_info* out)
{
  if (cfg == nullptr || out == nullptr) {
    return PG_ERR_INVALID;
  }
  const pg_ulsch_info_config& c = *cfg;
  const unsigned qm = c.modulation_order, nl = c.nof_layers;
  const uint32_t alloc = ((1u << (c.start_symbol + c.nof_symbols)) - 1u) & ~((1u << c.start_symbol) - 1u);
  const uint32_t dm    = c.dmrs_symbol_mask & 0x3fffu;
  const bool     sch   = c.tbs_bits > 0;
  if (!(qm == 1 || qm == 2 || qm == 4 || qm == 6 || qm == 8) || nl < 1 || nl > 4 || c.nof_rb == 0 ||
      c.nof_symbols == 0 || c.start_symbol + c.nof_symbols > 14 || dm == 0 || (dm & ~alloc) != 0 ||
      c.nof_cdm_groups_without_data < 1 || c.nof_cdm_groups_without_data > 2 ||
      (sch && c.base_graph != 1 && c.base_graph != 2) || (!sch && !(c.target_code_rate > 0.f && c.target_code_rate < 1.f))) {
    return PG_ERR_INVALID;
  }
  // Codeblocks of the UL-SCH: sum of K_r (including filler bits), TS 38.212 Section 5.2.2.
  const unsigned nd         = (unsigned)__builtin_popcount(dm);
  const unsigned re_dmrs_rb = nd * c.nof_cdm_groups_without_data * 6u; // DM-RS type 1: 6 REs per CDM group
  const unsigned re_total   = c.nof_rb * (c.nof_symbols * 12u - re_dmrs_rb);
  unsigned       sum_cb     = 0;
  if (sch) {
    pg_sch_segmentation seg = {};
    if (pg_sch_segment(c.tbs_bits, c.base_graph, qm, (int)nl, re_total * nl, &seg) != PG_OK) {
      return PG_ERR_INVALID;
    }
    sum_cb = seg.nof_cbs * seg.cb_length;
  }
  const unsigned re_uci     = (c.nof_symbols - nd) * c.nof_rb * 12u;
  // UCI-capable REs from the first DM-RS symbol on.
  unsigned re_uci_l0 = 0;
  for (unsigned s = (unsigned)__builtin_ctz(dm); s < c.start_symbol + c.nof_symbols; ++s) {
    re_uci_l0 += ((dm >> s) & 1u) ? 0u : c.nof_rb * 12u;
  }
  const unsigned cap_ack = (unsigned)std::ceil(c.alpha_scaling * (float)re_uci_l0);
  auto ack_re = [&](unsigned bits) {
    if (bits == 0) {
      return 0u;
    }
    const unsigned left = sch ? uci_re_with_sch(bits, c.beta_offset_harq_ack, re_uci, sum_cb)
                              : uci_re_without_sch(bits, c.beta_offset_harq_ack, c.target_code_rate, qm);
    return std::min(left, cap_ack);
  };
  const unsigned harq_re = ack_re(c.nof_harq_ack_bits);
  // Up to two HARQ-ACK bits reserve the REs of two.
  unsigned rvd_re = 0;
  if (c.nof_harq_ack_bits < 2) {
    rvd_re = ack_re(2);
  } else if (c.nof_harq_ack_bits == 2) {
    rvd_re = harq_re;
  }
  const unsigned ack_for_csi1 = c.nof_harq_ack_bits <= 2 ? rvd_re : harq_re;
  unsigned       csi1_re      = 0;
  if (c.nof_csi_part1_bits > 0) {
    if (sch) {
      const unsigned left  = uci_re_with_sch(c.nof_csi_part1_bits, c.beta_offset_csi_part1, re_uci, sum_cb);
      const unsigned right = (unsigned)std::ceil(c.alpha_scaling * (float)re_uci) - ack_for_csi1;
      csi1_re              = std::min(left, right);
    } else if (c.nof_csi_part2_bits == 0) {
      csi1_re = re_uci - ack_for_csi1;
    } else {
      csi1_re = std::min(uci_re_without_sch(c.nof_csi_part1_bits, c.beta_offset_csi_part1, c.target_code_rate, qm),
                         re_uci - ack_for_csi1);
    }
  }
  const unsigned ack_for_csi2 = c.nof_harq_ack_bits <= 2 ? 0u : harq_re;
  unsigned       csi2_re      = 0;
  if (c.nof_csi_part2_bits > 0) {
    if (sch) {
      const unsigned left  = uci_re_with_sch(c.nof_csi_part2_bits, c.beta_offset_csi_part2, re_uci, sum_cb);
      const unsigned right = (unsigned)std::ceil(c.alpha_scaling * (float)re_uci) - ack_for_csi2 - csi1_re;
      csi2_re              = std::min(left, right);
    } else {
      csi2_re = re_uci - ack_for_csi2 - csi1_re;
    }
  }
  const unsigned ack_used = c.nof_harq_ack_bits > 2 ? harq_re : 0u;
  const unsigned sch_re   = sch ? re_total - ack_used - csi1_re - csi2_re : 0u;
  const unsigned per_re   = nl * qm;
  *out                     = pg_ulsch_info{};
  out->nof_ul_sch_bits     = sch_re * per_re;
  out->nof_harq_ack_bits   = harq_re * per_re;
  out->nof_harq_ack_rvd    = rvd_re * per_re;
  out->nof_csi_part1_bits  = csi1_re * per_re;
  out->nof_csi_part2_bits  = csi2_re * per_re;
  out->nof_harq_ack_re     = harq_re;
  out->nof_csi_part1_re    = csi1_re;
  out->nof_csi_part2_re    = csi2_re;
  out->nof_dc_overlap_bits = c.contains_dc ? c.nof_symbols * qm : 0u;
  return PG_OK;
}

int pg_ulsch_demultiplex_sizes(const pg_ulsch_demux_config* cfg, uint32_t* sizes)
{
  if (cfg == nullptr || sizes == nullptr) {
    return PG_ERR_INVALID;
  }
  demux_layout L;
  if (!ulsch_demux_layout(*cfg, L).empty()) {
    return PG_ERR_INVALID;
  }
  sizes[0] = L.sizes[0];
  sizes[1] = L.sizes[1];
  sizes[2] = L.sizes[2];
  return PG_OK;
}

int pg_ulsch_demultiplex_device(pg_context* ctx, const pg_ulsch_demux_config* cfgs, int n, const int8_t* llrs,
                                int8_t* sch, int8_t* harq_ack, int8_t* csi_part1, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (n < 0 || (n > 0 && (cfgs == nullptr || llrs == nullptr || sch == nullptr))) {
    return set_error(ctx, PG_ERR_INVALID, "null argument");
  }
  std::vector<uint8_t>                 blob;
  uci_demux_work                       w;
  std::vector<std::array<uint32_t, 3>> sizes;
  const std::string                    err = uci_demux_blob(cfgs, n, blob, w, &sizes);
  if (!err.empty()) {
    return set_error(ctx, PG_ERR_INVALID, err);
  }
  for (int u = 0; u < n; ++u) {
    if ((sizes[u][1] > 0 && harq_ack == nullptr) || (sizes[u][2] > 0 && csi_part1 == nullptr)) {
      return set_error(ctx, PG_ERR_INVALID, "UE " + std::to_string(u) + ": null UCI output");
    }
  }
  if (w.nitems == 0) {
    return PG_OK;
  }
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  void*        dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_UCI, blob.data(), blob.size(), s, &dev)) {
    return rc;
  }
  const unsigned int rec = timing_record_flags(ctx, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, s, rec);
  }
  const int rc = uci_demux_launch(ctx, dev, w, llrs, sch, harq_ack, csi_part1, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, s, rec);
  }
  // The staged blob stays in use until the kernel has read it.
  return rc != PG_OK ? rc : release_slot_after(ctx, SLOT_UCI, s);
}

int pg_uci_short_block_detect_device(pg_context* ctx, const pg_uci_short_block* items, int n, const int8_t* llrs,
                                     uint8_t* bits, uint8_t* valid, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (n < 0 || (n > 0 && (items == nullptr || llrs == nullptr || bits == nullptr || valid == nullptr))) {
    return set_error(ctx, PG_ERR_INVALID, "null argument");
  }
  if (n == 0) {
    return PG_OK;
  }
  std::vector<uint8_t> blob;
  const std::string    err = uci_short_blob(items, n, blob);
  if (!err.empty()) {
    return set_error(ctx, PG_ERR_INVALID, err);
  }
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  void*        dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_UCI_SHORT, blob.data(), blob.size(), s, &dev)) {
    return rc;
  }
  const unsigned int rec = timing_record_flags(ctx, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, s, rec);
  }
  const int rc = uci_detect_launch(ctx, dev, n, llrs, bits, valid, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, s, rec);
  }
  return rc != PG_OK ? rc : release_slot_after(ctx, SLOT_UCI_SHORT, s);
}

} // extern "C"

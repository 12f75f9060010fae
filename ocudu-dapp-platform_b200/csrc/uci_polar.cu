// Polar-coded UCI on PUSCH (HARQ-ACK or CSI Part 1 of 12 to 1706 bits): the reference's
// uci_decoder_impl::decode_codeword_polar (lib/phy/upper/channel_processors/uci/uci_decoder_impl.cpp:25-99)
// with its polar code construction (lib/phy/upper/channel_coding/polar/polar_code_impl.cpp:330-480),
// rate dematcher (polar_rate_dematcher_impl.cpp), simplified successive-cancellation decoder
// (polar_decoder_impl.cpp) and deallocator (polar_deallocator_impl.cpp), on the GPU.
//
// The host builds each codeblock's code (N, the information and parity-check sub-channels) once
// per call; one CTA of two warps decodes one message, one warp per codeblock (a message longer than
// 359 bits with at least 1088 soft bits, or of 1013 bits and more, has two codeblocks). A warp runs
// the whole chain on its codeblock in shared memory: channel de-interleaving, bit selection and
// sub-block de-interleaving into the decoder's input, the decoder's depth-first walk over rate-0,
// rate-1 and rate-R nodes with the f / g / re-encoding steps spread over the 32 lanes, the
// deallocation and the codeblock CRC. Every LLR operation is the reference's int8 arithmetic
// (log_likelihood_ratio: saturated sum at +-120 with +-127 as infinity, soft_xor, hard bit v <= 0,
// promotion sum on repetition).
#include "pg_internal.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace {

#include "polar_tables.inc"

__constant__ uint8_t c_polar_subblock[32] = {PG_POLAR_SUBBLOCK_PATTERN};

constexpr int kPolarNMax   = 1024; // polar_code::NMAX
constexpr int kPolarEMax   = 8192; // polar_code::EMAX
constexpr int kPolarNMaxLg = 10;   // uplink nMax
constexpr int kPolarMaxA   = 1706; // uci_decoder_impl MAX_CODEBLOCK_SIZE (TS 38.212 5.2.1)

// One codeblock as the decoding warp reads it.
struct polar_cb {
  uint32_t llr_offset; // first soft bit of the codeblock
  uint32_t E;          // rate-matched length (0: no codeblock)
  uint32_t out_offset; // first output byte of the payload bits
  uint16_t K;          // polar K: filler + payload + CRC bits
  uint16_t nbits;      // payload bits
  uint8_t  n;          // log2 N
  uint8_t  crc_size;   // 6 or 11
  uint8_t  nof_filler; // leading zero bits of the first codeblock
  uint8_t  reserved;
  uint16_t pc[4];      // sorted parity-check sub-channels, terminated by kPolarNMax
  uint32_t info[kPolarNMax / 32]; // K_set: sub-channels that carry payload, CRC, filler or parity bits
};
static_assert(sizeof(polar_cb) == 156, "polar_cb layout");

// The code of one codeblock: polar_code_impl::set_code_params (polar_code_impl.cpp:330-421) and
// polar_code_impl::set (:432-480) for nMax = 10 (uplink).
struct polar_code_host {
  int      n = 0, N = 0, K = 0, E = 0, nPC = 0, nWmPC = 0;
  uint16_t pc[4]                 = {kPolarNMax, kPolarNMax, kPolarNMax, kPolarNMax};
  uint32_t info[kPolarNMax / 32] = {};
};

uint16_t subblock_index(int j, int N)
{
  const int b = N / 32;
  return (uint16_t)(kPolarSubblock[(32 * j) / N] * b + j % b);
}

std::string polar_code_build(unsigned K, unsigned E, polar_code_host& c)
{
  if (E > (unsigned)kPolarEMax) {
    return "E above 8192";
  }
  if (K < 18 || (K > 25 && K < 31) || K > 1023) {
    return "K out of the uplink range (18..25, 31..1023)";
  }
  c.K     = (int)K;
  c.E     = (int)E;
  c.nPC   = K <= 25 ? 3 : 0;
  c.nWmPC = (K <= 25 && E > K + 189) ? 1 : 0;
  if (!(K + (unsigned)c.nPC < E)) {
    return "E not above K + nPC";
  }
  unsigned e = 1;
  for (; e <= 13; ++e) {
    if ((1u << e) >= E) {
      break;
    }
  }
  const unsigned n1 = ((8 * E <= 9 * (1u << (e - 1))) && (16 * K < 9 * E)) ? e - 1 : e;
  unsigned       k  = 0;
  for (; k <= 10; ++k) {
    if ((1u << k) >= K) {
      break;
    }
  }
  unsigned n = std::min(n1, k + 3);
  n          = std::min(n, (unsigned)kPolarNMaxLg);
  n          = std::max(n, 5u);
  c.n        = (int)n;
  c.N        = 1 << n;
  const int N = c.N;
  if (!((int)K < N)) {
    return "K not below N";
  }
  // The sequence for N (ascending reliability).
  std::vector<uint16_t> mother;
  mother.reserve(N);
  for (int i = 0; i < kPolarNMax; ++i) {
    if (kPolarQ[i] < N) {
      mother.push_back(kPolarQ[i]);
    }
  }
  const int             nk = (int)K + c.nPC;
  std::vector<uint16_t> kset(mother.end() - nk, mother.end());
  if (N > (int)E) {
    // Sub-channels frozen by puncturing or shortening, then the stable set difference that also
    // drops every index <= T (polar_code_impl.cpp:443-467, setdiff_stable :284-313).
    unsigned              T  = 0;
    const int             nf = N - (int)E;
    std::vector<uint16_t> fset(nf);
    if (16 * K <= 7 * E) {
      const unsigned nth = 3u * (unsigned)N / 4u;
      T                  = E >= nth ? nth - (E >> 1) - 1 : 9u * (unsigned)N / 16u - (E >> 2);
      for (int i = 0; i < nf; ++i) {
        fset[i] = subblock_index(i, N);
      }
    } else {
      for (int i = 0; i < nf; ++i) {
        fset[i] = subblock_index((int)E + i, N);
      }
    }
    std::vector<uint8_t> frozen(N, 0);
    for (const uint16_t x : fset) {
      frozen[x] = 1;
    }
    std::vector<uint16_t> kept;
    for (const uint16_t x : mother) {
      if (x <= T || frozen[x] != 0) {
        continue;
      }
      kept.push_back(x);
    }
    if ((int)kept.size() < nk) {
      return "too few sub-channels left after puncturing or shortening";
    }
    kset.assign(kept.end() - nk, kept.end());
  }
  // Parity-check sub-channels: the nPC - nWmPC least reliable of K_set, and 252 (K <= 21) or 248
  // for the minimum-weight one (polar_code_impl.cpp:469-480).
  for (int i = 0; i < c.nPC - c.nWmPC; ++i) {
    c.pc[i] = kset[i];
  }
  if (c.nWmPC == 1) {
    c.pc[c.nPC - 1] = K <= 21 ? 252 : 248;
  }
  std::sort(c.pc, c.pc + c.nPC);
  for (const uint16_t x : kset) {
    c.info[x >> 5] |= 1u << (x & 31);
  }
  return std::string();
}

// UCI segmentation and CRC size (include/ocudu/ran/uci/uci_info.h:22-47).
int uci_nof_codeblocks(unsigned A, unsigned E)
{
  return ((A >= 360 && E >= 1088) || A >= 1013) ? 2 : 1;
}
int uci_crc_size(unsigned A)
{
  return A < 12 ? 0 : (A < 20 ? 6 : 11);
}

// ---------------------------------------------------------------------------------------------
// Device side.

constexpr int kLlrMax = 120;
constexpr int kLlrInf = 127;

// log_likelihood_ratio::operator+ (lib/phy/upper/log_likelihood_ratio.cpp:21-55): opposite values
// give 0, an infinite term wins, otherwise the sum saturated at +-120.
__device__ __forceinline__ int llr_sat_sum(int a, int b)
{
  if (a == -b) {
    return 0;
  }
  if (a > kLlrMax || a < -kLlrMax) {
    return a;
  }
  if (b > kLlrMax || b < -kLlrMax) {
    return b;
  }
  return max(-kLlrMax, min(kLlrMax, a + b));
}

// log_likelihood_ratio::promotion_sum (log_likelihood_ratio.cpp:57-70): as the saturated sum, but a
// finite sum above 120 in magnitude becomes infinite.
__device__ __forceinline__ int llr_promotion_sum(int a, int b)
{
  if (a == -b) {
    return 0;
  }
  if (a > kLlrMax || a < -kLlrMax) {
    return a;
  }
  if (b > kLlrMax || b < -kLlrMax) {
    return b;
  }
  const int t = a + b;
  return t > kLlrMax ? kLlrInf : (t < -kLlrMax ? -kLlrInf : t);
}

// log_likelihood_ratio::soft_xor: sign(x y) min(|x|, |y|).
__device__ __forceinline__ int llr_soft_xor(int x, int y)
{
  const int m = min(abs(x), abs(y));
  return x * y < 0 ? -m : m;
}

constexpr int kRate0 = 0, kRateR = 2, kRate1 = 3; // polar_decoder_impl node_rate

struct polar_warp_smem {
  int8_t   e[kPolarEMax];          // de-interleaved soft bits, then the deallocated message bits
  int8_t   llr[2 * kPolarNMax];    // stage s at offset 2^s - 1, 2^s values (s = 0 .. n)
  uint8_t  est[kPolarNMax];        // codeword estimates (partial sums)
  uint8_t  u[kPolarNMax];          // decoded sub-channel bits
  uint8_t  type[2 * kPolarNMax];   // node types, stage s at offset 2N - (2N >> s)
  uint32_t info[kPolarNMax / 32];
  uint16_t pc[4];
  int      valid;
};

// Node types of every stage (polar_decoder_impl.cpp:74-107): a leaf is rate 1 when it is in K_set,
// rate 0 otherwise; a node of stage s is rate 0 (rate 1) when both children are, rate R otherwise.
__device__ __forceinline__ void node_types(polar_warp_smem& sm, int n, int lane)
{
  const int N = 1 << n;
  for (int j = lane; j < N; j += 32) {
    sm.type[j] = ((sm.info[j >> 5] >> (j & 31)) & 1u) ? kRate1 : kRate0;
  }
  __syncwarp();
  for (int st = 1; st <= n; ++st) {
    const uint8_t* c = sm.type + (2 * N - ((2 * N) >> (st - 1)));
    uint8_t*       t = sm.type + (2 * N - ((2 * N) >> st));
    for (int j = lane; j < (N >> st); j += 32) {
      const int a = c[2 * j], b = c[2 * j + 1];
      t[j]        = (uint8_t)(a == b && a != kRateR ? a : kRateR);
    }
    __syncwarp();
  }
}

// One codeblock by one warp.
__device__ void polar_decode_codeblock(const polar_cb& d, polar_warp_smem& sm, const int8_t* __restrict__ llrs,
                                       uint8_t* __restrict__ bits)
{
  const int lane = threadIdx.x & 31;
  const int n    = d.n;
  const int N    = 1 << n;
  const int E    = (int)d.E;
  const int K    = d.K;
  const int8_t* f = llrs + d.llr_offset;

  for (int w = lane; w < kPolarNMax / 32; w += 32) {
    sm.info[w] = d.info[w];
  }
  __syncwarp();
  node_types(sm, n, lane);
  if (lane < 4) {
    sm.pc[lane] = d.pc[lane];
  }
  for (int i = lane; i < N; i += 32) {
    sm.est[i] = 0;
    sm.u[i]   = 0;
  }

  // Channel de-interleaver (polar_rate_dematcher_impl.cpp:53-79): the triangle of T rows, T the
  // smallest with T (T + 1) / 2 >= E, filled row by row: row r holds positions
  // r + c T - c (c - 1) / 2 for c = 0, 1, ... while below E, taking the input in (r, c) order.
  int T = 1;
  while (T * (T + 1) / 2 < E) {
    ++T;
  }
  int base = 0; // input index of the first entry of rows r0 ..
  for (int r0 = 0; r0 < T; r0 += 32) {
    const int r   = r0 + lane;
    int       cnt = 0;
    if (r < T) {
      int i_in = r;
      for (int c = 0; c < T - r && i_in < E; ++c) {
        ++cnt;
        i_in += T - c;
      }
    }
    int incl = cnt; // inclusive prefix of the counts over the lanes
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) {
        incl += t;
      }
    }
    const int first = base + incl - cnt;
    if (r < T) {
      int i_in = r;
      for (int c = 0; c < cnt; ++c) {
        sm.e[i_in] = f[first + c];
        i_in += T - c;
      }
    }
    base += __shfl_sync(0xffffffffu, incl, 31);
  }
  __syncwarp();

  // Bit selection (:21-50) and sub-block de-interleaving (:12-19) into the stage-n LLRs.
  int8_t* const ln = sm.llr + (N - 1);
  const bool    rep   = E >= N;
  const bool    punct = !rep && 16 * K <= 7 * E;
  for (int j = lane; j < N; j += 32) {
    int y;
    if (rep) {
      y = sm.e[j];
      for (int k = j + N; k < E; k += N) {
        y = llr_promotion_sum(y, sm.e[k]);
      }
    } else if (punct) {
      y = j < N - E ? 0 : sm.e[j - (N - E)];
    } else {
      y = j < E ? sm.e[j] : kLlrInf;
    }
    const int b = N >> 5;
    ln[c_polar_subblock[(32 * j) / N] * b + j % b] = (int8_t)y;
  }
  __syncwarp();

  // Simplified successive cancellation (polar_decoder_impl.cpp:163-316), depth first. phases holds
  // two bits per stage: 0 = node entered, 1 = left child done, 2 = right child done.
  int      s = n, j = 0;
  uint32_t phases = 0;
  for (;;) {
    const int ph     = (int)((phases >> (2 * s)) & 3u);
    bool      ascend = false;
    const int h      = (1 << s) >> 1;
    int8_t*   ls     = sm.llr + ((1 << s) - 1);
    if (ph == 0) {
      const int t = sm.type[2 * N - ((2 * N) >> s) + j];
      if (t == kRate1) {
        // Hard decisions of the node's LLRs, re-encoded into its message bits (:180-205).
        const int p0 = j << s, sz = 1 << s;
        for (int i = lane; i < sz; i += 32) {
          const uint8_t b = ls[i] <= 0 ? 1 : 0;
          sm.est[p0 + i]  = b;
          sm.u[p0 + i]    = b;
        }
        __syncwarp();
        for (int st = 1; st < sz; st <<= 1) {
          for (int i = lane; i < sz; i += 32) {
            if ((i & st) == 0) {
              sm.u[p0 + i] ^= sm.u[p0 + i + st];
            }
          }
          __syncwarp();
        }
        ascend = true;
      } else if (t == kRate0) {
        ascend = true; // bits stay zero (:163-178)
      } else {
        // f: left child's LLRs soft_xor(first half, second half) (:214-218).
        int8_t* lc = sm.llr + (h - 1);
        for (int i = lane; i < h; i += 32) {
          lc[i] = (int8_t)llr_soft_xor(ls[i], ls[i + h]);
        }
        __syncwarp();
        phases = (phases & ~(3u << (2 * s))) | (1u << (2 * s));
        --s;
        j <<= 1;
        phases &= ~(3u << (2 * s));
        continue;
      }
    } else if (ph == 1) {
      // g: right child's LLRs second half +- first half by the left child's codeword (:228-233).
      int8_t*        lc = sm.llr + (h - 1);
      const uint8_t* eb = sm.est + (j << s);
      for (int i = lane; i < h; i += 32) {
        const int x = ls[i], y = ls[i + h];
        lc[i]       = (int8_t)llr_sat_sum(y, eb[i] == 0 ? x : -x);
      }
      __syncwarp();
      phases = (phases & ~(3u << (2 * s))) | (2u << (2 * s));
      --s;
      j = 2 * j + 1;
      phases &= ~(3u << (2 * s));
      continue;
    } else {
      // Both children done: left codeword ^= right codeword (:240-252).
      uint8_t* eb = sm.est + (j << s);
      for (int i = lane; i < h; i += 32) {
        eb[i] ^= eb[i + h];
      }
      __syncwarp();
      ascend = true;
    }
    if (ascend) {
      if (s == n) {
        break;
      }
      ++s;
      j >>= 1;
    }
  }

  // Deallocation (polar_deallocator_impl.cpp:10-24) and the codeblock CRC over the K bits
  // (uci_decoder_impl.cpp:74-92), one lane.
  if (lane == 0) {
    int     iPC = 0, iK = 0;
    int8_t* msg = sm.e;
    for (int w = 0; w < (N >> 5); ++w) {
      uint32_t x = sm.info[w];
      while (x != 0u) {
        const int i = (w << 5) + __ffs(x) - 1;
        x &= x - 1u;
        if (i == sm.pc[iPC]) {
          ++iPC;
        } else if (iK < K) {
          msg[iK++] = (int8_t)sm.u[i];
        }
      }
    }
    const int      L    = d.crc_size;
    const uint32_t poly = L == 11 ? 0x621u : 0x21u; // CRC11 0xE21, CRC6 0x61 without the x^L term
    const uint32_t mask = (1u << L) - 1u;
    uint32_t       reg  = 0;
    for (int i = 0; i < K; ++i) {
      const uint32_t top = ((reg >> (L - 1)) ^ (uint32_t)msg[i]) & 1u;
      reg                = (reg << 1) & mask;
      if (top) {
        reg ^= poly;
      }
    }
    sm.valid = reg == 0u ? 1 : 0;
  }
  __syncwarp();
  for (int i = lane; i < d.nbits; i += 32) {
    bits[d.out_offset + i] = (uint8_t)sm.e[d.nof_filler + i];
  }
}

constexpr int kPolarThreads = 64; // one warp per codeblock

__global__ void __launch_bounds__(kPolarThreads) uci_polar_kernel(const polar_cb* __restrict__ cbs, int n,
                                                                 const int8_t* __restrict__ llrs,
                                                                 uint8_t* __restrict__ bits,
                                                                 uint8_t* __restrict__ valid)
{
  __shared__ polar_warp_smem sm[2];
  const int msg  = blockIdx.x;
  const int warp = threadIdx.x >> 5;
  if (msg >= n) {
    return;
  }
  const polar_cb& d = cbs[2 * msg + warp];
  if (d.E > 0) {
    polar_decode_codeblock(d, sm[warp], llrs, bits);
  } else if ((threadIdx.x & 31) == 0) {
    sm[warp].valid = 1;
  }
  __syncthreads();
  // uci_decoder_impl.cpp:40-57: valid when every codeblock passes its CRC.
  if (threadIdx.x == 0) {
    valid[msg] = (uint8_t)((sm[0].valid && sm[1].valid) ? 1 : 0);
  }
}

// The device blob of n messages: two polar_cb per message (the second with E = 0 when the message
// has one codeblock). Returns an error text for an invalid message.
std::string polar_blob_cbs(const pg_uci_polar* items, int n, std::vector<polar_cb>& cbs)
{
  cbs.assign((size_t)2 * n, polar_cb{});
  for (int i = 0; i < n; ++i) {
    const pg_uci_polar& it = items[i];
    const unsigned      A  = it.nof_bits;
    const unsigned      Et = it.nof_llrs;
    if (A < 12 || A > (unsigned)kPolarMaxA) {
      return "message " + std::to_string(i) + ": 12 to 1706 bits";
    }
    const int      C   = uci_nof_codeblocks(A, Et);
    const int      L   = uci_crc_size(A);
    const unsigned A0  = A / C, E0 = Et / C, F = A % C;
    for (int c = 0; c < C; ++c) {
      const unsigned  Ac = c == 0 ? A0 : (A + C - 1) / C;
      const unsigned  Ec = c == 0 ? E0 : Et - E0;
      const unsigned  Fc = c == 0 ? F : 0;
      polar_code_host pc;
      const std::string err = polar_code_build(Ac + L + Fc, Ec, pc);
      if (!err.empty()) {
        return "message " + std::to_string(i) + " codeblock " + std::to_string(c) + ": " + err;
      }
      polar_cb& d  = cbs[2 * (size_t)i + c];
      d.llr_offset = it.llr_offset + (c == 0 ? 0 : E0);
      d.E          = Ec;
      d.out_offset = it.out_offset + (c == 0 ? 0 : A0);
      d.K          = (uint16_t)pc.K;
      d.nbits      = (uint16_t)Ac;
      d.n          = (uint8_t)pc.n;
      d.crc_size   = (uint8_t)L;
      d.nof_filler = (uint8_t)Fc;
      std::memcpy(d.pc, pc.pc, sizeof(d.pc));
      std::memcpy(d.info, pc.info, sizeof(d.info));
    }
  }
  return std::string();
}

} // namespace

namespace pg {

std::string uci_polar_blob(const pg_uci_polar* items, int n, std::vector<uint8_t>& blob)
{
  std::vector<polar_cb> cbs;
  const std::string     err = polar_blob_cbs(items, n, cbs);
  blob.resize(cbs.size() * sizeof(polar_cb));
  std::memcpy(blob.data(), cbs.data(), blob.size());
  return err;
}

int uci_polar_launch_dev(pg_context* ctx, const void* cbs_dev, int n, const int8_t* llrs, uint8_t* bits,
                         uint8_t* valid, cudaStream_t s)
{
  if (n == 0) {
    return PG_OK;
  }
  uci_polar_kernel<<<(unsigned)n, kPolarThreads, 0, s>>>(static_cast<const polar_cb*>(cbs_dev), n, llrs, bits,
                                                         valid);
  return check_cuda(ctx, cudaGetLastError(), "uci_polar_kernel launch");
}

int uci_polar_launch(pg_context* ctx, const pg_uci_polar* items, int n, const int8_t* llrs, uint8_t* bits,
                     uint8_t* valid, cudaStream_t s)
{
  std::vector<uint8_t> blob;
  const std::string    err = uci_polar_blob(items, n, blob);
  if (!err.empty()) {
    return set_error(ctx, PG_ERR_INVALID, err);
  }
  void* dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_UCI_POLAR, blob.data(), blob.size(), s, &dev)) {
    return rc;
  }
  if (int rc = uci_polar_launch_dev(ctx, dev, n, llrs, bits, valid, s)) {
    return rc;
  }
  return release_slot_after(ctx, SLOT_UCI_POLAR, s);
}

} // namespace pg

using namespace pg;

extern "C" {

int pg_polar_code(uint32_t K, uint32_t E, pg_polar_code_info* out)
{
  if (out == nullptr) {
    return PG_ERR_INVALID;
  }
  polar_code_host c;
  if (!polar_code_build(K, E, c).empty()) {
    return PG_ERR_INVALID;
  }
  std::memset(out, 0, sizeof(*out));
  out->n     = (uint16_t)c.n;
  out->N     = (uint16_t)c.N;
  out->K     = (uint16_t)c.K;
  out->E     = (uint16_t)c.E;
  out->nPC   = (uint8_t)c.nPC;
  out->nWmPC = (uint8_t)c.nWmPC;
  std::memcpy(out->pc_set, c.pc, sizeof(out->pc_set));
  std::memcpy(out->k_set, c.info, sizeof(out->k_set));
  for (int j = 0; j < c.N; ++j) {
    out->subblock[j] = subblock_index(j, c.N);
  }
  return PG_OK;
}

int pg_uci_polar_decode_device(pg_context* ctx, const pg_uci_polar* items, int n, const int8_t* llrs, uint8_t* bits,
                               uint8_t* valid, void* stream)
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
  // The codes are built and staged first, so that the kernel events time the kernel alone.
  cudaStream_t         s = static_cast<cudaStream_t>(stream);
  std::vector<uint8_t> blob;
  const std::string    err = uci_polar_blob(items, n, blob);
  if (!err.empty()) {
    return set_error(ctx, PG_ERR_INVALID, err);
  }
  void* dev = nullptr;
  if (int rc = stage_slot(ctx, SLOT_UCI_POLAR, blob.data(), blob.size(), s, &dev)) {
    return rc;
  }
  const unsigned int rec = timing_record_flags(ctx, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_start, s, rec);
  }
  const int rc = uci_polar_launch_dev(ctx, dev, n, llrs, bits, valid, s);
  if (ctx->timed) {
    cudaEventRecordWithFlags(ctx->ev_stop, s, rec);
  }
  return rc != PG_OK ? rc : release_slot_after(ctx, SLOT_UCI_POLAR, s);
}

} // extern "C"

// Test infrastructure only (checker, never shipped): a flat C ABI over the reference's own CPU
// block-floating-point IQ compression of Open Fronthaul (lib/ofh/compression), so tests can compare
// the GPU decompressor with it:
//   iq_decompressor::decompress  include/ocudu/ofh/compression/iq_decompressor.h
//   iq_compressor::compress      include/ocudu/ofh/compression/iq_compressor.h
// The class is the one create_iq_decompressor selects for BFP on an AVX-512 host
// (lib/ofh/compression/compression_factory.cpp:166-176), or the generic one on request.

#include "lib/ofh/compression/iq_compression_bfp_avx512.h"
#include "lib/ofh/compression/iq_compression_bfp_impl.h"
#include "ocudu/ocudulog/ocudulog.h"
#include "ocudu/ofh/compression/compression_properties.h"
#include <algorithm>
#include <memory>

using namespace ocudu;
using namespace ocudu::ofh;

namespace {

constexpr int kChunk = 256;

std::unique_ptr<iq_compression_bfp_impl> make(int generic)
{
  ocudulog::basic_logger& logger = ocudulog::fetch_basic_logger("OFH", false);
  if (generic) {
    return std::make_unique<iq_compression_bfp_impl>(logger);
  }
  return std::make_unique<iq_compression_bfp_avx512>(logger);
}

} // namespace

extern "C" {

// Compresses nof_prb PRBs of complex bf16 samples (12 per PRB, real in the low half of each word).
int ref_bfp_compress(int data_width, const uint32_t* iq, int nof_prb, uint8_t* out, int generic)
{
  auto                  c = make(generic);
  ru_compression_params p{compression_type::BFP, (unsigned)data_width};
  const unsigned        prb_bytes = (unsigned)get_compressed_prb_size(p).value();
  // The reference works on one (symbol, port) section at a time, at most MAX_NOF_PRBS PRBs.
  for (int p0 = 0; p0 < nof_prb; p0 += kChunk) {
    const int np = std::min(kChunk, nof_prb - p0);
    c->compress(span<uint8_t>(out + (size_t)prb_bytes * p0, (size_t)prb_bytes * np),
                span<const cbf16_t>(reinterpret_cast<const cbf16_t*>(iq) + (size_t)12 * p0, (size_t)12 * np), p);
  }
  return (int)prb_bytes;
}

// Decompresses nof_prb PRBs into complex bf16 samples.
int ref_bfp_decompress(int data_width, const uint8_t* in, int nof_prb, uint32_t* iq, int generic)
{
  auto                  c = make(generic);
  ru_compression_params p{compression_type::BFP, (unsigned)data_width};
  const unsigned        prb_bytes = (unsigned)get_compressed_prb_size(p).value();
  for (int p0 = 0; p0 < nof_prb; p0 += kChunk) {
    const int np = std::min(kChunk, nof_prb - p0);
    c->decompress(span<cbf16_t>(reinterpret_cast<cbf16_t*>(iq) + (size_t)12 * p0, (size_t)12 * np),
                  span<const uint8_t>(in + (size_t)prb_bytes * p0, (size_t)prb_bytes * np), p);
  }
  return (int)prb_bytes;
}

} // extern "C"

// C ABI entry points of pusch_b200 (declared in include/pusch_b200.h): context life cycle,
// argument validation, staging and launches.
#include "pg_internal.h"

#include <algorithm>

#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace pg {

int set_error(pg_context* ctx, int code, const std::string& msg)
{
  if (ctx != nullptr) {
    ctx->last_error = msg;
  }
  return code;
}

int check_cuda(pg_context* ctx, cudaError_t err, const char* what)
{
  if (err == cudaSuccess) {
    return PG_OK;
  }
  return set_error(ctx, PG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

int validate_ldpc_descs(pg_context* ctx, const pg_ldpc_cb* cbs, int n, size_t nof_llrs_total, size_t bits_bytes)
{
  if (n < 0 || (n > 0 && cbs == nullptr)) {
    return set_error(ctx, PG_ERR_INVALID, "invalid codeblock list");
  }
  if (n > ctx->max_codeblocks) {
    return set_error(ctx, PG_ERR_CAPACITY,
                     "batch of " + std::to_string(n) + " codeblocks exceeds max_codeblocks " +
                         std::to_string(ctx->max_codeblocks));
  }
  for (int i = 0; i < n; ++i) {
    const pg_ldpc_cb& d = cbs[i];
    char               buf[160];
    if (d.base_graph != 1 && d.base_graph != 2) {
      snprintf(buf, sizeof(buf), "codeblock %d: base graph %d", i, d.base_graph);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (lifting_set_index(d.lifting_size) < 0) {
      snprintf(buf, sizeof(buf), "codeblock %d: %d is not a lifting size", i, d.lifting_size);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    const int Z   = d.lifting_size;
    const int K   = kb_of(d.base_graph) * Z;
    const int Nmx = nshort_of(d.base_graph) * Z;
    if ((int)d.nof_llrs < K + 2 * Z || (int)d.nof_llrs > Nmx) {
      snprintf(buf, sizeof(buf), "codeblock %d: %u LLRs outside [%d, %d]", i, d.nof_llrs, K + 2 * Z, Nmx);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if ((int)d.nof_filler_bits >= K - 2 * Z) {
      snprintf(buf, sizeof(buf), "codeblock %d: %d filler bits", i, d.nof_filler_bits);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (d.crc_poly != PG_CRC16 && d.crc_poly != PG_CRC24A && d.crc_poly != PG_CRC24B && d.crc_poly != PG_CRC_NONE) {
      snprintf(buf, sizeof(buf), "codeblock %d: CRC polynomial %d", i, d.crc_poly);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (d.max_iterations == 0) {
      snprintf(buf, sizeof(buf), "codeblock %d: zero iterations", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (nof_llrs_total != 0 && (size_t)d.llr_offset + d.nof_llrs > nof_llrs_total) {
      snprintf(buf, sizeof(buf), "codeblock %d: LLRs beyond the buffer", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
    if (bits_bytes != 0 && (size_t)d.out_offset + (size_t)((K + 7) / 8) > bits_bytes) {
      snprintf(buf, sizeof(buf), "codeblock %d: output beyond the buffer", i);
      return set_error(ctx, PG_ERR_INVALID, buf);
    }
  }
  return PG_OK;
}

static int ensure_host_capacity(pg_context* ctx, size_t llrs, size_t bits)
{
  if (llrs > ctx->dev.llr_cap) {
    cudaFree(ctx->dev.llrs);
    ctx->dev.llrs    = nullptr;
    ctx->dev.llr_cap = 0;
    if (int rc = check_cuda(ctx, cudaMalloc(&ctx->dev.llrs, llrs), "cudaMalloc(llrs)")) {
      return rc;
    }
    ctx->dev.llr_cap = llrs;
  }
  if (bits > ctx->dev.bits_cap) {
    cudaFree(ctx->dev.bits);
    ctx->dev.bits     = nullptr;
    ctx->dev.bits_cap = 0;
    if (int rc = check_cuda(ctx, cudaMalloc(&ctx->dev.bits, bits), "cudaMalloc(bits)")) {
      return rc;
    }
    ctx->dev.bits_cap = bits;
  }
  return PG_OK;
}

// Copies descriptors into the pinned staging buffer and uploads them on stream s. The staging
// and device descriptor buffers are reused only after the previous kernel that read them has
// completed (see release_descs_after).
static int stage_descs(pg_context* ctx, const pg_ldpc_cb* cbs, int n, cudaStream_t s)
{
  if (ctx->desc_pending) {
    if (int rc = check_cuda(ctx, cudaEventSynchronize(ctx->ev_desc), "cudaEventSynchronize(descriptors)")) {
      return rc;
    }
    ctx->desc_pending = false;
  }
  std::memcpy(ctx->host_descs, cbs, (size_t)n * sizeof(pg_ldpc_cb));
  if (int rc = check_cuda(ctx,
                          cudaMemcpyAsync(ctx->dev.descs, ctx->host_descs, (size_t)n * sizeof(pg_ldpc_cb),
                                          cudaMemcpyHostToDevice, s),
                          "cudaMemcpyAsync(descriptors)")) {
    return rc;
  }
  return PG_OK;
}

// Marks the staged descriptors busy until the work enqueued on s so far (the kernel reading
// them included) has completed.
static int release_descs_after(pg_context* ctx, cudaStream_t s)
{
  if (int rc = check_cuda(ctx, cudaEventRecord(ctx->ev_desc, s), "cudaEventRecord(descriptors)")) {
    return rc;
  }
  ctx->desc_pending = true;
  return PG_OK;
}

int stage_slot(pg_context* ctx, int slot, const void* host, size_t bytes, cudaStream_t s, void** dev)
{
  staging_slot& sl = ctx->slots[slot];
  if (sl.pending) {
    if (int rc = check_cuda(ctx, cudaEventSynchronize(sl.ev), "cudaEventSynchronize(staging)")) {
      return rc;
    }
    sl.pending = false;
  }
  if (sl.ev == nullptr) {
    if (int rc = check_cuda(ctx, cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming), "cudaEventCreate")) {
      return rc;
    }
  }
  if (bytes > sl.cap) {
    cudaFree(sl.dev);
    cudaFreeHost(sl.host);
    sl.dev  = nullptr;
    sl.host = nullptr;
    sl.cap  = 0;
    size_t cap = bytes < 4096 ? 4096 : bytes * 2;
    if (int rc = check_cuda(ctx, cudaMalloc(&sl.dev, cap), "cudaMalloc(staging)")) {
      return rc;
    }
    if (int rc = check_cuda(ctx, cudaMallocHost(&sl.host, cap), "cudaMallocHost(staging)")) {
      return rc;
    }
    sl.cap = cap;
  }
  std::memcpy(sl.host, host, bytes);
  if (int rc = check_cuda(ctx, cudaMemcpyAsync(sl.dev, sl.host, bytes, cudaMemcpyHostToDevice, s),
                          "cudaMemcpyAsync(staging)")) {
    return rc;
  }
  *dev = sl.dev;
  return PG_OK;
}

int release_slot_after(pg_context* ctx, int slot, cudaStream_t s)
{
  staging_slot& sl = ctx->slots[slot];
  if (int rc = check_cuda(ctx, cudaEventRecord(sl.ev, s), "cudaEventRecord(staging)")) {
    return rc;
  }
  sl.pending = true;
  return PG_OK;
}

void free_slots(pg_context* ctx)
{
  for (auto& sl : ctx->slots) {
    if (sl.pending && sl.ev) {
      cudaEventSynchronize(sl.ev);
    }
    cudaFree(sl.dev);
    if (sl.host) {
      cudaFreeHost(sl.host);
    }
    if (sl.ev) {
      cudaEventDestroy(sl.ev);
    }
    sl = staging_slot();
  }
}

// Device scratch that grows on demand (owned by the context).
int ensure_scratch(pg_context* ctx, void** buf, size_t* cap, size_t bytes, const char* what)
{
  if (bytes <= *cap) {
    return PG_OK;
  }
  cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  if (int rc = check_cuda(ctx, cudaMalloc(buf, bytes), what)) {
    return rc;
  }
  *cap = bytes;
  return PG_OK;
}

} // namespace pg

using namespace pg;

extern "C" {

int pg_abi_version(void)
{
  return PG_ABI_VERSION;
}

const char* pg_last_error(const pg_context* ctx)
{
  return ctx ? ctx->last_error.c_str() : "null context";
}

int pg_ldpc_output_bytes(int base_graph, int lifting_size)
{
  return (kb_of(base_graph) * lifting_size + 7) / 8;
}

int pg_create(const pg_config* cfg, pg_context** out)
{
  if (cfg == nullptr || out == nullptr || cfg->max_codeblocks <= 0) {
    return PG_ERR_INVALID;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
    return PG_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major < 10) {
    return PG_ERR_NO_DEVICE;
  }
  pg_context* ctx = new (std::nothrow) pg_context();
  if (ctx == nullptr) {
    return PG_ERR_CAPACITY;
  }
  ctx->device         = cfg->device;
  ctx->max_codeblocks = cfg->max_codeblocks;
  ctx->sm_count       = prop.multiProcessorCount;
  int rc              = check_cuda(ctx, cudaSetDevice(cfg->device), "cudaSetDevice");
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreate(&ctx->ev_start), "cudaEventCreate");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreate(&ctx->ev_stop), "cudaEventCreate");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreate(&ctx->ev_le_start), "cudaEventCreate");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreate(&ctx->ev_le_stop), "cudaEventCreate");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_desc, cudaEventDisableTiming), "cudaEventCreate");
  }
  if (rc == PG_OK) {
    // One slab per resident decoder CTA: at most four per SM (two of twice the size for the Z = 384
    // decoder), and at most one per codeblock.
    rc = check_cuda(ctx,
                    cudaMalloc(&ctx->dev.c2v, (size_t)std::max(cfg->max_codeblocks, 4 * ctx->sm_count) * kC2vStride),
                    "cudaMalloc(check-to-variable scratch)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.descs, (size_t)cfg->max_codeblocks * sizeof(pg_ldpc_cb)),
                    "cudaMalloc(descriptors)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMallocHost(&ctx->host_descs, (size_t)cfg->max_codeblocks * sizeof(pg_ldpc_cb)),
                    "cudaMallocHost(descriptors)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.iterations, (size_t)cfg->max_codeblocks * sizeof(int32_t)),
                    "cudaMalloc(iterations)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.ldpc_counter, 2 * sizeof(int)), "cudaMalloc(ldpc counter)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.ldpc_keys, (size_t)cfg->max_codeblocks), "cudaMalloc(ldpc keys)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.ldpc_order, (size_t)cfg->max_codeblocks * sizeof(uint32_t)),
                    "cudaMalloc(ldpc order)");
  }
  if (rc == PG_OK) {
    ctx->ldpc_ctas = ldpc_resident_ctas(ctx);
    rc             = conv_setup(ctx);
  }
  if (rc == PG_OK) {
    // x^e mod g(x) for CRC16, CRC24A and CRC24B.
    std::vector<uint32_t> pow(3 * (size_t)kCrcPowLen);
    for (int p = 0; p < 3; ++p) {
      uint32_t g;
      int      order;
      crc_poly_params(p, &g, &order);
      const uint32_t mask = (1u << order) - 1u;
      uint32_t       x    = 1;
      for (int e = 0; e < kCrcPowLen; ++e) {
        pow[(size_t)p * kCrcPowLen + e] = x;
        const uint32_t top               = (x >> (order - 1)) & 1u;
        x                                = (x << 1) & mask;
        if (top) {
          x ^= g & mask;
        }
      }
    }
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.crc_pow, pow.size() * sizeof(uint32_t)), "cudaMalloc(crc tables)");
    if (rc == PG_OK) {
      rc = check_cuda(ctx,
                      cudaMemcpy(ctx->dev.crc_pow, pow.data(), pow.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                      "cudaMemcpy(crc tables)");
    }
  }
  if (rc == PG_OK) {
    std::vector<uint32_t> tabs(3 * 3072);
    crc_tables_host(tabs.data());
    rc = check_cuda(ctx, cudaMalloc(&ctx->dev.crc_tabs, tabs.size() * sizeof(uint32_t)), "cudaMalloc(crc tables)");
    if (rc == PG_OK) {
      rc = check_cuda(ctx,
                      cudaMemcpy(ctx->dev.crc_tabs, tabs.data(), tabs.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice),
                      "cudaMemcpy(crc tables)");
    }
  }
  if (rc == PG_OK) {
    rc = ldpc_upload_tables(ctx);
  }
  if (rc == PG_OK) {
    rc = demap_upload_tables(ctx);
  }
  if (rc == PG_OK) {
    rc = est_upload_tables(ctx);
  }
  if (rc == PG_OK) {
    rc = uci_upload_tables(ctx);
  }
  if (rc == PG_OK && cfg->max_llrs > 0) {
    rc = ensure_host_capacity(ctx, (size_t)cfg->max_llrs, (size_t)cfg->max_codeblocks * ((22 * kMaxZ) / 8));
  }
  if (rc != PG_OK) {
    fprintf(stderr, "pusch_b200: pg_create failed: %s\n", ctx->last_error.c_str());
    pg_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return PG_OK;
}

void pg_destroy(pg_context* ctx)
{
  if (ctx == nullptr) {
    return;
  }
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
  }
  cudaFree(ctx->dev.c2v);
  cudaFree(ctx->dev.descs);
  cudaFree(ctx->dev.crc_pow);
  cudaFree(ctx->dev.crc_tabs);
  cudaFree(ctx->dev.gold);
  cudaFree(ctx->scratch_a);
  cudaFree(ctx->est_partials);
  cudaFree(ctx->scratch_b);
  free_slots(ctx);
  cudaFree(ctx->dev.llrs);
  cudaFree(ctx->dev.bits);
  cudaFree(ctx->dev.iterations);
  cudaFree(ctx->dev.ldpc_counter);
  cudaFree(ctx->dev.ldpc_keys);
  cudaFree(ctx->dev.ldpc_order);
  cudaFree(ctx->dev.ldpc_scale);
  if (ctx->host_descs) {
    cudaFreeHost(ctx->host_descs);
  }
  if (ctx->host_stage) {
    cudaFreeHost(ctx->host_stage);
  }
  if (ctx->ev_start) {
    cudaEventDestroy(ctx->ev_start);
  }
  if (ctx->ev_stop) {
    cudaEventDestroy(ctx->ev_stop);
  }
  if (ctx->ev_le_start) {
    cudaEventDestroy(ctx->ev_le_start);
  }
  if (ctx->ev_le_stop) {
    cudaEventDestroy(ctx->ev_le_stop);
  }
  if (ctx->ev_desc) {
    cudaEventDestroy(ctx->ev_desc);
  }
  if (ctx->stream) {
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
}

int pg_ldpc_decode_batch_device(pg_context* ctx, const pg_ldpc_cb* cbs, int nof_cbs, const int8_t* llrs,
                                uint8_t* bits, int32_t* iterations, void* stream)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ldpc_descs(ctx, cbs, nof_cbs, 0, 0)) {
    return rc;
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  if (llrs == nullptr || bits == nullptr || iterations == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null device buffer");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = stage_descs(ctx, cbs, nof_cbs, s)) {
    return rc;
  }
  if (int rc = ldpc_launch(ctx, ctx->dev.descs, nof_cbs, llrs, bits, iterations, s)) {
    return rc;
  }
  return release_descs_after(ctx, s);
}

int pg_ldpc_decode_batch_resident(pg_context* ctx, const pg_ldpc_cb* cbs_dev, int nof_cbs, const int8_t* llrs,
                                  uint8_t* bits, int32_t* iterations, void* stream)
{
  if (ctx == nullptr || nof_cbs < 0 || nof_cbs > ctx->max_codeblocks) {
    return ctx ? set_error(ctx, PG_ERR_CAPACITY, "batch exceeds max_codeblocks") : PG_ERR_INVALID;
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  if (cbs_dev == nullptr || llrs == nullptr || bits == nullptr || iterations == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null device buffer");
  }
  return ldpc_launch(ctx, cbs_dev, nof_cbs, llrs, bits, iterations, static_cast<cudaStream_t>(stream));
}

int pg_ldpc_decode_batch_host(pg_context* ctx, const pg_ldpc_cb* cbs, int nof_cbs, const int8_t* llrs,
                              size_t nof_llrs_total, uint8_t* bits, size_t bits_bytes, int32_t* iterations)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (int rc = validate_ldpc_descs(ctx, cbs, nof_cbs, nof_llrs_total, bits_bytes)) {
    return rc;
  }
  if (nof_cbs == 0) {
    return PG_OK;
  }
  if (llrs == nullptr || bits == nullptr || iterations == nullptr) {
    return set_error(ctx, PG_ERR_INVALID, "null host buffer");
  }
  if (int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice")) {
    return rc;
  }
  if (int rc = ensure_host_capacity(ctx, nof_llrs_total, bits_bytes)) {
    return rc;
  }
  cudaStream_t s  = ctx->stream;
  int          rc = stage_descs(ctx, cbs, nof_cbs, s);
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(ctx->dev.llrs, llrs, nof_llrs_total, cudaMemcpyHostToDevice, s),
                    "cudaMemcpyAsync(llrs)");
  }
  if (rc == PG_OK) {
    rc = ldpc_launch(ctx, ctx->dev.descs, nof_cbs, ctx->dev.llrs, ctx->dev.bits, ctx->dev.iterations, s);
  }
  if (rc == PG_OK) {
    rc = release_descs_after(ctx, s);
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaMemcpyAsync(bits, ctx->dev.bits, bits_bytes, cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync(bits)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx,
                    cudaMemcpyAsync(iterations, ctx->dev.iterations, (size_t)nof_cbs * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync(iterations)");
  }
  if (rc == PG_OK) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return rc;
}

int pg_set_kernel_timing(pg_context* ctx, int enabled)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  ctx->timed = enabled != 0;
  return PG_OK;
}

int pg_set_ldpc_kernel(pg_context* ctx, int kernel)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (kernel < PG_LDPC_KERNEL_ONE_LANE || kernel > PG_LDPC_KERNEL_Z384_SPLIT) {
    return set_error(ctx, PG_ERR_INVALID, "unknown LDPC kernel " + std::to_string(kernel));
  }
  ctx->ldpc_kernel = kernel;
  return PG_OK;
}

int pg_set_ldpc_order(pg_context* ctx, int mode)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (mode != PG_LDPC_ORDER_GIVEN && mode != PG_LDPC_ORDER_LONGEST_FIRST) {
    return set_error(ctx, PG_ERR_INVALID, "unknown LDPC work order " + std::to_string(mode));
  }
  ctx->ldpc_order_mode = mode;
  return PG_OK;
}

int pg_get_ldpc_kernel(const pg_context* ctx)
{
  return ctx == nullptr ? PG_ERR_INVALID : ctx->ldpc_kernel;
}

int pg_set_ldpc_ctas_per_sm(pg_context* ctx, int ctas_per_sm)
{
  if (ctx == nullptr) {
    return PG_ERR_INVALID;
  }
  if (ctas_per_sm < 0 || ctas_per_sm > 4) {
    return set_error(ctx, PG_ERR_INVALID, "LDPC CTAs per SM must be 0-4, not " + std::to_string(ctas_per_sm));
  }
  ctx->ldpc_ctas_per_sm = ctas_per_sm;
  return PG_OK;
}

static float elapsed_ms(cudaEvent_t a, cudaEvent_t b)
{
  float ms = -1.0f;
  if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    // Clear the error of the failed query, so that it is not reported by a later launch check.
    (void)cudaGetLastError();
    return -1.0f;
  }
  return ms;
}

float pg_last_kernel_ms(pg_context* ctx)
{
  if (ctx == nullptr || !ctx->timed) {
    return -1.0f;
  }
  return elapsed_ms(ctx->ev_start, ctx->ev_stop);
}

float pg_last_learned_ms(pg_context* ctx)
{
  if (ctx == nullptr || !ctx->timed || !ctx->le_recorded) {
    return -1.0f;
  }
  return elapsed_ms(ctx->ev_le_start, ctx->ev_le_stop);
}

} // extern "C"

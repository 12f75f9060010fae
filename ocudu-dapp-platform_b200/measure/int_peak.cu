// Integer-ALU throughput probe for the LDPC roofline denominator (B200 has no published INT32
// figure and the measured-peaks file carries none). Each thread runs eight independent chains
// of the integer operations the decoder's inner loop issues (add, min/max, logic, select); the
// probe reports executed integer instructions per second over the whole GPU.
#include <cuda_runtime.h>
#include <cstdint>

namespace {

constexpr int kChains = 8;
constexpr int kOpsPerStep = 4; // add, min, max, xor per chain and step

__global__ void int_mix_kernel(int32_t* out, int steps, int seed)
{
  int32_t a[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    a[c] = seed + threadIdx.x * 7 + c;
  }
  for (int s = 0; s < steps; ++s) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      int32_t x = a[c] + s;
      x         = min(x, 1 << 29);
      x         = max(x, -(1 << 29));
      a[c]      = x ^ (c + 3);
    }
  }
  int32_t acc = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    acc ^= a[c];
  }
  if (acc == 0x7fffffff) {
    out[blockIdx.x] = acc;
  }
}

// One instruction class per KIND, eight independent chains per thread (inline PTX so the
// compiler cannot fold the chains).
template <int KIND>
__global__ void inst_class_kernel(uint32_t* out, int steps, uint32_t seed)
{
  uint32_t a[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    a[c] = seed * (threadIdx.x + 1) + c * 0x00030007u;
  }
  const uint32_t b = seed ^ 0x00050003u, cc = seed + 0x00110013u;
  for (int s = 0; s < steps; ++s) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      uint32_t x = a[c];
      if (KIND == 0) asm volatile("add.s32 %0, %0, %1;" : "+r"(x) : "r"(b));
      if (KIND == 1) asm volatile("min.s32 %0, %0, %1;" : "+r"(x) : "r"(b));
      if (KIND == 2) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(b), "r"(cc));
      if (KIND == 3) asm volatile("prmt.b32 %0, %0, %1, 0x5410;" : "+r"(x) : "r"(b));
      if (KIND == 4) asm volatile("min.s16x2 %0, %0, %1;" : "+r"(x) : "r"(b));
      if (KIND == 5) asm volatile("add.f16x2 %0, %0, %1;" : "+r"(x) : "r"(b));
      if (KIND == 6) asm volatile("min.f16x2 %0, %0, %1;" : "+r"(x) : "r"(b));
      if (KIND == 7) asm volatile("fma.rn.f16x2 %0, %0, %1, %2;" : "+r"(x) : "r"(b), "r"(cc));
      a[c] = x;
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    acc ^= a[c];
  }
  if (acc == 0x12345678u) {
    out[blockIdx.x] = acc;
  }
}

template <int KIND>
double time_class(uint32_t* out, int blocks, int threads, int steps)
{
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  inst_class_kernel<KIND><<<blocks, threads>>>(out, 64, 1);
  cudaEventRecord(e0);
  inst_class_kernel<KIND><<<blocks, threads>>>(out, steps, 1);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms > 0.f ? (double)blocks * threads * steps * kChains / (ms * 1e-3) : -1.0;
}

} // namespace

extern "C" {

/// Thread-instructions per second of eight instruction classes, in this order: add.s32,
/// min.s32, mad.lo.u32, prmt.b32, min.s16x2, add.f16x2, min.f16x2, fma.rn.f16x2. Returns 0 on
/// success.
int pg_probe_inst_classes(int device, double* out8)
{
  if (cudaSetDevice(device) != cudaSuccess) {
    return -1;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  const int blocks = prop.multiProcessorCount * 8, threads = 256, steps = 4096;
  uint32_t* out    = nullptr;
  if (cudaMalloc(&out, blocks * sizeof(uint32_t)) != cudaSuccess) {
    return -1;
  }
  out8[0] = time_class<0>(out, blocks, threads, steps);
  out8[1] = time_class<1>(out, blocks, threads, steps);
  out8[2] = time_class<2>(out, blocks, threads, steps);
  out8[3] = time_class<3>(out, blocks, threads, steps);
  out8[4] = time_class<4>(out, blocks, threads, steps);
  out8[5] = time_class<5>(out, blocks, threads, steps);
  out8[6] = time_class<6>(out, blocks, threads, steps);
  out8[7] = time_class<7>(out, blocks, threads, steps);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/// Runs the probe and returns integer operations per second (ops counted as issued integer
/// instructions per thread), or a negative value on error.
double pg_probe_int_ops_per_s(int device, int steps)
{
  if (cudaSetDevice(device) != cudaSuccess) {
    return -1.0;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  const int threads = 256;
  const int blocks  = prop.multiProcessorCount * 8;
  int32_t*  out     = nullptr;
  if (cudaMalloc(&out, blocks * sizeof(int32_t)) != cudaSuccess) {
    return -1.0;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int_mix_kernel<<<blocks, threads>>>(out, steps / 4, 1); // warm-up
  cudaEventRecord(e0);
  int_mix_kernel<<<blocks, threads>>>(out, steps, 1);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) {
    return -1.0;
  }
  const double ops = (double)blocks * threads * steps * kChains * kOpsPerStep;
  return ops / (ms * 1e-3);
}

} // extern "C"

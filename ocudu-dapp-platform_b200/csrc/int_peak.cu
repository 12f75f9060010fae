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

} // namespace

extern "C" {

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

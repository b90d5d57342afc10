// FP64 tensor-core (DMMA) and FP64 FMA peak microbenchmark.
//
// The roofline denominator of the FP64 sweep kernels: the measured rate of
// mma.sync f64 on this GPU (the driver-written peaks file carries only HBM
// and bf16 figures).  Built as its own small library (librgf_peak.so), loaded
// by bench.py, never by the product.
//
// Each kernel keeps 8 independent accumulator chains per warp in flight;
// 2 CTAs per SM, 8 warps per CTA.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tc32.cuh"

namespace {

// TF32 tensor-core peak: one CTA per SM issues back-to-back
// tcgen05.mma.cta_group::1.kind::tf32 of M = 128, N = 256, K = 8 from
// operands resident in shared memory into a TMEM accumulator (the shape the
// 3xTF32 GEMMs of the split-precision form issue), one commit at the end.
constexpr uint32_t kPkA = 128 * 32 * 4, kPkB = 256 * 32 * 4;
__global__ void __launch_bounds__(128, 1) k_tf32_peak(int iters, int* err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_sh;
  using namespace rgf::tc32;
  const uint32_t base = (su32(smem_raw) + 1023u) & ~1023u;
  float* f = reinterpret_cast<float*>(smem_raw + (base - su32(smem_raw)));
  for (int i = threadIdx.x; i < (int)((kPkA + kPkB) / 4); i += blockDim.x) f[i] = 1.0f / (1 + (i & 63));
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(su32(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_sh)), "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;
  GemmArgs g{};
  g.err = err;
  g.timeout = 20000000000LL;
  if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc =
        (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const uint64_t da = sw128_desc(base), db = sw128_desc(base + kPkA);
    for (int it = 0; it < iters; it++)
#pragma unroll
      for (int kk = 0; kk < 4; kk++) mma_tf32(tmem, da + 2 * kk, db + 2 * kk, idesc, (it | kk) != 0);
    mma_commit(su32(&done));
  }
  __syncwarp();
  mbar_wait(su32(&done), 0, g);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

__global__ void k_dmma884(double* out, int iters) {
  double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4;
  double c[8][2];
  for (int i = 0; i < 8; i++) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[i][0]), "+d"(c[i][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
  for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_dmma16816(double* out, int iters) {
  double a[8], b[4], c[8][4];
  for (int i = 0; i < 8; i++) a[i] = threadIdx.x * 1e-3 + i;
  for (int i = 0; i < 4; i++) b[i] = 1.0 + threadIdx.x * 1e-4 + i;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 4; j++) c[i][j] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++)
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
          "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
          : "+d"(c[i][0]), "+d"(c[i][1]), "+d"(c[i][2]), "+d"(c[i][3])
          : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
            "d"(b[1]), "d"(b[2]), "d"(b[3]));
  }
  double s = 0.0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 4; j++) s += c[i][j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_dfma(double* out, int iters) {
  double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4, c[16];
  for (int i = 0; i < 16; i++) c[i] = i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 16; i++) c[i] = fma(a, c[i], b);
  }
  double s = 0.0;
  for (int i = 0; i < 16; i++) s += c[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Measured FP64 rates (TFLOP/s) on `device`: mma.sync m8n8k4 (the shape the
// sweep issues), m16n8k16 and scalar DFMA.  `out` receives 3 doubles.
// Returns 0 on success, else the CUDA error code.
extern "C" __attribute__((visibility("default"))) int rgf_peak_fp64(int device, double* out) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int warps = 8, threads = warps * 32, blocks = 2 * sms, iters = 4000;
  double* buf = nullptr;
  if ((e = cudaMalloc(&buf, sizeof(double) * blocks * threads)) != cudaSuccess) return (int)e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const double per_warp_iter[3] = {2.0 * 8 * 8 * 4 * 8, 2.0 * 16 * 8 * 16 * 8, 2.0 * 16 * 32};
  for (int q = 0; q < 3; q++) {
    auto launch = [&](int it) {
      if (q == 0) k_dmma884<<<blocks, threads>>>(buf, it);
      else if (q == 1) k_dmma16816<<<blocks, threads>>>(buf, it);
      else k_dfma<<<blocks, threads>>>(buf, it);
    };
    launch(16);
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    out[q] = per_warp_iter[q] * iters * (double)blocks * warps / (ms * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

// Measured dense TF32 tensor-core rate (TFLOP/s) of tcgen05.mma kind::tf32 on
// `device` (one CTA per SM, M = 128, N = 256, K = 8).  Returns 0 on success,
// -2 if a wait timed out, else the CUDA error code.
extern "C" __attribute__((visibility("default"))) int rgf_peak_tf32(int device, double* out) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint32_t smem = 128 * 1024 + 1024;  // the operands use 48 KB; more keeps one CTA per SM
  if ((e = cudaFuncSetAttribute(k_tf32_peak, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
    return (int)e;
  int* err = nullptr;
  if ((e = cudaMalloc(&err, sizeof(int))) != cudaSuccess) return (int)e;
  cudaMemset(err, 0, sizeof(int));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 20000;
  k_tf32_peak<<<sms, 128, smem>>>(64, err);
  cudaEventRecord(e0);
  k_tf32_peak<<<sms, 128, smem>>>(iters, err);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  if (e == cudaSuccess && ms > 0.f) *out = 2.0 * 128 * 256 * 8 * 4.0 * iters * (double)sms / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(err);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return herr ? -2 : 0;
}

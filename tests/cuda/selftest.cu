// Unit-test kernels for device functions of librgf that have no C-ABI entry
// of their own (test infrastructure, built beside librgf.so by
// rgf_b200/build.py as tests/cuda/libselftest.so).
#include <cuda_runtime.h>

#include "../../rgf_b200/csrc/recip.cuh"

using rgf::crecip_nr;

// out[4i..4i+3] = crecip_nr(z_i) and conj(z_i) * (1 / |z_i|^2) by IEEE division
__global__ void k_crecip(const double2* z, double* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 v = z[i];
  const double2 r = crecip_nr(v);
  const double q = 1.0 / fma(v.x, v.x, v.y * v.y);
  out[4 * i + 0] = r.x;
  out[4 * i + 1] = r.y;
  out[4 * i + 2] = v.x * q;
  out[4 * i + 3] = -v.y * q;
}

// z: n complex (host), out: 4n doubles (host).  Returns a cudaError_t.
extern "C" __attribute__((visibility("default"))) int rgf_selftest_crecip(const double* z, double* out, int n) {
  if (n <= 0) return 0;
  double2* dz = nullptr;
  double* dout = nullptr;
  cudaError_t e = cudaMalloc(&dz, sizeof(double2) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 4 * n);
  if (e == cudaSuccess) e = cudaMemcpy(dz, z, sizeof(double2) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_crecip<<<(n + 255) / 256, 256>>>(dz, dout, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost);
  if (dz) cudaFree(dz);
  if (dout) cudaFree(dout);
  return (int)e;
}

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

// ---------------------------------------------------------------------------
// The 3xTF32 tcgen05 GEMM of librgf (rgf_b200/csrc/tc32.cuh) on host arrays:
// A_hi/A_lo [M x K], B_hi/B_lo [Nr x K] (K-major fp32, K a multiple of 32),
// out [ksplit x M x Nr] (kStore/kPartial) or [M x Nr] updated in place (kGJ).
// Returns a cudaError_t, or -1 if a tensor map was refused, -2 on a timeout.
// ---------------------------------------------------------------------------
#include "../../rgf_b200/csrc/tc32.cuh"

template <int BN>
static int tc32_run(int M, int Nr, int K, int ksplit, int mode, int gj_c0, int gj_nb, const float* a_hi,
                    const float* a_lo, const float* b_hi, const float* b_lo, float* out) {
  using namespace rgf::tc32;
  const size_t na = (size_t)M * K, nb = (size_t)Nr * K, no = (size_t)(mode == kPartial ? ksplit : 1) * M * Nr;
  float *d = nullptr, *dout = nullptr;
  int* derr = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(float) * (2 * na + 2 * nb));
  if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(float) * no);
  if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
  float *dah = d, *dal = d + na, *dbh = d + 2 * na, *dbl = d + 2 * na + nb;
  if (e == cudaSuccess) e = cudaMemcpy(dah, a_hi, sizeof(float) * na, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dal, a_lo, sizeof(float) * na, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dbh, b_hi, sizeof(float) * nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dbl, b_lo, sizeof(float) * nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dout, out, sizeof(float) * no, cudaMemcpyHostToDevice);
  int rc = (int)e;
  CUtensorMap m_ah, m_al, m_bh, m_bl;
  if (rc == 0 && !(make_map(&m_ah, dah, K, M, 1, K, 0, BM) && make_map(&m_al, dal, K, M, 1, K, 0, BM) &&
                   make_map(&m_bh, dbh, K, Nr, 1, K, 0, BN) && make_map(&m_bl, dbl, K, Nr, 1, K, 0, BN)))
    rc = -1;
  if (rc == 0) {
    GemmArgs g{};
    g.M = M;
    g.Nr = Nr;
    g.k_chunks = K / BK / ksplit;
    if ((K / BK) % ksplit) g.k_total = K / BK;  // ragged K-split
    g.mode = mode;
    g.out = dout;
    g.ldo = Nr;
    g.split_stride = (int64_t)M * Nr;
    g.gj_c0 = gj_c0;
    g.gj_nb = gj_nb;
    g.err = derr;
    g.timeout = 4000000000LL;
    e = cudaFuncSetAttribute(k_tc32_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg<BN>::SMEM);
    if (e == cudaSuccess) {
      dim3 grid((unsigned)((Nr + BN - 1) / BN), (unsigned)((M + BM - 1) / BM), (unsigned)ksplit);
      k_tc32_gemm<BN><<<grid, kThreads, Cfg<BN>::SMEM>>>(m_ah, m_al, m_bh, m_bl, g);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    rc = (int)e;
    int herr = 0;
    if (rc == 0) rc = (int)cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    if (rc == 0 && herr) rc = -2;
    if (rc == 0) rc = (int)cudaMemcpy(out, dout, sizeof(float) * no, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  cudaFree(dout);
  cudaFree(derr);
  return rc;
}

extern "C" __attribute__((visibility("default"))) int rgf_selftest_tc32(int M, int Nr, int K, int ksplit, int bn,
                                                                        int mode, int gj_c0, int gj_nb,
                                                                        const float* a_hi, const float* a_lo,
                                                                        const float* b_hi, const float* b_lo,
                                                                        float* out) {
  if (M < 1 || Nr < 1 || K < 32 || K % 32 || ksplit < 1 || ksplit > K / 32) return -3;
  switch (bn) {
    case 64: return tc32_run<64>(M, Nr, K, ksplit, mode, gj_c0, gj_nb, a_hi, a_lo, b_hi, b_lo, out);
    case 128: return tc32_run<128>(M, Nr, K, ksplit, mode, gj_c0, gj_nb, a_hi, a_lo, b_hi, b_lo, out);
    case 144: return tc32_run<144>(M, Nr, K, ksplit, mode, gj_c0, gj_nb, a_hi, a_lo, b_hi, b_lo, out);
    case 208: return tc32_run<208>(M, Nr, K, ksplit, mode, gj_c0, gj_nb, a_hi, a_lo, b_hi, b_lo, out);
    case 256: return tc32_run<256>(M, Nr, K, ksplit, mode, gj_c0, gj_nb, a_hi, a_lo, b_hi, b_lo, out);
  }
  return -3;
}

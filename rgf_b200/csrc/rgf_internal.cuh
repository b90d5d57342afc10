// Internal declarations shared by the librgf translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/rgf.h"

namespace rgf {

// ---------------------------------------------------------------------------
// complex helpers (double2 = {re, im}, the layout of rgf_cplx)
// ---------------------------------------------------------------------------
__host__ __device__ inline double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ inline double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 cneg(double2 a) { return cmk(-a.x, -a.y); }
__host__ __device__ inline double2 cconj(double2 a) { return cmk(a.x, -a.y); }
__host__ __device__ inline double2 cmul(double2 a, double2 b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 cscale(double2 a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ inline double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
// 1/a computed with Smith's scaling (Smith, CACM 5(8) 1962) to avoid overflow.
__host__ __device__ inline double2 cinv(double2 a) {
  if (fabs(a.x) >= fabs(a.y)) {
    double r = a.y / a.x, d = a.x + a.y * r;
    return cmk(1.0 / d, -r / d);
  } else {
    double r = a.x / a.y, d = a.x * r + a.y;
    return cmk(r / d, -1.0 / d);
  }
}

// probe vector of the a-posteriori slice-inverse check:
// v(i) = exp(2 pi i frac(i * golden ratio)), |v(i)| = 1
__device__ inline double2 probe_v(int64_t i) {
  double f = (double)i * 0.6180339887498949;
  f -= floor(f);
  double s, c;
  sincospi(2.0 * f, &s, &c);
  return make_double2(c, s);
}

// ---------------------------------------------------------------------------
// problem description shared by the host orchestrator and the kernels
// ---------------------------------------------------------------------------
enum { kMaxStencil = 5 };

struct Transverse {
  int dim;        // 2 or 3
  int64_t n0;     // 2D: ny; 3D: nx (fast index)
  int64_t n1;     // 2D: 1;  3D: ny
  int64_t N;      // n0*n1
  int bc;         // rgf_bc (3D: PERIODIC, DIRICHLET or BLOCH)
  double ka0;     // Bloch phase along the fast transverse axis (2D: ka)
  double ka1;     // 3D: Bloch phase along y
};

// device status word bits
enum : int {
  kStatusSingular = 1,
  kStatusNonfinite = 2,
  kStatusTimeout = 4,
};

// thread-local last error (rgf_api.cu)
void set_error(const std::string& msg);

}  // namespace rgf

// Device-side lead-channel set-up (see channels.cu).
#pragma once
#include "rgf_internal.cuh"

namespace rgf {

// per-side channel arrays on the device (all of length N unless noted)
struct SideDev {
  double2* kx;      // longitudinal wavenumber kxdx (2D) / kzdx (3D)
  double2* lam;     // exp(1i*kx)
  double2* sqrtmu;  // sqrt(sin(kx)) for every channel (used at propagating ones)
  int* isprop;      // 1 if 0 < Re z < 1
  int* prop;        // compacted propagating channel indices (0-based)
  int* nprop;       // number of propagating channels (1 int)
  int* conj;        // ind_prop_conj (0-based), when defined
};

void launch_transverse(const Transverse& tr, double* k0, double* k1, cudaStream_t s);
void launch_longitudinal(const Transverse& tr, const double* k0, const double* k1, double2 k2e,
                         const SideDev& side, cudaStream_t s);
void launch_compact(int64_t N, const SideDev& side, int conj_mode, int64_t ind_zero0, cudaStream_t s);
void launch_phi(const Transverse& tr, const double* k0, const double* k1, double2* phi, int64_t ld,
                cudaStream_t s);
void launch_stencil(const Transverse& tr, int* st_col, double2* st_val, cudaStream_t s);
void launch_laplacian_dense(int64_t n, int bc, double ka, double2* A, cudaStream_t s);

}  // namespace rgf

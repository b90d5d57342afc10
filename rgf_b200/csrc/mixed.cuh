// The split-precision form of the slice recursion (rgf_precision RGF_TF32X3):
// slice inverses factored in FP32 with 3xTF32 tensor-core updates, the
// S-matrix won back by FP64 iterative refinement of the block-tridiagonal
// solve (see mixed.cu).
#pragma once
#include <functional>

#include "rgf_internal.cuh"

namespace rgf {

// Everything the precision form reads; device pointers unless noted.
struct MixedProblem {
  int64_t N = 0, L = 0;          // transverse sites, slices (L >= 1)
  int niL = 0, niR = 0;          // requested input channels per side (S columns [in_L; in_R])
  int noL = 0, noR = 0;          // requested output channels per side (S rows [out_L; out_R])
  const double2* phi = nullptr;  // N x N transverse profiles, row-major (site, mode)
  const int* prop[2] = {nullptr, nullptr};       // compacted propagating mode indices per side
  const double2* sqrtmu[2] = {nullptr, nullptr};  // sqrt_mu per mode, per side
  const int* in_idx = nullptr;   // niL + niR channel indices (into prop[side])
  const int* out_idx = nullptr;  // noL + noR channel indices
  const int* pairs = nullptr;    // (row, column) of the Kronecker delta, npairs of them
  int npairs = 0;
  const double2* G0[2] = {nullptr, nullptr};  // lead surface Green's functions, N x N row-major
  const int* st_col = nullptr;   // slice stencil (kMaxStencil per row)
  const double2* st_val = nullptr;
  double2 k2{0, 0};              // k0dx^2
  const double2* eps = nullptr;  // N x L, slice k at eps + k*N
  double2* S = nullptr;          // n_out x n_in, column-major, ldS (device)
  int64_t ldS = 0;
};

struct MixedStats {
  int iterations = 0;      // refinement passes run (the first solve included)
  int converged = 0;
  double last_change = 0;  // relative size of the last correction (max of whole, first, last slice)
  double factor_ms = 0, solve_ms = 0;  // device time of the low-precision factorization / all solves
};

// device workspace slots the precision form asks its caller for
enum MixedSlot : int {
  kMxW, kMxT, kMxStoreHi, kMxStoreLo, kMxX, kMxY, kMxPart, kMxBt, kMxVec, kMxNorm, kMxStatus,
  kMxSlots
};
using MixedAlloc = std::function<rgf_status(int slot, size_t bytes, void** p)>;

// status the host reads as "refinement did not reach the tolerance": the
// caller then computes S with the FP64 form
constexpr rgf_status kMixedNotConverged = (rgf_status)1001;

rgf_status smatrix_mixed(const MixedProblem& mp, const MixedAlloc& alloc, cudaStream_t s, MixedStats* stats,
                         int64_t* launches);

// bytes of device workspace the precision form needs (the factor store dominates:
// 8 N lda L bytes with lda = 2N rounded up to 32)
size_t mixed_workspace_bytes(int64_t N, int64_t L, int64_t P);

}  // namespace rgf

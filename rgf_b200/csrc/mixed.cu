// The split-precision form (RGF_TF32X3) of the slice recursion of
// cal_smatrix_RGF.m:237-289 / cal_smatrix_RGF_3D.m (general branch and, since
// one solve serves every request, the partial branches :217-256 as well).
//
// The reference's G-recursion is the block LU factorization of the
// block-tridiagonal operator with the leads folded in: eliminating the lead
// surface pixels (n = 0, nx+1, whose blocks are G0^-1) leaves the slices
// k = 0..L-1 with
//     H_kk = A_k (- G0_L at k = 0) (- G0_R at k = L-1),   H_k,k+-1 = -I,
// sources b_0 = G0_L B_L (left inputs), b_{L-1} = G0_R B_R (right inputs), and
// S = -2i [C_L G0_L (B_L + x_0); C_R G0_R (B_R + x_{L-1})] - delta
// for the solution x of H x = b (B_L only in left-input columns, B_R only in
// right-input ones).  Here:
//
// 1. factor: g_k = (H_kk - g_{k-1})^-1 for every slice in FP32 (complex64),
//    each inverse by block Gauss-Jordan with 64-wide pivot blocks: the pivot
//    block's inverse T by one CTA (register-resident GJ, diagonal pivots), the
//    row panel U = T W'(J, :) in FP32, and the rank-64 update
//    W <- W' - V U on the tensor cores (tcgen05.mma kind::tf32, 3xTF32, TMEM
//    accumulators, TMA-staged operands: tc32.cuh).  Every g_k is kept (hi/lo
//    tf32 split, the solve's A operand).
// 2. refine in FP64: x = 0, then repeatedly r = b - H x with the FP64
//    stencil and FP64 lead blocks, d = (LU)^-1 r by the forward / backward
//    substitution over the stored g_k (3xTF32 GEMMs, FP32 vectors), x += d,
//    until the correction is below round-off.  The residual is exact in FP64,
//    so x converges to the FP64 solution whatever the factor's accuracy, as
//    long as the factor is a contraction (|I - (LU)^-1 H| < 1); if it is not
//    (a near-singular pivot block, strong gain), the caller falls back to the
//    FP64 form.
// 3. S from x in FP64 (lead blocks and Fisher-Lee projection).
#include <math.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "mixed.cuh"
#include "sweep.cuh"
#include "tc32.cuh"

namespace rgf {
namespace {

constexpr int NB = 32;            // pivot block width (complex)
constexpr int kMaxIter = 8;
// x has converged when the last correction is below kTolStop, or the
// correction the next pass would make (the last one times the observed
// contraction, measured over the whole solution and over its first and last
// slices, which S is formed from) is below kTolNext -- an order of magnitude
// under the 1e-10 the split-precision form is held to
constexpr double kTolStop = 1e-13;
constexpr double kTolNext = 1e-11;
constexpr long long kGemmTimeout = 4000000000LL;  // ~2 s of SM clock

#define RGF_CUDA_TRY_MX(call)                                                            \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);    \
      return e_ == cudaErrorMemoryAllocation ? RGF_ERR_OOM : RGF_ERR_CUDA;               \
    }                                                                                    \
  } while (0)

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
__device__ __forceinline__ void split2(float a, float b, float* hi, float* lo) {
  const float ah = tf32_hi(a), bh = tf32_hi(b);
  *reinterpret_cast<float2*>(hi) = make_float2(ah, bh);
  *reinterpret_cast<float2*>(lo) = make_float2(a - ah, b - bh);
}
__device__ __forceinline__ float2 fcmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// programmatic dependent launch: let the next kernel of the stream start its
// prologue, and wait for the previous one before touching its results
__device__ __forceinline__ void pdl_open() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// launch with programmatic stream serialization (every kernel launched this
// way waits for its predecessor with pdl_wait before it reads or writes)
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------------------
// factorization kernels
// ---------------------------------------------------------------------------

// W holds g_{k-1} (store != 0: written to the factor store as hi/lo) and is
// replaced by the next slice matrix (assemble != 0):
//   W = A_k - g_{k-1} - Ga - Gb - Wx,  A_k = stencil - k0dx^2 eps_k on the diagonal
// (Wx: the block of the other side at the junction slice of the two-sided form).
// Columns [N, ldw) are the zero padding of the store rows.
__global__ void k_mx_assemble(float2* W, int64_t ldw, int64_t N, float* st_hi, float* st_lo, int store,
                              int assemble, const int* st_col, const double2* st_val, double2 k2,
                              const double2* eps, const double2* Ga, const double2* Gb, const float2* Wx) {
  pdl_open();
  pdl_wait();
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= ldw) return;
  for (int64_t i = blockIdx.y; i < N; i += gridDim.y) {
    const int64_t o = i * ldw + j;
    if (j >= N) {
      if (store) {
        *reinterpret_cast<float2*>(st_hi + 2 * o) = make_float2(0.f, 0.f);
        *reinterpret_cast<float2*>(st_lo + 2 * o) = make_float2(0.f, 0.f);
      }
      continue;
    }
    const float2 w = W[o];
    if (store) split2(w.x, w.y, st_hi + 2 * o, st_lo + 2 * o);
    if (!assemble) continue;
    double2 v = store ? cmk(-(double)w.x, -(double)w.y) : cmk(0.0, 0.0);
    if (Ga) v = csub(v, Ga[i * N + j]);
    if (Gb) v = csub(v, Gb[i * N + j]);
    if (Wx) v = cmk(v.x - (double)Wx[o].x, v.y - (double)Wx[o].y);  // the other side's block (junction slice)
#pragma unroll
    for (int q = 0; q < kMaxStencil; q++)
      if (st_col[i * kMaxStencil + q] == j) v = cadd(v, st_val[i * kMaxStencil + q]);
    if (i == j) v = csub(v, cmul(k2, eps[i]));
    W[o] = make_float2((float)v.x, (float)v.y);
  }
}

// ---------------------------------------------------------------------------
// refinement kernels.  Vectors are N x P row-major per slice (site, column):
// x (FP64, L slices), y (FP32, L slices), the GEMM partials (ksplit x N x P
// FP32 complex), and the GEMM's right operand Bt (2P rows x lda, K = 2i, 2i+1).
// One block = 32 columns x 32 sites, threads (32, 8).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 sum_parts(const float2* part, int ksplit, int64_t stride, int64_t ip) {
  float2 s = make_float2(0.f, 0.f);
  for (int z = 0; z < ksplit; z++) {
    const float2 v = part[z * stride + ip];
    s.x += v.x;
    s.y += v.y;
  }
  return s;
}

// write the transposed tile (tile[p][i]) as rows 2p, 2p+1 of Bt
__device__ __forceinline__ void store_bt(float2 (&tile)[32][33], int64_t p0, int64_t i0, int64_t N, int64_t P,
                                         float* bt_hi, float* bt_lo, int64_t lda) {
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int q = threadIdx.y + 8 * u;
    const int64_t p = p0 + q, i = i0 + threadIdx.x;
    if (p < P && i < N) {
      const float2 v = tile[q][threadIdx.x];
      split2(v.x, -v.y, bt_hi + (2 * p) * lda + 2 * i, bt_lo + (2 * p) * lda + 2 * i);
      split2(v.y, v.x, bt_hi + (2 * p + 1) * lda + 2 * i, bt_lo + (2 * p + 1) * lda + 2 * i);
    }
  }
}

// residual of the whole solve in FP64, every slice at once:
//   r_k = b_k - (H x)_k = b_k - A_k x_k + x_{k-1} + x_{k+1} (+ G0_L x_0 at k = 0,
//   + G0_R x_{L-1} at k = L-1), stored in FP32 in r (= the y buffer: the
// forward pass replaces r_k by y_k once r_{k+1} has been read).
// Block: 32 columns x 8 sites of one slice (grid z = slice).
__global__ void __launch_bounds__(256) k_mx_residual(int64_t L, int64_t N, int64_t P, const double2* x,
                                                     float2* r, const double2* eps, const int* st_col,
                                                     const double2* st_val, double2 k2, const double2* b0,
                                                     const double2* bL, const double2* e0, const double2* e1) {
  pdl_open();
  pdl_wait();
  const int64_t NP = N * P;
  const int64_t p = blockIdx.x * 32 + threadIdx.x, i = blockIdx.y * 8 + threadIdx.y;
  if (p >= P || i >= N) return;
  const int64_t ip = i * P + p;
  for (int64_t k = blockIdx.z; k < L; k += gridDim.z) {
  const double2* xk = x + k * NP;
  double2 v = cmk(0.0, 0.0);
  if (k == 0) {
    v = cadd(v, b0[ip]);
    if (e0) v = cadd(v, e0[ip]);
  }
  if (k == L - 1) {
    v = cadd(v, bL[ip]);
    if (e1) v = cadd(v, e1[ip]);
  }
  double2 ax = cneg(cmul(cmul(k2, eps[k * N + i]), xk[ip]));
#pragma unroll
  for (int q = 0; q < kMaxStencil; q++) {
    const int c = st_col[i * kMaxStencil + q];
    if (c >= 0) ax = cadd(ax, cmul(st_val[i * kMaxStencil + q], xk[(int64_t)c * P + p]));
  }
  v = csub(v, ax);
  if (k > 0) v = cadd(v, xk[ip - NP]);
  if (k < L - 1) v = cadd(v, xk[ip + NP]);
  r[k * NP + ip] = make_float2((float)v.x, (float)v.y);
  }
}

// forward pass, slice k: y_kprev = (GEMM partials) -> ystore[kprev] (over its
// r; kprev = k -+ 1 by the sweep's direction, < 0 at the sweep's first slice);
// v_k = r_k + y_kprev (+ y_kprev2 from part2 at the junction slice) -> Bt.
__global__ void __launch_bounds__(256) k_mx_fwd_prep(int64_t k, int64_t kprev, int64_t N, int64_t P, int64_t ldp,
                                                     int64_t poff, float2* ystore, const float2* part, int ksplit,
                                                     const float2* part2, int64_t kprev2, int ksplit2, float* bt_hi,
                                                     float* bt_lo, int64_t lda, const int* kdev) {
  pdl_open();
  pdl_wait();
  if (kdev) {  // slice index kept on the device (graph-captured sweeps)
    k += *kdev;
    kprev += *kdev;
  }
  __shared__ float2 tile[32][33];
  const int64_t p0 = blockIdx.x * 32, i0 = blockIdx.y * 32, NP = N * ldp;
  const int64_t p = p0 + threadIdx.x;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int q = threadIdx.y + 8 * u;
    const int64_t i = i0 + q;
    float2 v = make_float2(0.f, 0.f);
    if (i < N && p < P) {
      const int64_t ip = i * ldp + poff + p;
      v = ystore[k * NP + ip];  // r_k
      if (kprev >= 0) {  // y of the neighbour slice swept before (over its r)
        const float2 yp = sum_parts(part, ksplit, N * P, i * P + p);
        ystore[kprev * NP + ip] = yp;
        v.x += yp.x;
        v.y += yp.y;
      }
      if (part2) {  // junction slice: the other side's neighbour too
        const float2 yq = sum_parts(part2, ksplit2, N * P, i * P + p);
        ystore[kprev2 * NP + ip] = yq;
        v.x += yq.x;
        v.y += yq.y;
      }
    }
    tile[threadIdx.x][q] = v;
  }
  __syncthreads();
  store_bt(tile, p0, i0, N, P, bt_hi, bt_lo, lda);
}

// backward pass, slice k: d_k = (GEMM partials) + y_k (add_y; without it the
// partials are d_k itself: the sweep's first slice); x_k += d_k in FP64; norms
// of d and x (whole; slice 0; slice L-1); d_k -> Bt (write_bt) and -> Bt2 (the
// junction slice feeds both sides).  add_y, write_bt < 0: the one-sided rule.
__global__ void __launch_bounds__(256) k_mx_bwd_prep(int64_t k, int64_t L, int64_t N, int64_t P, int64_t ldp,
                                                     int64_t poff, double2* x,
                                                     const float2* ystore, const float2* part, int ksplit,
                                                     float* bt_hi, float* bt_lo, int64_t lda, double* norms,
                                                     const int* kdev, int add_y, int write_bt, float* bt2_hi,
                                                     float* bt2_lo) {
  pdl_open();
  pdl_wait();
  if (kdev) k += *kdev;  // slice index kept on the device (graph-captured sweeps)
  if (add_y < 0) add_y = k < L - 1;   // one-sided sweep: y_k enters except at the first slice
  if (write_bt < 0) write_bt = k > 0;  // ... and the next GEMM needs d_k except after slice 0
  __shared__ float2 tile[32][33];
  __shared__ double red[2][8];
  const int64_t p0 = blockIdx.x * 32, i0 = blockIdx.y * 32, NP = N * ldp;
  const int64_t p = p0 + threadIdx.x;
  double dd = 0.0, xx = 0.0;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int q = threadIdx.y + 8 * u;
    const int64_t i = i0 + q;
    float2 d = make_float2(0.f, 0.f);
    if (i < N && p < P) {
      const int64_t ip = i * ldp + poff + p;
      d = sum_parts(part, ksplit, N * P, i * P + p);
      if (add_y) {
        const float2 y = ystore[k * NP + ip];
        d.x += y.x;
        d.y += y.y;
      }
      double2* xp = x + k * NP + ip;
      const double2 xn = cmk(xp->x + (double)d.x, xp->y + (double)d.y);
      *xp = xn;
      dd += (double)d.x * d.x + (double)d.y * d.y;
      xx += xn.x * xn.x + xn.y * xn.y;
    }
    tile[threadIdx.x][q] = d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    dd += __shfl_xor_sync(0xffffffffu, dd, o);
    xx += __shfl_xor_sync(0xffffffffu, xx, o);
  }
  if (threadIdx.x == 0) {
    red[0][threadIdx.y] = dd;
    red[1][threadIdx.y] = xx;
  }
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; w++) {
      a += red[0][w];
      b += red[1][w];
    }
    atomicAdd(norms + 0, a);
    atomicAdd(norms + 1, b);
    if (k == 0) {
      atomicAdd(norms + 2, a);
      atomicAdd(norms + 3, b);
    }
    if (k == L - 1) {
      atomicAdd(norms + 4, a);
      atomicAdd(norms + 5, b);
    }
  }
  if (write_bt) store_bt(tile, p0, i0, N, P, bt_hi, bt_lo, lda);
  if (bt2_hi) store_bt(tile, p0, i0, N, P, bt2_hi, bt2_lo, lda);
}

// B columns in S order: left inputs into Bl, right inputs into Br (N x P row-major)
__global__ void k_mx_fill_B(const double2* phi, int64_t N, const int* propL, const int* propR,
                            const double2* muL, const double2* muR, const int* in_idx, int niL, int64_t P,
                            double2* Bl, double2* Br) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= N * P) return;
  const int64_t i = e / P;
  const int p = (int)(e % P);
  const double2 z = cmk(0.0, 0.0);
  if (p < niL) {
    const int m = propL[in_idx[p]];
    Bl[e] = cmul(phi[i * N + m], muL[m]);
    Br[e] = z;
  } else {
    const int m = propR[in_idx[p]];
    Bl[e] = z;
    Br[e] = cmul(phi[i * N + m], muR[m]);
  }
}

__global__ void k_mx_add(const double2* a, const double2* b, double2* c, int64_t n) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < n) c[e] = cadd(a[e], b[e]);
}

// S(o, p) = -2i mu_m sum_i conj(phi(i, m)) X(i, p), X = G0_L (B_L + x_0) for
// left outputs, G0_R (B_R + x_{L-1}) for right ones; one warp per entry.
__global__ void k_mx_extract(const double2* phi, int64_t N, const int* propL, const int* propR,
                             const double2* muL, const double2* muR, const int* out_idx, int noL, int n_out,
                             int64_t P, const double2* XL, const double2* XR, double2* S, int64_t ldS) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= (int64_t)n_out * P) return;
  const int o = (int)(w % n_out);
  const int64_t p = w / n_out;
  const bool left = o < noL;
  const int m = (left ? propL : propR)[out_idx[o]];
  const double2* X = left ? XL : XR;
  double2 acc = cmk(0.0, 0.0);
  for (int64_t i = lane; i < N; i += 32) acc = cadd(acc, cmul(cconj(phi[i * N + m]), X[i * P + p]));
  for (int s = 16; s > 0; s >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, s);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, s);
  }
  if (lane == 0) {
    const double2 v = cmul((left ? muL : muR)[m], acc);
    S[o + p * ldS] = cmk(2.0 * v.y, -2.0 * v.x);
  }
}

__global__ void k_mx_delta(double2* S, int64_t ldS, const int* pairs, int npairs) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < npairs) S[pairs[2 * q] + (int64_t)pairs[2 * q + 1] * ldS].x -= 1.0;
}

// ---------------------------------------------------------------------------
// One Gauss-Jordan step of the slice inverse in a single launch:
//   W_dst = W' - V U,  V = W(:, J) - E_J,  U = T W'(J, :),  T = W(J, J)^-1,
//   W' = W_src with the columns J replaced by those of the identity (E_J).
// Every CTA owns a 128 x 128 real tile of W (64 complex columns) and forms
// T itself (redundantly: the 32-pivot chain sets the step time anyway, and
// no CTA waits for another), U for its columns straight into the swizzled
// shared-memory operand, the 3xTF32 product on tcgen05 (TMEM accumulator)
// and the update.  W_src and W_dst are different buffers, so a CTA that
// finishes early never overwrites what another still reads.  256 threads.
// ---------------------------------------------------------------------------
namespace gjs {
constexpr int BN = 128;                 // real columns per tile
constexpr uint32_t CH = 16384;          // one operand K-chunk: 128 rows x 32 fp32 (128-byte rows)
// A = V (hi, lo); B = U (hi, lo), which first holds the U product's left
// operand realify_right(W'(J, tile columns)) in the same geometry
constexpr uint32_t OFF_AH = 0, OFF_AL = 2 * CH, OFF_BH = 4 * CH, OFF_BL = 6 * CH;  // 32 KB each
constexpr uint32_t OFF_WP = 8 * CH;     // W' tile: 4 chunks [chunk][row][32 fp32], unswizzled
constexpr uint32_t TU_CH = 8192;        // one K-chunk of the T image: 64 rows x 128 bytes
constexpr uint32_t TU_HALF = 2 * TU_CH; // hi image, then lo image
constexpr uint32_t TU_BYTES = 2 * TU_HALF;
constexpr uint32_t OFF_TU = 12 * CH;    // the realified T image (right operand of the U product)
constexpr uint32_t SMEM = OFF_TU + TU_BYTES + 1024;
constexpr uint32_t TMEM_COLS = 256;     // update accumulator: columns [0, 128); U product: [128, 192)
constexpr int TP = BN + 4;              // pitch of the epilogue staging tile (over the operands)
static_assert(128 * TP * 4 <= OFF_WP, "staging tile");
static_assert(SMEM <= 227 * 1024, "shared memory of one CTA");
}  // namespace gjs

__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, int* status, long long timeout) {
  if (tc32::mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!tc32::mbar_try(bar, parity)) {
    if (clock64() - t0 > timeout) {
      atomicOr(status, kStatusTimeout);
      return false;
    }
  }
  return true;
}

// Development builds only (-DRGF_MX_STAMPS, never in the shipped library):
// %globaltimer at the phase boundaries of one CTA of the step kernel.
#ifdef RGF_MX_STAMPS
__device__ unsigned long long g_mx_stamps[16];
#define MX_STAMP(i)                                                                     \
  do {                                                                                  \
    if (blockIdx.x == 1 && blockIdx.y == 0 && threadIdx.x == 0) {                       \
      unsigned long long t_;                                                            \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                           \
      g_mx_stamps[i] = t_;                                                              \
    }                                                                                   \
  } while (0)
// per launch (in launch order, up to 512): server phase times [0, 10), tile (0, 0) start/end [14, 16)
__device__ unsigned long long g_mx_tl[512][16];
__device__ unsigned int g_mx_tl_n[2];
#define MX_SSTAMP(i)                                                                    \
  do {                                                                                  \
    if (threadIdx.x == 0) {                                                             \
      unsigned long long t_;                                                            \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                           \
      g_mx_stamps[10 + (i)] = t_;                                                       \
      if ((i) == 0) mx_sslot = atomicAdd(&g_mx_tl_n[0], 1u) & 511u;                     \
      g_mx_tl[mx_sslot][(i)] = t_;                                                      \
    }                                                                                   \
  } while (0)
#define MX_TSTAMP(i)                                                                    \
  do {                                                                                  \
    if (blockIdx.x == 1 && blockIdx.y == 0 && threadIdx.x == 0) {                       \
      unsigned long long t_;                                                            \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                           \
      if ((i) == 0) mx_tslot = atomicAdd(&g_mx_tl_n[1], 1u) & 511u;                     \
      g_mx_tl[mx_tslot][14 + (i)] = t_;                                                 \
    }                                                                                   \
  } while (0)
#else
#define MX_STAMP(i) \
  do {              \
  } while (0)
#define MX_SSTAMP(i) \
  do {               \
  } while (0)
#define MX_TSTAMP(i) \
  do {               \
  } while (0)
#endif
#ifdef RGF_MX_STAMPS
#define MX_DECL unsigned mx_sslot = 0, mx_tslot = 0
#else
#define MX_DECL \
  do {          \
  } while (0)
#endif

// X = M^-1 for a 16 x 16 complex block by one warp: Gauss-Jordan on diagonal
// pivots with lane l holding row l/2, columns (l%2) + 2q; the pivot row, the
// multiplier and the pivot come by shuffles, so no barrier is needed.  A zero
// or non-finite pivot sets *bad.
__device__ __forceinline__ void inv16_warp(const float2* M, int ldm, float2* X, int ldx, int lane, int* bad) {
  const int r = lane >> 1, h = lane & 1;
  float2 a[8];
#pragma unroll
  for (int q = 0; q < 8; q++) a[q] = M[r * ldm + h + 2 * q];
  bool badl = false;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    float2 rk[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      rk[q].x = __shfl_sync(0xffffffffu, a[q].x, 2 * k + h);
      rk[q].y = __shfl_sync(0xffffffffu, a[q].y, 2 * k + h);
    }
    const float2 src = a[k >> 1];
    float2 f, p;
    f.x = __shfl_sync(0xffffffffu, src.x, 2 * r + (k & 1));
    f.y = __shfl_sync(0xffffffffu, src.y, 2 * r + (k & 1));
    p.x = __shfl_sync(0xffffffffu, src.x, 2 * k + (k & 1));
    p.y = __shfl_sync(0xffffffffu, src.y, 2 * k + (k & 1));
    const float d = p.x * p.x + p.y * p.y;
    float id;  // approximate reciprocal (one instruction): the factor only preconditions the refinement
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(id) : "f"(d));
    if (!(d > 0.f) || !isfinite(id)) badl = true;
    const float2 pinv = make_float2(p.x * id, -p.y * id);
    const bool me = (r == k);
    const float2 fp = fcmul(f, pinv);
    const float2 coef = me ? make_float2(-pinv.x, -pinv.y) : fp;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float2 u = fcmul(coef, rk[q]);
      const float2 base = me ? make_float2(0.f, 0.f) : a[q];
      a[q] = make_float2(base.x - u.x, base.y - u.y);
    }
    if (h == (k & 1)) a[k >> 1] = me ? pinv : make_float2(-fp.x, -fp.y);
  }
#pragma unroll
  for (int q = 0; q < 8; q++) X[r * ldx + h + 2 * q] = a[q];
  if (badl) *bad = 1;
}

// C (16 x 16) = sign * A B (+ D), row-major with the given leading dimensions;
// thread t of the block computes element (t / 16, t % 16)
__device__ __forceinline__ void mm16(const float2* A, int lda_, const float2* B, int ldb, const float2* D, int ldd,
                                     float sign, float2* C, int ldc, int t) {
  const int i = t >> 4, j = t & 15;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int s = 0; s < 16; s++) {
    const float2 u = fcmul(A[i * lda_ + s], B[s * ldb + j]);
    acc.x += u.x;
    acc.y += u.y;
  }
  float2 v = make_float2(sign * acc.x, sign * acc.y);
  if (D) {
    v.x += D[i * ldd + j].x;
    v.y += D[i * ldd + j].y;
  }
  C[i * ldc + j] = v;
}

// C (32 x 32) = sign * A B (+ D) in shared memory (leading dimension 33) by
// 256 threads: thread t computes rows i, i + 16 and columns c, c + 16
// (i = t / 16, c = t % 16)
__device__ __forceinline__ void mm32(const float2* A, const float2* B, const float2* D, float sign, float2* C,
                                     int t) {
  constexpr int LD = NB + 1;
  const int i = t >> 4, c = t & 15;
  float2 acc[2][2];
#pragma unroll
  for (int u = 0; u < 2; u++)
#pragma unroll
    for (int v = 0; v < 2; v++) acc[u][v] = make_float2(0.f, 0.f);
#pragma unroll 8
  for (int s = 0; s < NB; s++) {
    const float2 a0 = A[i * LD + s], a1 = A[(i + 16) * LD + s];
    const float2 b0 = B[s * LD + c], b1 = B[s * LD + c + 16];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const float2 av = u ? a1 : a0, bv = v ? b1 : b0;
        acc[u][v].x = fmaf(av.x, bv.x, fmaf(-av.y, bv.y, acc[u][v].x));
        acc[u][v].y = fmaf(av.x, bv.y, fmaf(av.y, bv.x, acc[u][v].y));
      }
  }
#pragma unroll
  for (int u = 0; u < 2; u++)
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const int o = (i + 16 * u) * LD + c + 16 * v;
      float2 w = make_float2(sign * acc[u][v].x, sign * acc[u][v].y);
      if (D) {
        w.x += D[o].x;
        w.y += D[o].y;
      }
      C[o] = w;
    }
}

// T = M^-1 for the identity-padded 32 x 32 pivot block M (shared memory,
// leading dimension 33) by 2 x 2 blocks of 16 (A, B; C, D): X = A^-1,
// S = D - C X B, Y = S^-1, T = [[X - X B T21, -X B Y], [-Y C X, Y]]; the two
// 16 x 16 inverses by warp 0 (shuffles only), the products by all 256
// threads.  tmp: 5 x 16 x 17 float2 of shared memory.  T is zeroed beyond jn.
__device__ __forceinline__ void inv32_block(const float2* Mb, float2* Ts, float2* tmp, int jn, int tid, int* bad) {
  constexpr int LD = NB + 1, L16 = 17;
  const int warp = tid >> 5, lane = tid & 31;
  float2* Xs = tmp;
  float2* P1 = Xs + 16 * L16;
  float2* P2 = P1 + 16 * L16;
  float2* Ss = P2 + 16 * L16;
  float2* Ys = Ss + 16 * L16;
  if (warp == 0) inv16_warp(Mb, LD, Xs, L16, lane, bad);
  __syncthreads();
  mm16(Xs, L16, Mb + 16, LD, nullptr, 0, 1.f, P1, L16, tid);           // P1 = X B
  mm16(Mb + 16 * LD, LD, Xs, L16, nullptr, 0, 1.f, P2, L16, tid);      // P2 = C X
  __syncthreads();
  mm16(Mb + 16 * LD, LD, P1, L16, Mb + 16 * LD + 16, LD, -1.f, Ss, L16, tid);  // S = D - C P1
  __syncthreads();
  if (warp == 0) inv16_warp(Ss, L16, Ys, L16, lane, bad);
  __syncthreads();
  mm16(P1, L16, Ys, L16, nullptr, 0, -1.f, Ts + 16, LD, tid);            // T12 = -P1 Y
  mm16(Ys, L16, P2, L16, nullptr, 0, -1.f, Ts + 16 * LD, LD, tid);       // T21 = -Y P2
  Ts[(16 + (tid >> 4)) * LD + 16 + (tid & 15)] = Ys[(tid >> 4) * L16 + (tid & 15)];  // T22 = Y
  __syncthreads();
  mm16(P1, L16, Ts + 16 * LD, LD, Xs, L16, -1.f, Ts, LD, tid);          // T11 = X - P1 T21
  __syncthreads();
  if (jn < NB) {
    const int r = tid >> 3, cq = tid & 7;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int c = cq + 8 * q;
      if (r >= jn || c >= jn) Ts[r * LD + c] = make_float2(0.f, 0.f);
    }
    __syncthreads();
  }
}

// what the pivot-block server of a Gauss-Jordan step needs: the current
// block inverse (Tin), where the next one goes (Tout), the next pivot block
// J' = [j1, j1 + jn1) and, at the last step of a slice, the next slice's
// stencil, permittivity and right-lead block (its first pivot block is then
// A_{n+1}(J', J') - g_n(J', J') [- G0_R(J', J')])
// The pivot-block inverse T as the right operand of the step's U product
// (U = T W'(J, :), computed on the tensor core as conj(U)^T in realified
// form): image rows 2t = T(t, :) and 2t + 1 = i T(t, :), K = (re, im) of
// column m, K-major with the 128-byte swizzle, 2 K-chunks of 64 rows; the tf32
// hi image, then the lo image.  Ts: T in shared memory, row pitch ldt.
__device__ __forceinline__ void publish_tu(const float2* Ts, int ldt, uint8_t* img, int tid) {
  const int r = tid >> 3, cq = tid & 7;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int m = cq + 8 * q, kf = 2 * m, kc = kf >> 5, gq = (kf & 31) >> 2, ofs = (kf & 3) * 4;
    const float2 t = Ts[r * ldt + m];
#pragma unroll
    for (int rr = 0; rr < 2; rr++) {
      const int n = 2 * r + rr;
      const float x0 = rr ? -t.y : t.x, x1 = rr ? t.x : t.y;
      const uint32_t off = kc * gjs::TU_CH + n * 128 + ((gq ^ (n & 7)) << 4) + ofs;
      const float h0 = tf32_hi(x0), h1 = tf32_hi(x1);
      *reinterpret_cast<float2*>(img + off) = make_float2(h0, h1);
      *reinterpret_cast<float2*>(img + gjs::TU_HALF + off) = make_float2(x0 - h0, x1 - h1);
    }
  }
}

struct GjNext {
  const float2* Tin;
  float2* Tout;
  const uint8_t* tu_in;  // image of Tin (publish_tu)
  uint8_t* tu_out;       // image of Tout
  int j1, jn1;
  int next_slice;        // 1: J' is the next slice's first block
  int same_block;        // 1: J' is the current block (one block per slice)
  const double2* eps_next;
  const double2* g0r;    // non-null: subtract G0_R(J', J') (the next slice is the last)
  int64_t ldg;           // leading dimension of g0r (N)
  const int* st_col;
  const double2* st_val;
  double2 k2;
};

// The pivot-block server (one CTA of the step's grid): the next pivot block
// after this step, W_{j+1}(J', J') = W(J', J') - W(J', J) T W(J, J') (J' and J
// disjoint), or T itself when J' = J, assembled with the next slice's matrix
// at a slice boundary, then its inverse into ns.Tout -- computed while the
// tile CTAs apply this step, so that the next step starts with its T ready.
#ifdef RGF_MX_STAMPS
#define MX_PSTAMP(i)                                                                    \
  do {                                                                                  \
    if (threadIdx.x == 0) {                                                             \
      unsigned long long t_;                                                            \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                           \
      g_mx_tl[(g_mx_tl_n[0] - 1u) & 511u][(i)] = t_;                                    \
    }                                                                                   \
  } while (0)
#else
#define MX_PSTAMP(i) \
  do {               \
  } while (0)
#endif
__device__ void t_server(const float* __restrict__ Wsrc, int64_t lda, int j0, int jn, const GjNext& ns,
                         uint8_t* gb, int* bad) {
  constexpr int LD = NB + 1;
  const int tid = threadIdx.x, r = tid >> 3, cq = tid & 7;
  float2* Tj = reinterpret_cast<float2*>(gb);
  float2* B1 = Tj + NB * LD;  // W(J, J')
  float2* B2 = B1 + NB * LD;  // W(J', J)
  float2* B3 = B2 + NB * LD;  // W(J', J')
  float2* U1 = B3 + NB * LD;
  float2* Mn = U1 + NB * LD;
  float2* To = Mn + NB * LD;
  float2* tmp = To + NB * LD;
  const int j1 = ns.j1, jn1 = ns.jn1;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cq + 8 * q;
    Tj[r * LD + c] = ns.Tin[r * NB + c];
    const float2 z = make_float2(0.f, 0.f);
    B1[r * LD + c] = (r < jn && c < jn1) ? *reinterpret_cast<const float2*>(Wsrc + (int64_t)(j0 + r) * lda + 2 * (j1 + c)) : z;
    B2[r * LD + c] = (r < jn1 && c < jn) ? *reinterpret_cast<const float2*>(Wsrc + (int64_t)(j1 + r) * lda + 2 * (j0 + c)) : z;
    B3[r * LD + c] = (r < jn1 && c < jn1) ? *reinterpret_cast<const float2*>(Wsrc + (int64_t)(j1 + r) * lda + 2 * (j1 + c)) : z;
  }
  __syncthreads();
  MX_PSTAMP(2);
  if (!ns.same_block) {
    mm32(Tj, B1, nullptr, 1.f, U1, tid);  // U1 = T W(J, J')
    __syncthreads();
    MX_PSTAMP(3);
    mm32(B2, U1, B3, -1.f, Mn, tid);      // W(J', J') - W(J', J) U1
  } else {
#pragma unroll
    for (int q = 0; q < 4; q++) Mn[r * LD + cq + 8 * q] = Tj[r * LD + cq + 8 * q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cq + 8 * q;
    float2 v = Mn[r * LD + c];
    if (r < jn1 && c < jn1) {
      if (ns.next_slice) {  // A_{n+1}(J', J') - g_n(J', J') [- G0_R(J', J')]
        double2 a = cmk(-(double)v.x, -(double)v.y);
        const int gi = j1 + r, gc = j1 + c;
#pragma unroll
        for (int qq = 0; qq < kMaxStencil; qq++)
          if (ns.st_col[gi * kMaxStencil + qq] == gc) a = cadd(a, ns.st_val[gi * kMaxStencil + qq]);
        if (gi == gc) a = csub(a, cmul(ns.k2, ns.eps_next[gi]));
        if (ns.g0r) a = csub(a, ns.g0r[gi * ns.ldg + gc]);
        v = make_float2((float)a.x, (float)a.y);
      }
    } else {
      v = make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    Mn[r * LD + c] = v;
  }
  __syncthreads();
  MX_PSTAMP(4);
  inv32_block(Mn, To, tmp, jn1, tid, bad);
  MX_PSTAMP(5);
#pragma unroll
  for (int q = 0; q < 4; q++) ns.Tout[r * NB + cq + 8 * q] = To[r * LD + cq + 8 * q];
  publish_tu(To, LD, ns.tu_out, tid);
}

__global__ void __launch_bounds__(256, 1)
    k_mx_gj_step(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapW,
                 const float* __restrict__ Wsrc, float* __restrict__ Wdst, int64_t lda, int N, int j0, int jn,
                 const GjNext ns, int* status, long long timeout) {
  using namespace gjs;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_ld;
  __shared__ __align__(8) uint64_t bar_tu;
  __shared__ __align__(8) uint64_t bar_mu;
  __shared__ __align__(8) uint64_t bar_mma;
  __shared__ uint32_t tmem_sh;
  __shared__ int bad;
  pdl_open();
  MX_DECL;
  MX_STAMP(0);
  const uint32_t sb = (tc32::su32(smem_raw) + 1023u) & ~1023u;
  uint8_t* gb = smem_raw + (sb - tc32::su32(smem_raw));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // grid column 0: the pivot-block server (row 0) only -- the first CTA of the
  // grid to be scheduled, so that it never waits for an SM behind tiles (of
  // this grid or of the other side's)
  if (blockIdx.x == 0) {
    if (blockIdx.y != 0) return;
    if (tid == 0) bad = 0;
    pdl_wait();
    MX_SSTAMP(0);
    __syncthreads();
    if (ns.Tout) t_server(Wsrc, lda, j0, jn, ns, gb, &bad);
    __syncthreads();
    MX_SSTAMP(1);
    if (bad && tid == 0) atomicOr(status, kStatusSingular);
    return;
  }
  const int m0 = blockIdx.y * 128, n0 = (blockIdx.x - 1) * BN;
  if (tid == 0) {
    tc32::mbar_init(tc32::su32(&bar_ld), 1);
    tc32::mbar_init(tc32::su32(&bar_tu), 1);
    tc32::mbar_init(tc32::su32(&bar_mu), 1);
    tc32::mbar_init(tc32::su32(&bar_mma), 1);
    bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc32::su32(&tmem_sh)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;
  pdl_wait();
  MX_STAMP(1);
  MX_TSTAMP(0);

  // (1) the image of this step's pivot-block inverse (published by the server
  //     of the step before); TMA: V's rows W_src(m0.., 2 j0 .. 2 j0 + 63)
  //     swizzled for the MMA, and the W' tile
  const uint32_t bl = tc32::su32(&bar_ld), btu = tc32::su32(&bar_tu);
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(btu), "r"(TU_BYTES) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sb + OFF_TU),
                 "l"(ns.tu_in), "r"(TU_BYTES), "r"(btu)
                 : "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bl), "r"(6 * CH) : "memory");
    for (int kc = 0; kc < 2; kc++) tc32::tma_load_3d(sb + OFF_AH + kc * CH, &mapA, 2 * j0 + 32 * kc, m0, 0, bl);
    for (int kc = 0; kc < 4; kc++) tc32::tma_load_3d(sb + OFF_WP + kc * CH, &mapW, n0 + 32 * kc, m0, 0, bl);
  }
  // (2) the U product's left operand realify_right(W'(J, tile columns)), W' =
  //     W with the pivot columns replaced by the identity's: lane = pivot row m
  //     (K = 2m, 2m + 1), warp = 8 complex columns j (rows 2j: conj W'(m, j),
  //     2j + 1: i conj W'(m, j)), split hi/lo into the B area
  {
    const int m = lane, kf = 2 * m, kc = kf >> 5, gq = (kf & 31) >> 2, ofs = (kf & 3) * 4;
    float4 wv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int n = n0 + 16 * warp + 4 * q;
      wv[q] = (m < jn && n < lda) ? *reinterpret_cast<const float4*>(Wsrc + (int64_t)(j0 + m) * lda + n)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    MX_STAMP(2);
#pragma unroll
    for (int q = 0; q < 4; q++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = 8 * warp + 2 * q + h, c = (n0 >> 1) + j;
        float re = h ? wv[q].z : wv[q].x, im = h ? wv[q].w : wv[q].y;
        if (c >= j0 && c < j0 + jn) {
          re = (j0 + m == c && m < jn) ? 1.f : 0.f;
          im = 0.f;
        }
#pragma unroll
        for (int rr = 0; rr < 2; rr++) {
          const int n = 2 * j + rr;
          const float x0 = rr ? im : re, x1 = rr ? re : -im;
          const uint32_t off = kc * CH + n * 128 + ((gq ^ (n & 7)) << 4) + ofs;
          const float h0 = tf32_hi(x0), h1 = tf32_hi(x1);
          *reinterpret_cast<float2*>(gb + OFF_BH + off) = make_float2(h0, h1);
          *reinterpret_cast<float2*>(gb + OFF_BL + off) = make_float2(x0 - h0, x1 - h1);
        }
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // operand writes -> tensor core
  __syncthreads();
  MX_STAMP(3);
  // (3) the U product on tcgen05 (3xTF32, M = 128, N = 64, K = 64) into TMEM
  //     columns [128, 192): row n of the result is row n of U's operand
  const uint32_t bmu = tc32::su32(&bar_mu);
  if (tid == 0) {
    wait_bar(btu, 0, status, timeout);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int kc = 0; kc < 2; kc++) {
      const uint64_t ah = tc32::sw128_desc(sb + OFF_BH + kc * CH), al = tc32::sw128_desc(sb + OFF_BL + kc * CH);
      const uint64_t th = tc32::sw128_desc(sb + OFF_TU + kc * TU_CH);
      const uint64_t tl = tc32::sw128_desc(sb + OFF_TU + TU_HALF + kc * TU_CH);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const uint64_t o = (uint64_t)(kk * 2);
        tc32::mma_tf32(tmem + 128, al + o, th + o, tc32::Cfg<64>::IDESC, (kc | kk) != 0);
        tc32::mma_tf32(tmem + 128, ah + o, tl + o, tc32::Cfg<64>::IDESC, 1);
        tc32::mma_tf32(tmem + 128, ah + o, th + o, tc32::Cfg<64>::IDESC, 1);
      }
    }
    tc32::mma_commit(bmu);
  }
  __syncwarp();
  // (4) V = W(:, J) - E_J, split hi/lo in place over the swizzled TMA tile (while the U product runs)
  const bool ok_ld = wait_bar(bl, 0, status, timeout);
  MX_STAMP(4);
#pragma unroll
  for (int u = 0; u < 8; u++) {
    const int g = tid + 256 * u, kc = g >> 10, gi = g & 1023, row = gi >> 3, gp = gi & 7;
    const int kf = kc * 32 + ((gp ^ (row & 7)) << 2);  // logical fp32 column of the granule
    const uint32_t off = OFF_AH + kc * CH + row * 128 + gp * 16;
    float4 x = *reinterpret_cast<const float4*>(gb + off);
    const int m = m0 + row, t = kf >> 1;
    if (t < jn && m == j0 + t) x.x -= 1.f;
    if (t + 1 < jn && m == j0 + t + 1) x.z -= 1.f;
    const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
    *reinterpret_cast<float4*>(gb + off) = h;
    *reinterpret_cast<float4*>(gb + off + (OFF_AL - OFF_AH)) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
  }
  MX_STAMP(5);
  // (5) the update's right operand from TMEM: row n (= tile column n) holds
  //     (Re U(t, j), -Im U(t, j)) for n = 2j and (Im U, Re U) for n = 2j + 1
  //     over K = 2t, 2t + 1; split hi/lo over the U product's left operand,
  //     which the completed product no longer reads.  Warp w: rows
  //     32 (w mod 4) .., K-chunk w / 4.
  const bool ok_u = wait_bar(bmu, 0, status, timeout);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  {
    const int n = 32 * (warp & 3) + lane, kc = warp >> 2;
#pragma unroll
    for (int hf = 0; hf < 2; hf++) {
      float v[16];
      tc32::tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 + 32 * kc + 16 * hf), v);
#pragma unroll
      for (int g4 = 0; g4 < 4; g4++) {
        const int g = 4 * hf + g4;
        const float4 x = make_float4(v[4 * g4], v[4 * g4 + 1], v[4 * g4 + 2], v[4 * g4 + 3]);
        const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
        const uint32_t off = kc * CH + n * 128 + ((g ^ (n & 7)) << 4);
        *reinterpret_cast<float4*>(gb + OFF_BH + off) = h;
        *reinterpret_cast<float4*>(gb + OFF_BL + off) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // operand writes -> tensor core
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  MX_STAMP(6);
  // (6) 2 K-chunks x 4 K-steps x 3 products on tcgen05
  const uint32_t bm = tc32::su32(&bar_mma);
  if (tid == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int kc = 0; kc < 2; kc++) {
      const uint64_t ah = tc32::sw128_desc(sb + OFF_AH + kc * CH), al = tc32::sw128_desc(sb + OFF_AL + kc * CH);
      const uint64_t bh = tc32::sw128_desc(sb + OFF_BH + kc * CH), blo = tc32::sw128_desc(sb + OFF_BL + kc * CH);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const uint64_t o = (uint64_t)(kk * 2);
        tc32::mma_tf32(tmem, al + o, bh + o, tc32::Cfg<BN>::IDESC, (kc | kk) != 0);
        tc32::mma_tf32(tmem, ah + o, blo + o, tc32::Cfg<BN>::IDESC, 1);
        tc32::mma_tf32(tmem, ah + o, bh + o, tc32::Cfg<BN>::IDESC, 1);
      }
    }
    tc32::mma_commit(bm);
  }
  __syncwarp();
  const bool ok = wait_bar(bm, 0, status, timeout) && ok_ld && ok_u;
  MX_STAMP(7);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // (7) epilogue: D (TMEM) -> staging over the operands -> W_dst = W' - D, one warp per row
  float* stg = reinterpret_cast<float*>(gb + OFF_AH);
  if (warp < 4) {
    const int row = warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tc32::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      float4* t4 = reinterpret_cast<float4*>(stg + row * TP + c);
#pragma unroll
      for (int j = 0; j < 4; j++) t4[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
  }
  __syncthreads();
  MX_STAMP(8);
  if (ok) {
    const int cc = lane * 4, n = n0 + cc;
    const float* wp = reinterpret_cast<const float*>(gb + OFF_WP) + (cc >> 5) * (CH / 4) + (cc & 31);
#pragma unroll 4
    for (int rr = warp; rr < 128; rr += 8) {
      const int m = m0 + rr;
      if (m >= N || n >= lda) continue;
      const float4 d = *reinterpret_cast<const float4*>(stg + rr * TP + cc);
      float4 w = *reinterpret_cast<const float4*>(wp + rr * 32);
      const int c0 = n >> 1;  // complex columns c0, c0 + 1
      if (c0 >= j0 && c0 < j0 + jn) {
        w.x = (c0 == m) ? 1.f : 0.f;
        w.y = 0.f;
      }
      if (c0 + 1 >= j0 && c0 + 1 < j0 + jn) {
        w.z = (c0 + 1 == m) ? 1.f : 0.f;
        w.w = 0.f;
      }
      *reinterpret_cast<float4*>(Wdst + (int64_t)m * lda + n) = make_float4(w.x - d.x, w.y - d.y, w.z - d.z, w.w - d.w);
    }
  }
  MX_STAMP(9);
  MX_TSTAMP(1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// the first pivot-block inverse of the first slice (later ones come from the
// step kernels' server): T = W(J0, J0)^-1, one CTA
__global__ void __launch_bounds__(256) k_mx_t0(const float* __restrict__ W, int64_t lda, int jn, float2* Tout,
                                               uint8_t* tu_out, int* status) {
  pdl_open();
  pdl_wait();
  constexpr int LD = NB + 1;
  __shared__ float2 Mb[NB * LD];
  __shared__ float2 To[NB * LD];
  __shared__ float2 tmp[5 * 16 * 17];
  __shared__ int bad;
  const int tid = threadIdx.x, r = tid >> 3, cq = tid & 7;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cq + 8 * q;
    Mb[r * LD + c] = (r < jn && c < jn) ? *reinterpret_cast<const float2*>(W + (int64_t)r * lda + 2 * c)
                                        : make_float2(r == c ? 1.f : 0.f, 0.f);
  }
  if (tid == 0) bad = 0;
  __syncthreads();
  inv32_block(Mb, To, tmp, jn, tid, &bad);
#pragma unroll
  for (int q = 0; q < 4; q++) Tout[r * NB + cq + 8 * q] = To[r * LD + cq + 8 * q];
  publish_tu(To, LD, tu_out, tid);
  if (bad && tid == 0) atomicOr(status, kStatusSingular);
}

inline int64_t lda_of(int64_t N) { return (2 * N + 31) / 32 * 32; }

template <int BN>
rgf_status gemm_attr() {
  static thread_local int done_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (done_dev == dev) return RGF_OK;
  if (cudaFuncSetAttribute(tc32::k_tc32_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           tc32::Cfg<BN>::SMEM) != cudaSuccess) {
    set_error("cannot configure the tcgen05 GEMM's shared memory");
    return RGF_ERR_CUDA;
  }
  done_dev = dev;
  return RGF_OK;
}

// ksplit: the largest divisor of the K-chunk count that keeps tiles*ksplit <= SMs
int choose_ksplit(int64_t tiles, int64_t kchunks, int sms) {
  int best = 1;
  for (int64_t z = 1; z <= kchunks; z++)
    if (kchunks % z == 0 && tiles * z <= sms) best = (int)z;
  return best;
}

}  // namespace

#ifdef RGF_MX_STAMPS
extern "C" __attribute__((visibility("default"))) int rgf_dev_mx_stamps(unsigned long long* out) {
  return (int)cudaMemcpyFromSymbol(out, g_mx_stamps, sizeof(g_mx_stamps));
}
extern "C" __attribute__((visibility("default"))) int rgf_dev_mx_timeline(unsigned long long* out, unsigned* n) {
  cudaMemcpyFromSymbol(n, g_mx_tl_n, sizeof(g_mx_tl_n));
  const unsigned z[2] = {0, 0};
  cudaMemcpyToSymbol(g_mx_tl_n, z, sizeof(z));
  return (int)cudaMemcpyFromSymbol(out, g_mx_tl, sizeof(g_mx_tl));
}
#endif

size_t mixed_workspace_bytes(int64_t N, int64_t L, int64_t P) {
  const int64_t lda = lda_of(N), ldw = lda / 2;
  size_t b = 0;
  b += 2 * sizeof(float2) * N * ldw;          // W, two buffers
  b += 2 * sizeof(float) * N * lda * L;       // factor store hi/lo
  b += sizeof(double2) * N * P * L;           // x
  b += sizeof(float2) * N * P * L;            // y
  b += sizeof(float2) * N * P * 148;          // partials (at most one per SM)
  b += 2 * sizeof(float) * 2 * P * lda;       // Bt hi/lo
  b += sizeof(double2) * N * P * 6;           // Bl, Br, b0, bL, e0/e1 (also G0 (B + x) at the end)
  b += 4 * (sizeof(float2) * NB * NB + gjs::TU_BYTES);  // pivot-block inverses and their images
  return b;
}

rgf_status smatrix_mixed(const MixedProblem& mp, const MixedAlloc& alloc, cudaStream_t s, MixedStats* stats,
                         int64_t* launches) {
  const int64_t N = mp.N, L = mp.L, P = mp.niL + mp.niR, n_out = mp.noL + mp.noR;
  const int64_t lda = lda_of(N), ldw = lda / 2, NP = N * P;
  rgf_status st;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_mx_gj_step, cudaFuncAttributeMaxDynamicSharedMemorySize, gjs::SMEM) != cudaSuccess) {
    set_error("cannot configure the Gauss-Jordan step kernel's shared memory");
    return RGF_ERR_CUDA;
  }
  void *pW, *pT, *pSh, *pSl, *pX, *pY, *pPart, *pBt, *pVec, *pNorm, *pStat;
  const int ntile_m = (int)((N + tc32::BM - 1) / tc32::BM);
  const int kchunks = (int)(lda / tc32::BK);
  // Two-sided form (L >= 8): the slices [0, c-1) are factored from the left
  // lead and [c, L) from the right lead, concurrently on two streams; the
  // junction slice c-1 is then inverted with both sides' blocks,
  // (A_{c-1} - g_{c-2} - g_c)^-1, and every solve sweeps both halves at once
  // and meets there.  Below 8 slices one chain from the left (the reference's
  // order) does it all.
  const bool two = L >= 8;
  const int64_t cj = two ? (L + 1) / 2 : L;  // junction slice + 1 (two-sided)
  const int nside = two ? 2 : 1;
  // solve GEMM tile width: 64 real columns for narrow requests, else 128 (a
  // three-deep TMA pipeline).  Measured slower at config 2 (2P = 408): 256-wide
  // tiles (two stages only, stalled on the loads) and 3 tiles of 144 with a
  // ragged 3-way K-split (780 ms of solves against 715 ms for 4 x 128, 2-way).
  const int sbn = (2 * P <= 64) ? 64 : 128;
  if ((st = gemm_attr<64>()) || (st = gemm_attr<128>())) return st;
  int sTiles = (int)((2 * P + sbn - 1) / sbn);
  int sSplit = choose_ksplit((int64_t)ntile_m * sTiles, kchunks, sms / nside);
  if ((st = alloc(kMxW, 2 * nside * sizeof(float) * N * lda, &pW)) ||
      (st = alloc(kMxT, (sizeof(float2) * NB * NB + gjs::TU_BYTES) * 2 * nside, &pT)) ||
      (st = alloc(kMxStoreHi, sizeof(float) * N * lda * L, &pSh)) ||
      (st = alloc(kMxStoreLo, sizeof(float) * N * lda * L, &pSl)) ||
      (st = alloc(kMxX, sizeof(double2) * NP * L, &pX)) || (st = alloc(kMxY, sizeof(float2) * NP * L, &pY)) ||
      (st = alloc(kMxPart, sizeof(float2) * NP * sSplit * nside, &pPart)) ||
      (st = alloc(kMxBt, 2 * nside * sizeof(float) * 2 * P * lda, &pBt)) ||
      (st = alloc(kMxVec, sizeof(double2) * NP * 6, &pVec)) || (st = alloc(kMxNorm, sizeof(double) * 8, &pNorm)) ||
      (st = alloc(kMxStatus, 4 * sizeof(int), &pStat)))
    return st;
  float* st_hi = static_cast<float*>(pSh);
  float* st_lo = static_cast<float*>(pSl);
  double2* x = static_cast<double2*>(pX);
  float2* y = static_cast<float2*>(pY);
  float* bt_hi = static_cast<float*>(pBt);
  double2* Bl = static_cast<double2*>(pVec);
  double2* Br = Bl + NP;
  double2* b0 = Br + NP;
  double2* bL = b0 + NP;
  double2* e0 = bL + NP;
  double2* e1 = e0 + NP;
  double* norms = static_cast<double*>(pNorm);
  int* mstat = static_cast<int*>(pStat);

  // per side: two W buffers with their tensor maps (swizzled 32-column boxes
  // for the update's left operand, unswizzled ones for the W' tile), two
  // pivot-block inverses, the solve's right operand Bt (2P rows x lda, hi/lo)
  // and its GEMM partials; the factor store (N rows x lda, L slices) is shared
  struct Side {
    float* W[2];
    CUtensorMap mA[2], mWp[2], mBh, mBl;
    float2* Tb;
    uint8_t* Tu;  // images of the two inverses (publish_tu)
    float* bh;
    float* bl;
    float2* part;
    int cur = 0;
    int64_t gstep = 0;
    cudaStream_t q = nullptr;
    int64_t first = 0, count = 0, dir = 1;  // the side's slices: first, first + dir, ... (count of them)
  } sd[2];
  CUtensorMap mSh, mSl;
  bool maps_ok = tc32::make_map(&mSh, st_hi, lda, N, L, lda, N * lda, tc32::BM) &&
                 tc32::make_map(&mSl, st_lo, lda, N, L, lda, N * lda, tc32::BM);
  for (int q = 0; q < nside; q++) {
    Side& d = sd[q];
    d.W[0] = static_cast<float*>(pW) + (2 * q) * N * lda;
    d.W[1] = d.W[0] + N * lda;
    d.Tb = static_cast<float2*>(pT) + 2 * q * NB * NB;
    d.Tu = static_cast<uint8_t*>(pT) + sizeof(float2) * NB * NB * 2 * nside + 2 * q * gjs::TU_BYTES;
    d.bh = bt_hi + q * 4 * P * lda;
    d.bl = d.bh + 2 * P * lda;
    d.part = static_cast<float2*>(pPart) + q * NP * sSplit;
    for (int w = 0; w < 2; w++)
      maps_ok = maps_ok && tc32::make_map(&d.mA[w], d.W[w], lda, N, 1, lda, 0, tc32::BM) &&
                tc32::make_map(&d.mWp[w], d.W[w], lda, N, 1, lda, 0, tc32::BM, CU_TENSOR_MAP_SWIZZLE_NONE);
    maps_ok = maps_ok && tc32::make_map(&d.mBh, d.bh, lda, 2 * P, 1, lda, 0, sbn) &&
              tc32::make_map(&d.mBl, d.bl, lda, 2 * P, 1, lda, 0, sbn);
  }
  if (!maps_ok) {
    set_error("tensor-map encoding for the tcgen05 GEMM failed");
    return RGF_ERR_CUDA;
  }
  sd[0].q = s;
  sd[0].first = 0;
  sd[0].count = two ? cj - 1 : L;
  sd[0].dir = 1;
  cudaStream_t s2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  struct StreamGuard {
    cudaStream_t* st;
    cudaEvent_t* f;
    cudaEvent_t* j;
    ~StreamGuard() {
      if (*st) cudaStreamDestroy(*st);
      if (*f) cudaEventDestroy(*f);
      if (*j) cudaEventDestroy(*j);
    }
  } sgd{&s2, &fork, &join};
  if (two) {
    RGF_CUDA_TRY_MX(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    RGF_CUDA_TRY_MX(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    RGF_CUDA_TRY_MX(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    sd[1].q = s2;
    sd[1].first = L - 1;
    sd[1].count = L - cj;
    sd[1].dir = -1;
  }
  auto fork_sides = [&]() -> rgf_status {
    if (!two) return RGF_OK;
    RGF_CUDA_TRY_MX(cudaEventRecord(fork, s));
    RGF_CUDA_TRY_MX(cudaStreamWaitEvent(s2, fork, 0));
    return RGF_OK;
  };
  auto join_sides = [&]() -> rgf_status {
    if (!two) return RGF_OK;
    RGF_CUDA_TRY_MX(cudaEventRecord(join, s2));
    RGF_CUDA_TRY_MX(cudaStreamWaitEvent(s, join, 0));
    return RGF_OK;
  };
  RGF_CUDA_TRY_MX(cudaMemsetAsync(mstat, 0, sizeof(int), s));
  RGF_CUDA_TRY_MX(cudaMemsetAsync(pW, 0, 2 * nside * sizeof(float) * N * lda, s));
  RGF_CUDA_TRY_MX(cudaMemsetAsync(bt_hi, 0, 2 * nside * sizeof(float) * 2 * P * lda, s));  // zero K padding
  RGF_CUDA_TRY_MX(cudaMemsetAsync(x, 0, sizeof(double2) * NP * L, s));
  cudaEvent_t ev[3];
  for (int q = 0; q < 3; q++) RGF_CUDA_TRY_MX(cudaEventCreate(&ev[q]));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int q = 0; q < 3; q++) cudaEventDestroy(e[q]);
    }
  } evg{ev};
  int64_t nl = 0;

  // (1) low-precision factorization
  RGF_CUDA_TRY_MX(cudaEventRecord(ev[0], s));
  const dim3 ga((unsigned)((ldw + 255) / 256), (unsigned)std::min<int64_t>(N, 8192));
  // one grid column more than the tiles (column 0): its first CTA serves the next pivot block
  const dim3 ggj((unsigned)((lda + gjs::BN - 1) / gjs::BN + 1), (unsigned)ntile_m);
  auto lead = [&](int64_t k, int side) -> const double2* {  // lead block in slice k's matrix
    if (side == 0) return (k == 0) ? mp.G0[0] : nullptr;
    return (k == L - 1) ? mp.G0[1] : nullptr;
  };
  // slice k of side d: store the side's previous slice (kprev >= 0) and assemble
  //   W = A_k - g_kprev - leads (- Wx at the junction)
  auto assemble = [&](Side& d, int64_t k, int64_t kprev, const float2* Wx) {
    float* sh = kprev >= 0 ? st_hi + kprev * N * lda : st_hi;
    float* sl = kprev >= 0 ? st_lo + kprev * N * lda : st_lo;
    launch_pdl(k_mx_assemble, ga, dim3(256), 0, d.q, reinterpret_cast<float2*>(d.W[d.cur]), ldw, N, sh, sl,
               (int)(kprev >= 0), 1, mp.st_col, mp.st_val, mp.k2, mp.eps + k * N, lead(k, 0),
               two ? lead(k, 1) : (k == L - 1 ? mp.G0[1] : nullptr), Wx);
    nl++;
  };
  auto store_only = [&](Side& d, int64_t k) {
    launch_pdl(k_mx_assemble, ga, dim3(256), 0, d.q, reinterpret_cast<float2*>(d.W[d.cur]), ldw, N,
               st_hi + k * N * lda, st_lo + k * N * lda, 1, 0, mp.st_col, mp.st_val, mp.k2, mp.eps,
               (const double2*)nullptr, (const double2*)nullptr, (const float2*)nullptr);
    nl++;
  };
  auto first_t = [&](Side& d) {
    launch_pdl(k_mx_t0, dim3(1), dim3(256), 0, d.q, (const float*)d.W[d.cur], lda, (int)std::min<int64_t>(NB, N),
               d.Tb + (d.gstep & 1) * NB * NB, d.Tu + (d.gstep & 1) * gjs::TU_BYTES, mstat);
    nl++;
  };
  // one Gauss-Jordan step of side d's slice k; knext: the slice whose first
  // pivot block the server prepares after the last step (< 0: none)
  auto gj_step = [&](Side& d, int64_t j0, int64_t knext) {
    const int jn = (int)std::min<int64_t>(NB, N - j0);
    GjNext ns{};
    ns.Tin = d.Tb + (d.gstep & 1) * NB * NB;
    ns.Tout = d.Tb + ((d.gstep + 1) & 1) * NB * NB;
    ns.tu_in = d.Tu + (d.gstep & 1) * gjs::TU_BYTES;
    ns.tu_out = d.Tu + ((d.gstep + 1) & 1) * gjs::TU_BYTES;
    ns.st_col = mp.st_col;
    ns.st_val = mp.st_val;
    ns.k2 = mp.k2;
    ns.ldg = N;
    if (j0 + NB < N) {
      ns.j1 = (int)(j0 + NB);
      ns.jn1 = (int)std::min<int64_t>(NB, N - j0 - NB);
    } else if (knext >= 0) {  // the next slice's first block
      ns.j1 = 0;
      ns.jn1 = (int)std::min<int64_t>(NB, N);
      ns.next_slice = 1;
      ns.same_block = N <= NB;
      ns.eps_next = mp.eps + knext * N;
      ns.g0r = (knext == L - 1) ? mp.G0[1] : (knext == 0 ? mp.G0[0] : nullptr);
    } else {
      ns.Tout = nullptr;  // nothing follows this step within the side
    }
    launch_pdl(k_mx_gj_step, ggj, dim3(256), gjs::SMEM, d.q, d.mA[d.cur], d.mWp[d.cur], (const float*)d.W[d.cur],
               d.W[d.cur ^ 1], lda, (int)N, (int)j0, jn, ns, mstat, kGemmTimeout);
    d.cur ^= 1;
    d.gstep++;
    nl++;
  };
  if ((st = fork_sides())) return st;
  const int64_t nmax = std::max(sd[0].count, two ? sd[1].count : 0);
  for (int64_t i = 0; i < nmax; i++) {
    for (int q = 0; q < nside; q++) {
      Side& d = sd[q];
      if (i >= d.count) continue;
      const int64_t k = d.first + d.dir * i;
      assemble(d, k, i > 0 ? k - d.dir : -1, nullptr);
      if (i == 0) first_t(d);
    }
    for (int64_t j0 = 0; j0 < N; j0 += NB)
      for (int q = 0; q < nside; q++) {
        Side& d = sd[q];
        if (i >= d.count) continue;
        const int64_t k = d.first + d.dir * i;
        gj_step(d, j0, i + 1 < d.count ? k + d.dir : -1);
      }
  }
  if ((st = join_sides())) return st;
  if (two) {
    // the right side's last slice (cj) into the store, then the junction slice
    // cj - 1 = A - g_{cj-2} (left side's W) - g_{cj} (right side's W)
    Side& dl = sd[0];
    Side& dr = sd[1];
    dr.q = s;
    store_only(dr, cj);
    assemble(dl, cj - 1, cj - 2, reinterpret_cast<const float2*>(dr.W[dr.cur]));
    first_t(dl);
    for (int64_t j0 = 0; j0 < N; j0 += NB) gj_step(dl, j0, -1);
    store_only(dl, cj - 1);
    dr.q = s2;
  } else {
    store_only(sd[0], L - 1);
  }
  RGF_CUDA_TRY_MX(cudaGetLastError());
  RGF_CUDA_TRY_MX(cudaEventRecord(ev[1], s));

  // (2) sources in FP64: B columns, b_0 = G0_L B_L, b_{L-1} = G0_R B_R
  k_mx_fill_B<<<(unsigned)((NP + 255) / 256), 256, 0, s>>>(mp.phi, N, mp.prop[0], mp.prop[1], mp.sqrtmu[0],
                                                           mp.sqrtmu[1], mp.in_idx, mp.niL, P, Bl, Br);
  const double2 one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  launch_zgemm(N, P, N, one, ZOp{mp.G0[0], N, 0}, ZOp{Bl, P, 0}, zero, b0, P, s);
  launch_zgemm(N, P, N, one, ZOp{mp.G0[1], N, 0}, ZOp{Br, P, 0}, zero, bL, P, s);
  nl += 3;

  // (3) refinement
  tc32::GemmArgs gs[2];
  for (int q = 0; q < nside; q++) {
    gs[q] = tc32::GemmArgs{};
    gs[q].M = (int)N;
    gs[q].Nr = (int)(2 * P);
    gs[q].k_chunks = kchunks / sSplit;
    gs[q].mode = tc32::kPartial;
    gs[q].out = reinterpret_cast<float*>(sd[q].part);
    gs[q].ldo = 2 * P;
    gs[q].split_stride = 2 * NP;
    gs[q].err = mstat;
    gs[q].timeout = kGemmTimeout;
  }
  const dim3 gsg((unsigned)sTiles, (unsigned)ntile_m, (unsigned)sSplit);
  const dim3 gp((unsigned)((P + 31) / 32), (unsigned)((N + 31) / 32));
  const dim3 tp(32, 8);
  // side q's GEMM: partials = g_k Bt (Bt of side qb, default q)
  auto gemm = [&](int q, int64_t k, cudaStream_t qs) {
    gs[q].a_z = (int)k;
    if (sbn == 64)
      launch_pdl(tc32::k_tc32_gemm<64>, gsg, dim3(tc32::kThreads), tc32::Cfg<64>::SMEM, qs, mSh, mSl, sd[q].mBh,
                 sd[q].mBl, gs[q]);
    else
      launch_pdl(tc32::k_tc32_gemm<128>, gsg, dim3(tc32::kThreads), tc32::Cfg<128>::SMEM, qs, mSh, mSl, sd[q].mBh,
                 sd[q].mBl, gs[q]);
    nl++;
  };
  auto fwd_prep = [&](int q, int64_t k, int64_t kprev, cudaStream_t qs, int q2 = -1, int64_t kprev2 = -1) {
    launch_pdl(k_mx_fwd_prep, gp, tp, 0, qs, k, kprev, N, P, P, (int64_t)0, y, (const float2*)sd[q].part, sSplit,
               (const float2*)(q2 >= 0 ? sd[q2].part : nullptr), kprev2, sSplit, sd[q].bh, sd[q].bl, lda,
               (const int*)nullptr);
    nl++;
  };
  auto bwd_prep = [&](int q, int64_t k, int add_y, int write_bt, cudaStream_t qs, int q2 = -1) {
    launch_pdl(k_mx_bwd_prep, gp, tp, 0, qs, k, L, N, P, P, (int64_t)0, x, (const float2*)y,
               (const float2*)sd[q].part, sSplit, sd[q].bh, sd[q].bl, lda, norms, (const int*)nullptr, add_y,
               write_bt, q2 >= 0 ? sd[q2].bh : nullptr, q2 >= 0 ? sd[q2].bl : nullptr);
    nl++;
  };
  double prev = 1.0, change = 1.0;
  bool conv = false;
  int it = 0;
  for (; it < kMaxIter; it++) {
    const bool have_x = it > 0;
    if (have_x) {  // lead blocks of the residual: G0_L x_0, G0_R x_{L-1}
      launch_zgemm(N, P, N, one, ZOp{mp.G0[0], N, 0}, ZOp{x, P, 0}, zero, e0, P, s);
      launch_zgemm(N, P, N, one, ZOp{mp.G0[1], N, 0}, ZOp{x + (L - 1) * NP, P, 0}, zero, e1, P, s);
      nl += 2;
    }
    RGF_CUDA_TRY_MX(cudaMemsetAsync(norms, 0, sizeof(double) * 8, s));
    launch_pdl(k_mx_residual, dim3((unsigned)((P + 31) / 32), (unsigned)((N + 7) / 8), (unsigned)std::min<int64_t>(L, 65535)),
               dim3(32, 8), 0, s, L, N, P, (const double2*)x, y, mp.eps, mp.st_col, mp.st_val, mp.k2,
               (const double2*)b0, (const double2*)bL, (const double2*)(have_x ? e0 : nullptr),
               (const double2*)(have_x ? e1 : nullptr));
    nl++;
    if (!two) {
      // forward y_k = g_k (r_k + y_{k-1}), backward d_k = y_k + g_k d_{k+1}
      for (int64_t k = 0; k < L; k++) {
        fwd_prep(0, k, k - 1, s);
        gemm(0, k, s);
      }
      for (int64_t k = L - 1; k >= 0; k--) {
        bwd_prep(0, k, k < L - 1, k > 0, s);
        if (k > 0) gemm(0, k - 1, s);
      }
    } else {
      // forward from both leads towards the junction slice cj - 1
      if ((st = fork_sides())) return st;
      const int64_t nmx = std::max(sd[0].count, sd[1].count);
      for (int64_t i = 0; i < nmx; i++)
        for (int q = 0; q < 2; q++) {
          if (i >= sd[q].count) continue;
          const int64_t k = sd[q].first + sd[q].dir * i;
          fwd_prep(q, k, i > 0 ? k - sd[q].dir : -1, sd[q].q);
          gemm(q, k, sd[q].q);
        }
      if ((st = join_sides())) return st;
      // junction: d_{cj-1} = G_{cj-1} (r + y_{cj-2} + y_{cj}), into both sides' Bt
      fwd_prep(0, cj - 1, cj - 2, s, 1, cj);
      gemm(0, cj - 1, s);
      bwd_prep(0, cj - 1, 0, 1, s, 1);
      // backward outwards: d_k = y_k + g_k d_{k +- 1}
      if ((st = fork_sides())) return st;
      for (int64_t i = nmx - 1; i >= 0; i--)
        for (int q = 0; q < 2; q++) {
          if (i >= sd[q].count) continue;
          const int64_t k = sd[q].first + sd[q].dir * i;
          gemm(q, k, sd[q].q);
          bwd_prep(q, k, 1, i > 0, sd[q].q);
        }
      if ((st = join_sides())) return st;
    }
    RGF_CUDA_TRY_MX(cudaGetLastError());
    double hn[8];
    int hs = 0;
    RGF_CUDA_TRY_MX(cudaMemcpyAsync(hn, norms, sizeof(hn), cudaMemcpyDeviceToHost, s));
    RGF_CUDA_TRY_MX(cudaMemcpyAsync(&hs, mstat, sizeof(int), cudaMemcpyDeviceToHost, s));
    RGF_CUDA_TRY_MX(cudaStreamSynchronize(s));
    if (hs & kStatusTimeout) {
      set_error("a device-side wait of the tensor-core GEMM timed out");
      return RGF_ERR_TIMEOUT;
    }
    auto ratio = [](double d, double xv) { return xv > 0.0 ? sqrt(d / xv) : (d > 0.0 ? 1e300 : 0.0); };
    change = std::max(ratio(hn[0], hn[1]), std::max(ratio(hn[2], hn[3]), ratio(hn[4], hn[5])));
    if (!isfinite(change) || (hs & kStatusSingular)) break;
    if (it > 0) {
      const double rho = change / prev;  // observed contraction of the refinement
      if (change <= kTolStop || (rho < 0.5 && change * rho <= kTolNext)) {
        conv = true;
        it++;
        break;
      }
      if (rho >= 0.5) break;  // the factor is too poor a preconditioner: FP64 form
    }
    prev = change;
  }
  RGF_CUDA_TRY_MX(cudaEventRecord(ev[2], s));
  if (stats) {
    stats->iterations = it;
    stats->converged = conv;
    stats->last_change = change;
  }
  if (launches) *launches += nl;
  if (!conv) {
    RGF_CUDA_TRY_MX(cudaStreamSynchronize(s));
    return kMixedNotConverged;
  }

  // (4) S: X_L = G0_L (B_L + x_0), X_R = G0_R (B_R + x_{L-1}), Fisher-Lee
  k_mx_add<<<(unsigned)((NP + 255) / 256), 256, 0, s>>>(Bl, x, b0, NP);
  k_mx_add<<<(unsigned)((NP + 255) / 256), 256, 0, s>>>(Br, x + (L - 1) * NP, bL, NP);
  launch_zgemm(N, P, N, one, ZOp{mp.G0[0], N, 0}, ZOp{b0, P, 0}, zero, e0, P, s);
  launch_zgemm(N, P, N, one, ZOp{mp.G0[1], N, 0}, ZOp{bL, P, 0}, zero, e1, P, s);
  const int64_t nw = n_out * P;
  k_mx_extract<<<(unsigned)((nw * 32 + 255) / 256), 256, 0, s>>>(mp.phi, N, mp.prop[0], mp.prop[1], mp.sqrtmu[0],
                                                                 mp.sqrtmu[1], mp.out_idx, mp.noL, (int)n_out, P, e0,
                                                                 e1, mp.S, mp.ldS);
  if (mp.npairs > 0) k_mx_delta<<<(mp.npairs + 255) / 256, 256, 0, s>>>(mp.S, mp.ldS, mp.pairs, mp.npairs);
  RGF_CUDA_TRY_MX(cudaGetLastError());
  if (launches) *launches += 6;
  if (stats) {
    float f = 0.f, g = 0.f;
    RGF_CUDA_TRY_MX(cudaEventSynchronize(ev[2]));
    cudaEventElapsedTime(&f, ev[0], ev[1]);
    cudaEventElapsedTime(&g, ev[1], ev[2]);
    stats->factor_ms = f;
    stats->solve_ms = g;
  }
  return RGF_OK;
}

}  // namespace rgf

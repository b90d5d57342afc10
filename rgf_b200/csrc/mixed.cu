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
#include <vector>

#include "mixed.cuh"
#include "sweep.cuh"
#include "tc32.cuh"

namespace rgf {
namespace {

constexpr int NB = 64;            // pivot block width (complex)
constexpr int KB = 2 * NB;        // real K of the update GEMM
constexpr int kSolveBN = 64;      // tile width of the solve GEMMs
constexpr int kUpdateBN = 128;    // tile width of the update GEMMs
constexpr int kMaxIter = 8;
// x has converged when the last correction, or the correction the next pass
// would make (the last one times the observed contraction), is below this
constexpr double kTolStop = 1e-13;
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

// ---------------------------------------------------------------------------
// factorization kernels
// ---------------------------------------------------------------------------

// W holds g_{k-1} (store != 0: written to the factor store as hi/lo) and is
// replaced by the next slice matrix (assemble != 0):
//   W = A_k - g_{k-1} - Ga - Gb,  A_k = stencil - k0dx^2 eps_k on the diagonal.
// Columns [N, ldw) are the zero padding of the store rows.
__global__ void k_mx_assemble(float2* W, int64_t ldw, int64_t N, float* st_hi, float* st_lo, int store,
                              int assemble, const int* st_col, const double2* st_val, double2 k2,
                              const double2* eps, const double2* Ga, const double2* Gb) {
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
#pragma unroll
    for (int q = 0; q < kMaxStencil; q++)
      if (st_col[i * kMaxStencil + q] == j) v = cadd(v, st_val[i * kMaxStencil + q]);
    if (i == j) v = csub(v, cmul(k2, eps[i]));
    W[o] = make_float2((float)v.x, (float)v.y);
  }
}

// Block 0: T = inverse of the jn x jn pivot block W(J, J) by Gauss-Jordan on
// diagonal pivots, register-resident (thread t holds row t/4, columns
// t%4 + 4q), one barrier per pivot; T is NB x NB with zero padding.  Flags
// kStatusSingular on a zero or non-finite pivot.
// Blocks 1..: the update's left operand V = W(:, J) - E_J (E_J the identity's
// columns J), split hi/lo, NB complex columns per row (zero beyond jn).
__global__ void __launch_bounds__(256) k_mx_panel(const float2* W, int64_t ldw, int64_t N, int64_t j0, int jn,
                                                  float2* T, float* V_hi, float* V_lo, int* status) {
  const int tid = threadIdx.x;
  if (blockIdx.x == 0) {
    __shared__ float2 rowb[2][NB];
    __shared__ float2 colb[2][NB];
    const int r = tid >> 2, cq = tid & 3;
    float2 a[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int c = cq + 4 * q;
      a[q] = (r < jn && c < jn) ? W[(j0 + r) * ldw + j0 + c] : make_float2(0.f, 0.f);
    }
    bool bad = false;
    for (int k = 0; k < jn; k++) {
      const int b = k & 1;
      if (r == k) {
#pragma unroll
        for (int q = 0; q < 16; q++) rowb[b][cq + 4 * q] = a[q];
      }
      if (cq == (k & 3)) {
#pragma unroll
        for (int q = 0; q < 16; q++)
          if (q == (k >> 2)) colb[b][r] = a[q];
      }
      __syncthreads();
      const float2 p = rowb[b][k];
      const float d = p.x * p.x + p.y * p.y;
      const float id = 1.f / d;
      const float2 pinv = make_float2(p.x * id, -p.y * id);
      if (!(d > 0.f) || !isfinite(id)) bad = true;
      if (r == k) {
#pragma unroll
        for (int q = 0; q < 16; q++) a[q] = (cq + 4 * q == k) ? pinv : fcmul(a[q], pinv);
      } else {
        const float2 fp = fcmul(colb[b][r], pinv);
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const int c = cq + 4 * q;
          const float2 u = fcmul(fp, rowb[b][c]);
          a[q] = (c == k) ? make_float2(-fp.x, -fp.y) : make_float2(a[q].x - u.x, a[q].y - u.y);
        }
      }
    }
    if (bad && tid == 0) atomicOr(status, kStatusSingular);
#pragma unroll
    for (int q = 0; q < 16; q++) T[r * NB + cq + 4 * q] = a[q];
    return;
  }
  const int64_t r0 = (int64_t)(blockIdx.x - 1) * 64;
  for (int e = tid; e < 64 * NB; e += 256) {
    const int64_t i = r0 + e / NB;
    const int t = e % NB;
    if (i >= N) break;
    float2 w = make_float2(0.f, 0.f);
    if (t < jn) {
      w = W[i * ldw + j0 + t];
      if (i == j0 + t) w.x -= 1.f;
    }
    split2(w.x, w.y, V_hi + i * KB + 2 * t, V_lo + i * KB + 2 * t);
  }
}

// Row panel U = T W'(J, :) (W'(J, J) = I, so U(:, J) = T) for 16 columns per
// block, written as the update's right operand: rows 2c, 2c+1 of Ut (K = 2t,
// 2t+1), Ut[2c][2t] = Re U[t][c], Ut[2c][2t+1] = -Im, Ut[2c+1][2t] = Im,
// Ut[2c+1][2t+1] = Re; hi/lo split.
__global__ void __launch_bounds__(256) k_mx_rowpanel(const float2* W, int64_t ldw, int64_t N, int64_t j0, int jn,
                                                     const float2* T, float* U_hi, float* U_lo) {
  __shared__ float2 Ts[NB][NB + 1];
  __shared__ float2 Ws[NB][17];
  const int tid = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * 16;
  for (int e = tid; e < NB * NB; e += 256) Ts[e / NB][e % NB] = T[e];
  for (int e = tid; e < NB * 16; e += 256) {
    const int sr = e / 16, cl = e % 16;
    const int64_t c = c0 + cl;
    float2 w = make_float2(0.f, 0.f);
    if (c < N && sr < jn) {
      if (c >= j0 && c < j0 + jn)
        w.x = (j0 + sr == c) ? 1.f : 0.f;
      else
        w = W[(j0 + sr) * ldw + c];
    }
    Ws[sr][cl] = w;
  }
  __syncthreads();
  const int t = tid >> 2, cl0 = (tid & 3) * 4;
  float2 acc[4] = {};
  for (int sr = 0; sr < NB; sr++) {
    const float2 tv = Ts[t][sr];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const float2 wv = Ws[sr][cl0 + u];
      acc[u].x += tv.x * wv.x - tv.y * wv.y;
      acc[u].y += tv.x * wv.y + tv.y * wv.x;
    }
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int64_t c = c0 + cl0 + u;
    if (c >= N) break;
    const float2 v = acc[u];
    split2(v.x, -v.y, U_hi + (2 * c) * KB + 2 * t, U_lo + (2 * c) * KB + 2 * t);
    split2(v.y, v.x, U_hi + (2 * c + 1) * KB + 2 * t, U_lo + (2 * c + 1) * KB + 2 * t);
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
  for (int q = threadIdx.y; q < 32; q += 8) {
    const int64_t p = p0 + q, i = i0 + threadIdx.x;
    if (p < P && i < N) {
      const float2 v = tile[q][threadIdx.x];
      split2(v.x, -v.y, bt_hi + (2 * p) * lda + 2 * i, bt_lo + (2 * p) * lda + 2 * i);
      split2(v.y, v.x, bt_hi + (2 * p + 1) * lda + 2 * i, bt_lo + (2 * p + 1) * lda + 2 * i);
    }
  }
}

// forward pass, slice k: y_{k-1} = (GEMM partials) -> ystore; r_k = b_k - (H x)_k
// in FP64; v_k = r_k + y_{k-1} -> Bt.
__global__ void __launch_bounds__(256) k_mx_fwd_prep(int64_t k, int64_t L, int64_t N, int64_t P, const double2* x,
                                                     float2* ystore, const float2* part, int ksplit,
                                                     const double2* eps_k, const int* st_col,
                                                     const double2* st_val, double2 k2, const double2* b0,
                                                     const double2* bL, const double2* e0, const double2* e1,
                                                     float* bt_hi, float* bt_lo, int64_t lda) {
  __shared__ float2 tile[32][33];
  const int64_t p0 = blockIdx.x * 32, i0 = blockIdx.y * 32, NP = N * P;
  const int64_t p = p0 + threadIdx.x;
  const double2* xk = x + k * NP;
  for (int q = threadIdx.y; q < 32; q += 8) {
    const int64_t i = i0 + q;
    float2 v = make_float2(0.f, 0.f);
    if (i < N && p < P) {
      const int64_t ip = i * P + p;
      float2 yp = make_float2(0.f, 0.f);
      if (k > 0) {
        yp = sum_parts(part, ksplit, NP, ip);
        ystore[(k - 1) * NP + ip] = yp;
      }
      double2 r = cmk(0.0, 0.0);
      if (k == 0) {
        r = cadd(r, b0[ip]);
        if (e0) r = cadd(r, e0[ip]);
      }
      if (k == L - 1) {
        r = cadd(r, bL[ip]);
        if (e1) r = cadd(r, e1[ip]);
      }
      double2 ax = cneg(cmul(cmul(k2, eps_k[i]), xk[ip]));
#pragma unroll
      for (int qq = 0; qq < kMaxStencil; qq++) {
        const int c = st_col[i * kMaxStencil + qq];
        if (c >= 0) ax = cadd(ax, cmul(st_val[i * kMaxStencil + qq], xk[(int64_t)c * P + p]));
      }
      r = csub(r, ax);
      if (k > 0) r = cadd(r, xk[ip - NP]);
      if (k < L - 1) r = cadd(r, xk[ip + NP]);
      v = make_float2((float)r.x + yp.x, (float)r.y + yp.y);
    }
    tile[threadIdx.x][q] = v;
  }
  __syncthreads();
  store_bt(tile, p0, i0, N, P, bt_hi, bt_lo, lda);
}

// backward pass, slice k: d_k = y_k + (GEMM partials) (k = L-1: the partials
// are y_{L-1}); x_k += d_k in FP64; norms of d and x (whole; slice 0; slice
// L-1); for k > 0 d_k -> Bt.
__global__ void __launch_bounds__(256) k_mx_bwd_prep(int64_t k, int64_t L, int64_t N, int64_t P, double2* x,
                                                     const float2* ystore, const float2* part, int ksplit,
                                                     float* bt_hi, float* bt_lo, int64_t lda, double* norms) {
  __shared__ float2 tile[32][33];
  __shared__ double red[2][8];
  const int64_t p0 = blockIdx.x * 32, i0 = blockIdx.y * 32, NP = N * P;
  const int64_t p = p0 + threadIdx.x;
  double dd = 0.0, xx = 0.0;
  for (int q = threadIdx.y; q < 32; q += 8) {
    const int64_t i = i0 + q;
    float2 d = make_float2(0.f, 0.f);
    if (i < N && p < P) {
      const int64_t ip = i * P + p;
      d = sum_parts(part, ksplit, NP, ip);
      if (k < L - 1) {
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
  if (k > 0) store_bt(tile, p0, i0, N, P, bt_hi, bt_lo, lda);
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

size_t mixed_workspace_bytes(int64_t N, int64_t L, int64_t P) {
  const int64_t lda = lda_of(N), ldw = lda / 2;
  size_t b = 0;
  b += sizeof(float2) * N * ldw;              // W
  b += 2 * sizeof(float) * N * KB;            // V hi/lo
  b += 2 * sizeof(float) * 2 * N * KB;        // U hi/lo
  b += sizeof(float2) * NB * NB;              // T
  b += 2 * sizeof(float) * N * lda * L;       // factor store hi/lo
  b += sizeof(double2) * N * P * L;           // x
  b += sizeof(float2) * N * P * L;            // y
  b += sizeof(float2) * N * P * 148;          // partials (at most one per SM)
  b += 2 * sizeof(float) * 2 * P * lda;       // Bt hi/lo
  b += sizeof(double2) * N * P * 6;           // Bl, Br, b0, bL, e0/e1 (also G0 (B + x) at the end)
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
  if ((st = gemm_attr<kSolveBN>()) || (st = gemm_attr<kUpdateBN>())) return st;
  void *pW, *pV, *pU, *pT, *pSh, *pSl, *pX, *pY, *pPart, *pBt, *pVec, *pNorm, *pStat;
  const int ntile_m = (int)((N + tc32::BM - 1) / tc32::BM);
  const int ntile_s = (int)((2 * P + kSolveBN - 1) / kSolveBN);
  const int kchunks = (int)(lda / tc32::BK);
  const int ksplit = choose_ksplit((int64_t)ntile_m * ntile_s, kchunks, sms);
  if ((st = alloc(kMxW, sizeof(float2) * N * ldw, &pW)) || (st = alloc(kMxV, 2 * sizeof(float) * N * KB, &pV)) ||
      (st = alloc(kMxU, 2 * sizeof(float) * 2 * N * KB, &pU)) || (st = alloc(kMxT, sizeof(float2) * NB * NB, &pT)) ||
      (st = alloc(kMxStoreHi, sizeof(float) * N * lda * L, &pSh)) ||
      (st = alloc(kMxStoreLo, sizeof(float) * N * lda * L, &pSl)) ||
      (st = alloc(kMxX, sizeof(double2) * NP * L, &pX)) || (st = alloc(kMxY, sizeof(float2) * NP * L, &pY)) ||
      (st = alloc(kMxPart, sizeof(float2) * NP * ksplit, &pPart)) ||
      (st = alloc(kMxBt, 2 * sizeof(float) * 2 * P * lda, &pBt)) ||
      (st = alloc(kMxVec, sizeof(double2) * NP * 6, &pVec)) || (st = alloc(kMxNorm, sizeof(double) * 8, &pNorm)) ||
      (st = alloc(kMxStatus, sizeof(int), &pStat)))
    return st;
  float2* W = static_cast<float2*>(pW);
  float* V_hi = static_cast<float*>(pV);
  float* V_lo = V_hi + N * KB;
  float* U_hi = static_cast<float*>(pU);
  float* U_lo = U_hi + 2 * N * KB;
  float2* T = static_cast<float2*>(pT);
  float* st_hi = static_cast<float*>(pSh);
  float* st_lo = static_cast<float*>(pSl);
  double2* x = static_cast<double2*>(pX);
  float2* y = static_cast<float2*>(pY);
  float2* part = static_cast<float2*>(pPart);
  float* bt_hi = static_cast<float*>(pBt);
  float* bt_lo = bt_hi + 2 * P * lda;
  double2* Bl = static_cast<double2*>(pVec);
  double2* Br = Bl + NP;
  double2* b0 = Br + NP;
  double2* bL = b0 + NP;
  double2* e0 = bL + NP;
  double2* e1 = e0 + NP;
  double* norms = static_cast<double*>(pNorm);
  int* mstat = static_cast<int*>(pStat);

  // tensor maps: update operands (V: N rows, Ut: 2N rows, K = 128), factor
  // store (N rows x lda, L slices), solve right operand (2P rows x lda)
  CUtensorMap mVh, mVl, mUh, mUl, mSh, mSl, mBh, mBl;
  if (!(tc32::make_map(&mVh, V_hi, KB, N, 1, KB, 0, tc32::BM) && tc32::make_map(&mVl, V_lo, KB, N, 1, KB, 0, tc32::BM) &&
        tc32::make_map(&mUh, U_hi, KB, 2 * N, 1, KB, 0, kUpdateBN) &&
        tc32::make_map(&mUl, U_lo, KB, 2 * N, 1, KB, 0, kUpdateBN) &&
        tc32::make_map(&mSh, st_hi, lda, N, L, lda, N * lda, tc32::BM) &&
        tc32::make_map(&mSl, st_lo, lda, N, L, lda, N * lda, tc32::BM) &&
        tc32::make_map(&mBh, bt_hi, lda, 2 * P, 1, lda, 0, kSolveBN) &&
        tc32::make_map(&mBl, bt_lo, lda, 2 * P, 1, lda, 0, kSolveBN))) {
    set_error("tensor-map encoding for the tcgen05 GEMM failed");
    return RGF_ERR_CUDA;
  }
  RGF_CUDA_TRY_MX(cudaMemsetAsync(mstat, 0, sizeof(int), s));
  RGF_CUDA_TRY_MX(cudaMemsetAsync(bt_hi, 0, 2 * sizeof(float) * 2 * P * lda, s));
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
  const unsigned panel_blocks = (unsigned)(1 + (N + 63) / 64);
  const unsigned row_blocks = (unsigned)((N + 15) / 16);
  const dim3 gu((unsigned)((2 * N + kUpdateBN - 1) / kUpdateBN), (unsigned)ntile_m, 1);
  tc32::GemmArgs gu_args{};
  gu_args.M = (int)N;
  gu_args.Nr = (int)(2 * N);
  gu_args.k_chunks = KB / tc32::BK;
  gu_args.mode = tc32::kGJ;
  gu_args.out = reinterpret_cast<float*>(W);
  gu_args.ldo = 2 * ldw;
  gu_args.err = mstat;
  gu_args.timeout = kGemmTimeout;
  for (int64_t k = 0; k < L; k++) {
    const double2* Ga = (k == 0) ? mp.G0[0] : nullptr;
    const double2* Gb = (k == L - 1) ? mp.G0[1] : nullptr;
    float* sh = k > 0 ? st_hi + (k - 1) * N * lda : st_hi;
    float* sl = k > 0 ? st_lo + (k - 1) * N * lda : st_lo;
    k_mx_assemble<<<ga, 256, 0, s>>>(W, ldw, N, sh, sl, k > 0, 1, mp.st_col, mp.st_val, mp.k2, mp.eps + k * N, Ga,
                                     Gb);
    nl++;
    for (int64_t j0 = 0; j0 < N; j0 += NB) {
      const int jn = (int)std::min<int64_t>(NB, N - j0);
      k_mx_panel<<<panel_blocks, 256, 0, s>>>(W, ldw, N, j0, jn, T, V_hi, V_lo, mstat);
      k_mx_rowpanel<<<row_blocks, 256, 0, s>>>(W, ldw, N, j0, jn, T, U_hi, U_lo);
      gu_args.gj_c0 = (int)j0;
      gu_args.gj_nb = jn;
      tc32::k_tc32_gemm<kUpdateBN><<<gu, tc32::kThreads, tc32::Cfg<kUpdateBN>::SMEM, s>>>(mVh, mVl, mUh, mUl,
                                                                                           gu_args);
      nl += 3;
    }
  }
  k_mx_assemble<<<ga, 256, 0, s>>>(W, ldw, N, st_hi + (L - 1) * N * lda, st_lo + (L - 1) * N * lda, 1, 0,
                                   mp.st_col, mp.st_val, mp.k2, mp.eps, nullptr, nullptr);
  nl++;
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
  tc32::GemmArgs gs{};
  gs.M = (int)N;
  gs.Nr = (int)(2 * P);
  gs.k_chunks = kchunks / ksplit;
  gs.mode = tc32::kPartial;
  gs.out = reinterpret_cast<float*>(part);
  gs.ldo = 2 * P;
  gs.split_stride = 2 * NP;
  gs.err = mstat;
  gs.timeout = kGemmTimeout;
  const dim3 gsg((unsigned)ntile_s, (unsigned)ntile_m, (unsigned)ksplit);
  const dim3 gp((unsigned)((P + 31) / 32), (unsigned)((N + 31) / 32));
  const dim3 tp(32, 8);
  auto gemm = [&](int64_t k) {
    gs.a_z = (int)k;
    tc32::k_tc32_gemm<kSolveBN><<<gsg, tc32::kThreads, tc32::Cfg<kSolveBN>::SMEM, s>>>(mSh, mSl, mBh, mBl, gs);
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
    for (int64_t k = 0; k < L; k++) {
      k_mx_fwd_prep<<<gp, tp, 0, s>>>(k, L, N, P, x, y, part, ksplit, mp.eps + k * N, mp.st_col, mp.st_val, mp.k2,
                                      b0, bL, have_x ? e0 : nullptr, have_x ? e1 : nullptr, bt_hi, bt_lo, lda);
      gemm(k);
      nl += 2;
    }
    for (int64_t k = L - 1; k >= 0; k--) {
      k_mx_bwd_prep<<<gp, tp, 0, s>>>(k, L, N, P, x, y, part, ksplit, bt_hi, bt_lo, lda, norms);
      nl++;
      if (k > 0) {
        gemm(k - 1);
        nl++;
      }
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
      if (change <= kTolStop || (rho < 0.5 && change * rho <= kTolStop)) {
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

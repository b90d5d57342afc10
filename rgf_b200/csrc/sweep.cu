// Slice recursion kernels: complex FP64 tensor-core (DMMA) GEMM, the blocked
// Gauss-Jordan sweep of the augmented slice matrix, slice assembly, lead
// attachment and the Fisher-Lee extraction.
//
// The recursion of cal_smatrix_RGF.m:257-280 is carried as one augmented
// matrix per slice n
//
//         [ A_n - G_{n-1}   X ]        X = G_RL B_L   (N x P_in)
//   W_n = [                   ]        Z = C_L G_LR   (P_out x N)
//         [ -Z              Y ]        Y = C_L G_LL B_L
//
// and sweeping (block Gauss-Jordan pivoting) its first N indices yields
//
//         [ G_n        G_n X       ]
//         [ Z G_n      Y + Z G_n X ]
//
// i.e. G_RR = inv(A_n - G_RR), G_RL = G_RR G_RL, G_LL += G_LR G_RL and
// G_LR = G_LR G_RR (cal_smatrix_RGF.m:265-268) projected on the requested
// channels, in one pass.  The lead on the far side is attached the same way
// (cal_smatrix_RGF.m:272-275) with G0_R^{-1} = A_lead - G0_R, and the last
// sweep's corner block is the Fisher-Lee S/(-2i) (cal_smatrix_RGF.m:279).
#include "sweep.cuh"

namespace rgf {

__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ double2 zop_load(const ZOp& o, int64_t r, int64_t c) {
  if (o.op == 0) return o.p[r * o.ld + c];
  double2 v = o.p[c * o.ld + r];
  return (o.op == 2) ? cconj(v) : v;
}

// ---------------------------------------------------------------------------
// C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C, complex FP64 on
// the FP64 tensor cores (mma.sync m8n8k4 .f64, four real products per complex
// product).  64x64 output tile per CTA, 4 warps of 32x32, K staged in
// 32-wide chunks through shared memory.  With kMask the old C is read as
// zero on rows and columns [j0, j0+jn) (the pivot block of a sweep step).
// ---------------------------------------------------------------------------
constexpr int kBM = 64, kBN = 64, kBK = 32;
constexpr int kAS = kBK + 4;  // smem row stride (complex) of the A tile: conflict-free fragment loads
constexpr int kBS = kBN + 2;  // smem row stride of the B tile
constexpr size_t kGemmSmem = sizeof(double2) * (kBM * kAS + kBK * kBS);

template <bool kMask>
__global__ void __launch_bounds__(128) k_zgemm(int64_t M, int64_t N, int64_t K, double2 alpha, ZOp A,
                                               ZOp B, double2 beta, double2* C, int64_t ldc,
                                               int64_t j0, int64_t jn, ZAdd add) {
  extern __shared__ double2 smem[];
  double2* As = smem;               // [kBM][kAS]
  double2* Bs = smem + kBM * kAS;   // [kBK][kBS]
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, wr = warp >> 1, wc = warp & 1;
  const int64_t m0 = (int64_t)blockIdx.y * kBM, n0 = (int64_t)blockIdx.x * kBN;
  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

  for (int64_t k0 = 0; k0 < K; k0 += kBK) {
    // stage A (kBM x kBK) and B (kBK x kBN)
#pragma unroll 4
    for (int i = 0; i < (kBM * kBK) / 128; i++) {
      int e = t + 128 * i, r, k;
      if (A.op == 0) { r = e >> 5; k = e & 31; } else { r = e & 63; k = e >> 6; }
      int64_t gr = m0 + r, gk = k0 + k;
      As[r * kAS + k] = (gr < M && gk < K) ? zop_load(A, gr, gk) : cmk(0.0, 0.0);
    }
#pragma unroll 4
    for (int i = 0; i < (kBK * kBN) / 128; i++) {
      int e = t + 128 * i, k, c;
      if (B.op == 0) { k = e >> 6; c = e & 63; } else { k = e & 31; c = e >> 5; }
      int64_t gk = k0 + k, gc = n0 + c;
      Bs[k * kBS + c] = (gk < K && gc < N) ? zop_load(B, gk, gc) : cmk(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK / 4; kk++) {
      double2 a[4], b[4];
#pragma unroll
      for (int mi = 0; mi < 4; mi++) a[mi] = As[(wr * 32 + mi * 8 + (lane >> 2)) * kAS + kk * 4 + (lane & 3)];
#pragma unroll
      for (int ni = 0; ni < 4; ni++) b[ni] = Bs[(kk * 4 + (lane & 3)) * kBS + wc * 32 + ni * 8 + (lane >> 2)];
#pragma unroll
      for (int mi = 0; mi < 4; mi++) {
        const double nai = -a[mi].y;
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
          dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi].x, b[ni].x);
          dmma884(acc[mi][ni][0], acc[mi][ni][1], nai, b[ni].y);
          dmma884(acc[mi][ni][2], acc[mi][ni][3], a[mi].x, b[ni].y);
          dmma884(acc[mi][ni][2], acc[mi][ni][3], a[mi].y, b[ni].x);
        }
      }
    }
    __syncthreads();
  }
  // epilogue
  const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
  for (int mi = 0; mi < 4; mi++) {
    const int64_t r = m0 + wr * 32 + mi * 8 + (lane >> 2);
    if (r >= M) continue;
    const bool rmask = kMask && (r >= j0 && r < j0 + jn);
#pragma unroll
    for (int ni = 0; ni < 4; ni++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t c = n0 + wc * 32 + ni * 8 + (lane & 3) * 2 + h;
        if (c >= N) continue;
        double2 v = cmul(alpha, cmk(acc[mi][ni][h], acc[mi][ni][2 + h]));
        if (use_beta) {
          const bool masked = kMask && (rmask || (c >= j0 && c < j0 + jn));
          if (!masked) v = cadd(v, cmul(beta, C[r * ldc + c]));
        }
        if (add.p && r < add.rows && c < add.cols) v = cadd(v, add.p[r * add.ld + c]);
        C[r * ldc + c] = v;
      }
    }
  }
}

static void zgemm_attr() {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_zgemm<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    cudaFuncSetAttribute(k_zgemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    attr = true;
  }
}

void launch_zgemm(int64_t M, int64_t N, int64_t K, double2 alpha, ZOp A, ZOp B, double2 beta,
                  double2* C, int64_t ldc, cudaStream_t s) {
  zgemm_attr();
  dim3 grid((unsigned)((N + kBN - 1) / kBN), (unsigned)((M + kBM - 1) / kBM));
  k_zgemm<false><<<grid, 128, kGemmSmem, s>>>(M, N, K, alpha, A, B, beta, C, ldc, 0, 0, ZAdd{nullptr, 0, 0, 0});
}

// C = A B + add (add read in its rows x cols corner, zero elsewhere)
void launch_zgemm_add(int64_t M, int64_t N, int64_t K, ZOp A, ZOp B, ZAdd add, double2* C, int64_t ldc,
                      cudaStream_t s) {
  zgemm_attr();
  dim3 grid((unsigned)((N + kBN - 1) / kBN), (unsigned)((M + kBM - 1) / kBM));
  k_zgemm<false><<<grid, 128, kGemmSmem, s>>>(M, N, K, cmk(1.0, 0.0), A, B, cmk(0.0, 0.0), C, ldc, 0, 0, add);
}

// ---------------------------------------------------------------------------
// Sweep step, part 1 (panel): every CTA inverts the jn x jn pivot block
// M[J,J] (J = [j0, j0+jn)) in shared memory -- Gauss-Jordan with partial
// pivoting inside the block, pivot search by warp shuffles -- then writes
//   U[:, c]  = T * M[J, c]     (c not in J),   U[:, J] = T        (kSw x Cc)
//   Pc[i, :] = M[i, J]         (i not in J),   Pc[J, :] = -I      (R x kSw)
// for its chunk of columns / rows.  T = M[J,J]^{-1}.
// ---------------------------------------------------------------------------
constexpr int kSw = 32;  // pivot-block width (K of the rank-kSw update)

__device__ void invert_block(double2 (*Ts)[kSw + 1], int* perm, int jn, int* status) {
  __shared__ int piv_s;
  __shared__ double2 prow[kSw], fcol[kSw];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int p = 0; p < jn; p++) {
    if (warp == 0) {
      // |re| + |im|, the magnitude LAPACK's izamax compares
      double mag = (lane >= p && lane < jn) ? fabs(Ts[lane][p].x) + fabs(Ts[lane][p].y) : -1.0;
      int idx = lane;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double om = __shfl_down_sync(0xffffffffu, mag, off);
        int oi = __shfl_down_sync(0xffffffffu, idx, off);
        if (om > mag || (om == mag && oi < idx)) { mag = om; idx = oi; }
      }
      if (lane == 0) {
        piv_s = idx;
        if (!(mag > 0.0) || !isfinite(mag)) atomicOr(status, kStatusSingular);
      }
    }
    __syncthreads();
    const int q = piv_s;
    if (q != p && t < kSw) {
      double2 tmp = Ts[p][t];
      Ts[p][t] = Ts[q][t];
      Ts[q][t] = tmp;
      if (t == 0) { int ti = perm[p]; perm[p] = perm[q]; perm[q] = ti; }
    }
    __syncthreads();
    const double2 d = cinv(Ts[p][p]);
    if (t < kSw) {
      prow[t] = (t == p) ? d : cmul(Ts[p][t], d);
      fcol[t] = Ts[t][p];
    }
    __syncthreads();
    for (int e = t; e < kSw * kSw; e += blockDim.x) {
      int i = e / kSw, j = e % kSw;
      if (i == p) Ts[i][j] = prow[j];
      else if (j == p) Ts[i][j] = cneg(cmul(fcol[i], d));
      else Ts[i][j] = csub(Ts[i][j], cmul(fcol[i], prow[j]));
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_sweep_panel(const double2* __restrict__ M, int64_t ldm, int64_t R,
                                                     int64_t Cc, int64_t j0, int jn, double2* __restrict__ Pc,
                                                     double2* __restrict__ U, int64_t ldu, int* status) {
  __shared__ double2 Ts[kSw][kSw + 1];
  __shared__ double2 Ms[kSw][kSw + 1];
  __shared__ int perm[kSw], pinv[kSw];
  const int t = threadIdx.x;
  for (int e = t; e < kSw * kSw; e += blockDim.x) {
    int i = e / kSw, j = e % kSw;
    Ts[i][j] = (i < jn && j < jn) ? M[(j0 + i) * ldm + j0 + j] : cmk(i == j ? 1.0 : 0.0, 0.0);
  }
  if (t < kSw) perm[t] = t;
  __syncthreads();
  invert_block(Ts, perm, jn, status);
  // the pivoted sweep leaves inv(P M_JJ) = inv(M_JJ) P^T: inv(M_JJ)[r][c] = Ts[r][pinv[c]]
  if (t < kSw) pinv[perm[t]] = t;
  __syncthreads();
  // U for columns [c0, c0+64), in two 32-wide chunks
  const int64_t c0 = (int64_t)blockIdx.x * 64;
  for (int sub = 0; sub < 2; sub++) {
    const int64_t cb = c0 + sub * kSw;
    if (cb >= Cc) break;
    for (int e = t; e < kSw * kSw; e += blockDim.x) {
      int q = e / kSw, c = e % kSw;
      int64_t gc = cb + c;
      Ms[q][c] = (q < jn && gc < Cc) ? M[(j0 + q) * ldm + gc] : cmk(0.0, 0.0);
    }
    __syncthreads();
    for (int e = t; e < kSw * kSw; e += blockDim.x) {
      int r = e / kSw, c = e % kSw;
      int64_t gc = cb + c;
      if (gc >= Cc) continue;
      double2 v = cmk(0.0, 0.0);
      if (r < jn) {
        if (gc >= j0 && gc < j0 + jn) {
          v = Ts[r][pinv[gc - j0]];
        } else {
          for (int q = 0; q < jn; q++) v = cadd(v, cmul(Ts[r][pinv[q]], Ms[q][c]));
        }
      }
      U[r * ldu + gc] = v;
    }
    __syncthreads();
  }
  // Pc for rows [r0, r0+64)
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  if (r0 < R) {
    for (int e = t; e < 64 * kSw; e += blockDim.x) {
      int r = e / kSw, q = e % kSw;
      int64_t gr = r0 + r;
      if (gr >= R) continue;
      double2 v;
      if (gr >= j0 && gr < j0 + jn) v = cmk((gr - j0 == q) ? -1.0 : 0.0, 0.0);
      else v = (q < jn) ? M[gr * ldm + j0 + q] : cmk(0.0, 0.0);
      Pc[gr * kSw + q] = v;
    }
  }
}

void launch_sweep_panel(const double2* M, int64_t ldm, int64_t R, int64_t Cc, int64_t j0, int jn, double2* Pc,
                        double2* U, int64_t ldu, int* status, cudaStream_t s) {
  int64_t nblk = ((R > Cc ? R : Cc) + 63) / 64;
  k_sweep_panel<<<(unsigned)nblk, 256, 0, s>>>(M, ldm, R, Cc, j0, jn, Pc, U, ldu, status);
}

void launch_sweep_update(double2* M, int64_t ldm, int64_t R, int64_t Cc, int64_t j0, int jn, const double2* Pc,
                         const double2* U, int64_t ldu, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_zgemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    attr = true;
  }
  ZOp A{Pc, kSw, 0}, B{U, ldu, 0};
  dim3 grid((unsigned)((Cc + kBN - 1) / kBN), (unsigned)((R + kBM - 1) / kBM));
  k_zgemm<true><<<grid, 128, kGemmSmem, s>>>(R, Cc, kSw, cmk(-1.0, 0.0), A, B, cmk(1.0, 0.0), M, ldm, j0, jn,
                                             ZAdd{nullptr, 0, 0, 0});
}

const char* sweep_update_kernel_name() { return "k_zgemm<true> (sweep rank-32 update, FP64 DMMA)"; }

int sweep_block_width() { return kSw; }

// ---------------------------------------------------------------------------
// Partial pivoting over the whole remaining column (the row choice of LAPACK
// zgetrf, which MATLAB's inv uses at cal_smatrix_RGF.m:265).
//
// Before sweep step J = [j0, j0+jn), k_panel_gepp factors the panel
// W(j0:N, J) by LU with partial pivoting in a scratch copy (the largest
// |re| + |im| of the column, the first row on ties: LAPACK's izamax) and
// records the rows it chose, LAPACK style: swaps[j0+q] = row exchanged with
// row j0+q at step q.  k_laswp applies these exchanges to every column of W,
// so that the step's pivot block holds the chosen rows and the in-block
// pivoting of k_sweep_panel then takes them in the same order.  The rows of
// the unswept part (rows >= j0) of a partially swept matrix can be exchanged
// freely: sweeping commutes with it.  After the last step W's first N
// columns hold inv(P M) = inv(M) P^T (P = all exchanges of the slice), and
// k_perm_src + k_colperm undo that by exchanging the columns in reverse
// order.  The Schur complement the panel starts from is the trailing matrix
// of a right-looking LU, so the choices are those of unblocked LU with
// partial pivoting up to rounding.
// ---------------------------------------------------------------------------
constexpr int kGeppThreads = 512;
constexpr int kGeppSharedRows = 400;  // panels of up to 400 rows in shared memory (200 KB)

__device__ __forceinline__ void argmax_merge(double& m, int& i, double om, int oi) {
  if (om > m || (om == m && oi >= 0 && (i < 0 || oi < i))) {
    m = om;
    i = oi;
  }
}

// The panel lives in shared memory when its n x 32 entries fit (n <= 400),
// in the scratch copy (L2-resident) otherwise.
template <bool kShared>
__global__ void __launch_bounds__(kGeppThreads) k_panel_gepp(const double2* __restrict__ M, int64_t ldm,
                                                             int64_t N, int64_t j0, int jn, double2* __restrict__ Pg,
                                                             int* __restrict__ swaps, int* status) {
  extern __shared__ double2 Ps[];
  __shared__ double wmag[kGeppThreads / 32];
  __shared__ int widx[kGeppThreads / 32];
  __shared__ double2 prow[kSw];
  __shared__ int piv_s;
  double2* P = kShared ? Ps : Pg;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5;
  const int n = (int)(N - j0);
  for (int64_t e = t; e < (int64_t)n * kSw; e += blockDim.x) {
    const int i = (int)(e / kSw), q = (int)(e % kSw);
    P[e] = (q < jn) ? M[(j0 + i) * ldm + j0 + q] : cmk(0.0, 0.0);
  }
  __syncthreads();
  for (int q = 0; q < jn; q++) {
    double best = -1.0;
    int bi = -1;
    for (int i = q + t; i < n; i += blockDim.x) {  // rows in increasing order: first index kept on ties
      const double2 v = P[(int64_t)i * kSw + q];
      double m = fabs(v.x) + fabs(v.y);
      if (m != m) m = INFINITY;  // a NaN entry wins, so that it is flagged below
      if (m > best) {
        best = m;
        bi = i;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, off), __shfl_down_sync(0xffffffffu, bi, off));
    if (lane == 0) {
      wmag[warp] = best;
      widx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      best = lane < nwarps ? wmag[lane] : -1.0;
      bi = lane < nwarps ? widx[lane] : -1;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        argmax_merge(best, bi, __shfl_down_sync(0xffffffffu, best, off), __shfl_down_sync(0xffffffffu, bi, off));
      if (lane == 0) {
        const int r = bi < 0 ? q : bi;
        piv_s = r;
        swaps[j0 + q] = (int)(j0 + r);
        if (!(best > 0.0) || !isfinite(best)) atomicOr(status, kStatusSingular);
        // the pivot row (after the exchange) for every thread
      }
    }
    __syncthreads();
    const int r = piv_s;
    if (t < kSw) {
      const double2 a = P[(int64_t)q * kSw + t], b = P[(int64_t)r * kSw + t];
      prow[t] = b;
      if (r != q) {
        P[(int64_t)q * kSw + t] = b;
        P[(int64_t)r * kSw + t] = a;
      }
    }
    __syncthreads();
    const double2 d = cinv(prow[q]);
    for (int i = q + 1 + t; i < n; i += blockDim.x) {
      double2* __restrict__ row = P + (int64_t)i * kSw;
      const double2 l = cmul(row[q], d);
      row[q] = l;
#pragma unroll 8
      for (int c = q + 1; c < jn; c++) row[c] = csub(row[c], cmul(l, prow[c]));
    }
    __syncthreads();
  }
}

// rows j0+q <-> swaps[j0+q], q = 0..jn-1 in order, over columns [0, Cc)
__global__ void k_laswp(double2* M, int64_t ldm, int64_t Cc, int64_t j0, int jn, const int* __restrict__ swaps) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= Cc) return;
  for (int q = 0; q < jn; q++) {
    const int64_t a = j0 + q, r = swaps[a];
    if (r != a) {
      const double2 x = M[a * ldm + c];
      M[a * ldm + c] = M[r * ldm + c];
      M[r * ldm + c] = x;
    }
  }
}

// src[c] = the column of the swept matrix that column c of inv(M) is:
// the column exchanges (q, swaps[q]) applied for q = N-1 down to 0.
__global__ void k_perm_src(const int* __restrict__ swaps, int N, int* __restrict__ src) {
  extern __shared__ int ps[];
  int* sw = ps;
  int* sc = ps + N;
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    sw[c] = swaps[c];
    sc[c] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = N - 1; q >= 0; q--) {
      const int s = sw[q];
      if (s != q) {
        const int x = sc[q];
        sc[q] = sc[s];
        sc[s] = x;
      }
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < N; c += blockDim.x) src[c] = sc[c];
}

// W(i, c) <- W(i, src[c]) for rows [0, R), columns [0, N); each CTA stages
// its row in its own scratch row rowtmp + blockIdx.x * N
__global__ void k_colperm(double2* M, int64_t ldm, int64_t R, int64_t N, const int* __restrict__ src,
                          double2* __restrict__ rowtmp) {
  double2* tmp = rowtmp + (int64_t)blockIdx.x * N;
  for (int64_t i = blockIdx.x; i < R; i += gridDim.x) {
    for (int64_t c = threadIdx.x; c < N; c += blockDim.x) tmp[c] = M[i * ldm + c];
    __syncthreads();
    for (int64_t c = threadIdx.x; c < N; c += blockDim.x) M[i * ldm + c] = tmp[src[c]];
    __syncthreads();
  }
}

constexpr int kColpermCtas = 64;

size_t gepp_scratch_bytes(int64_t N) {
  // panel N x kSw, rowtmp kColpermCtas x N (complex); swaps and src (N ints each)
  return sizeof(double2) * (size_t)N * (kSw + kColpermCtas) + sizeof(int) * 2 * (size_t)N + 256;
}

void launch_gepp_step(double2* M, int64_t ldm, int64_t N, int64_t Cc, int64_t j0, int jn, void* scratch,
                      int* status, cudaStream_t s) {
  double2* P = reinterpret_cast<double2*>(scratch);
  int* swaps = reinterpret_cast<int*>(P + (size_t)N * (kSw + kColpermCtas));
  const int64_t n = N - j0;
  const size_t sm = sizeof(double2) * (size_t)n * kSw;
  if (n <= kGeppSharedRows) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_panel_gepp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(double2) * kGeppSharedRows * kSw));
      attr = true;
    }
    k_panel_gepp<true><<<1, kGeppThreads, sm, s>>>(M, ldm, N, j0, jn, P, swaps, status);
  } else {
    k_panel_gepp<false><<<1, kGeppThreads, 0, s>>>(M, ldm, N, j0, jn, P, swaps, status);
  }
  k_laswp<<<(unsigned)((Cc + 255) / 256), 256, 0, s>>>(M, ldm, Cc, j0, jn, swaps);
}

cudaError_t launch_gepp_unpermute(double2* M, int64_t ldm, int64_t R, int64_t N, void* scratch, cudaStream_t s) {
  double2* P = reinterpret_cast<double2*>(scratch);
  double2* rowtmp = P + (size_t)N * kSw;
  int* swaps = reinterpret_cast<int*>(P + (size_t)N * (kSw + kColpermCtas));
  int* src = swaps + N;
  const size_t sm = sizeof(int) * 2 * (size_t)N;
  if (sm > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_perm_src, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
  }
  k_perm_src<<<1, 256, sm, s>>>(swaps, (int)N, src);
  const int64_t ctas = R < kColpermCtas ? R : kColpermCtas;
  k_colperm<<<(unsigned)ctas, 256, 0, s>>>(M, ldm, R, N, src, rowtmp);
  return cudaGetLastError();
}

// max_i |W(i, pc1 + 1) - v(i)|, i < N, into the bits of probe_max (a NaN
// residual is recorded as +inf)
__global__ void k_probe_check(const double2* M, int64_t ldm, int64_t N, int64_t pc1,
                              unsigned long long* probe_max) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double r = 0.0;
  if (i < N) {
    const double2 d = csub(M[i * ldm + pc1 + 1], probe_v(i));
    r = sqrt(cabs2(d));
    if (r != r) r = INFINITY;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
  if ((threadIdx.x & 31) == 0 && r > 0.0) atomicMax(probe_max, (unsigned long long)__double_as_longlong(r));
}

void launch_probe_check(const double2* M, int64_t ldm, int64_t N, int64_t pc1, unsigned long long* probe_max,
                        cudaStream_t s) {
  k_probe_check<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(M, ldm, N, pc1, probe_max);
}

// ---------------------------------------------------------------------------
// Slice assembly: rows [0, N) x cols [0, N) of the augmented matrix become
//   A0 - k0dx^2 diag(eps) - G_src (- G_extra)
// (cal_smatrix_RGF.m:264-265; the attach step uses G_extra = G0 of the far
// lead, since (I - G0 G)^{-1} G0 = (G0^{-1} - G)^{-1} with G0^{-1} = A_lead - G0).
// Rows [N, Rz) x cols [0, N) are negated (-Z).  eps == nullptr means the
// uniform permittivity eps_u.
// ---------------------------------------------------------------------------
__global__ void k_assemble(double2* M, int64_t ldm, int64_t N, int64_t Rz, const double2* Gsrc,
                           int64_t ldg, const double2* Gextra, int64_t lde, const int* st_col,
                           const double2* st_val, double2 k2, const double2* eps, double2 eps_u) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t i = blockIdx.y;
  for (; i < Rz; i += gridDim.y) {
    if (j >= N) return;
    if (i >= N) {
      M[i * ldm + j] = cneg(M[i * ldm + j]);
      continue;
    }
    double2 v = cneg(Gsrc[i * ldg + j]);
    if (Gextra) v = csub(v, Gextra[i * lde + j]);
#pragma unroll
    for (int q = 0; q < kMaxStencil; q++)
      if (st_col[i * kMaxStencil + q] == j) v = cadd(v, st_val[i * kMaxStencil + q]);
    if (i == j) v = csub(v, cmul(k2, eps ? eps[i] : eps_u));
    M[i * ldm + j] = v;
  }
}

void launch_assemble(double2* M, int64_t ldm, int64_t N, int64_t Rz, const double2* Gsrc, int64_t ldg,
                     const double2* Gextra, int64_t lde, const int* st_col, const double2* st_val,
                     double2 k2, const double2* eps, double2 eps_u, cudaStream_t s) {
  dim3 grid((unsigned)((N + 127) / 128), (unsigned)(Rz < 8192 ? Rz : 8192));
  k_assemble<<<grid, 128, 0, s>>>(M, ldm, N, Rz, Gsrc, ldg, Gextra, lde, st_col, st_val, k2, eps, eps_u);
}

// ---------------------------------------------------------------------------
// Carrier blocks.  With p = prop index of a requested channel, lam = exp(i kx)
// and mu = sqrt_mu (cal_smatrix_RGF.m:191-203):
//   init  : X0 = G0_s B_s = phi(:,p) lam_p mu_p,   -Z0 = -(C_s G0_s) = -mu_p lam_p phi(:,p)^H,
//           Y0 = C_s G0_s B_s = mu lam mu on coinciding channels   (phi is unitary)
//   attach: B_e = phi(:,p) mu_p (extra columns),   -C_e = -mu_p phi(:,p)^H (extra rows)
// ---------------------------------------------------------------------------
__global__ void k_fill_init(double2* M, int64_t ldm, int64_t N, const double2* phi, int64_t ldp,
                            const int* prop, const double2* lam, const double2* mu, const int* in_s,
                            int n_in, const int* out_s, int n_out) {
  int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t nx = N * n_in, nz = (int64_t)n_out * N, ny = (int64_t)n_out * n_in;
  if (idx < nx) {
    int64_t m = idx / n_in;
    int i = (int)(idx % n_in);
    int p = prop[in_s[i]];
    M[m * ldm + N + i] = cmul(phi[m * ldp + p], cmul(lam[p], mu[p]));
  } else if (idx < nx + nz) {
    int64_t e = idx - nx;
    int o = (int)(e / N);
    int64_t m = e % N;
    int p = prop[out_s[o]];
    M[(N + o) * ldm + m] = cneg(cmul(cmul(mu[p], lam[p]), cconj(phi[m * ldp + p])));
  } else if (idx < nx + nz + ny) {
    int64_t e = idx - nx - nz;
    int o = (int)(e / n_in), i = (int)(e % n_in);
    int po = prop[out_s[o]], pi = prop[in_s[i]];
    M[(N + o) * ldm + N + i] = (po == pi) ? cmul(cmul(mu[po], lam[po]), mu[pi]) : cmk(0.0, 0.0);
  }
}

void launch_fill_init(double2* M, int64_t ldm, int64_t N, const double2* phi, int64_t ldp, const int* prop,
                      const double2* lam, const double2* mu, const int* in_s, int n_in, const int* out_s,
                      int n_out, cudaStream_t s) {
  int64_t tot = N * n_in + (int64_t)n_out * N + (int64_t)n_out * n_in;
  if (tot == 0) return;
  k_fill_init<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(M, ldm, N, phi, ldp, prop, lam, mu, in_s, n_in,
                                                            out_s, n_out);
}

// attach-step extra rows/columns; rows [N, N+no_s) and columns [N, N+ni_s)
// hold the carried Z/X, the new ones follow them.
__global__ void k_fill_attach(double2* M, int64_t ldm, int64_t N, int ni_s, int no_s, const double2* phi,
                              int64_t ldp, const int* prop, const double2* mu, const int* in_e, int ni_e,
                              const int* out_e, int no_e) {
  int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t Ct = N + ni_s + ni_e;
  int64_t nb = N * ni_e;                        // B_e block
  int64_t nzr = (int64_t)no_s * ni_e;           // zeros: Z rows x B_e cols
  int64_t nc = (int64_t)no_e * Ct;              // whole C_e rows
  if (idx < nb) {
    int64_t m = idx / ni_e;
    int i = (int)(idx % ni_e);
    int p = prop[in_e[i]];
    M[m * ldm + N + ni_s + i] = cmul(phi[m * ldp + p], mu[p]);
  } else if (idx < nb + nzr) {
    int64_t e = idx - nb;
    int64_t o = e / ni_e, i = e % ni_e;
    M[(N + o) * ldm + N + ni_s + i] = cmk(0.0, 0.0);
  } else if (idx < nb + nzr + nc) {
    int64_t e = idx - nb - nzr;
    int o = (int)(e / Ct);
    int64_t c = e % Ct;
    double2 v = cmk(0.0, 0.0);
    if (c < N) {
      int p = prop[out_e[o]];
      v = cneg(cmul(mu[p], cconj(phi[c * ldp + p])));
    }
    M[(N + no_s + o) * ldm + c] = v;
  }
}

void launch_fill_attach(double2* M, int64_t ldm, int64_t N, int ni_s, int no_s, const double2* phi,
                        int64_t ldp, const int* prop, const double2* mu, const int* in_e, int ni_e,
                        const int* out_e, int no_e, cudaStream_t s) {
  int64_t tot = N * ni_e + (int64_t)no_s * ni_e + (int64_t)no_e * (N + ni_s + ni_e);
  if (tot == 0) return;
  k_fill_attach<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(M, ldm, N, ni_s, no_s, phi, ldp, prop, mu,
                                                              in_e, ni_e, out_e, no_e);
}

// ---------------------------------------------------------------------------
// Fisher-Lee extraction (cal_smatrix_RGF.m:279, 286-289):
//   S(o, i) = -2i * W[N + row_of[o], N + col_of[i]] - delta(o, i)
// written column-major with leading dimension ldS; delta pairs come from the
// host (MATLAB intersect semantics).
// ---------------------------------------------------------------------------
__global__ void k_extract(const double2* M, int64_t ldm, int64_t N, const int* row_of, int no,
                          const int* col_of, int ni, double2* S, int64_t ldS) {
  int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)no * ni) return;
  int o = (int)(idx % no), i = (int)(idx / no);
  double2 w = M[(N + row_of[o]) * ldm + N + col_of[i]];
  S[o + (int64_t)i * ldS] = cmk(2.0 * w.y, -2.0 * w.x);
}

__global__ void k_delta(double2* S, int64_t ldS, const int* pairs, int npairs) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  int o = pairs[2 * k], i = pairs[2 * k + 1];
  S[o + (int64_t)i * ldS].x -= 1.0;
}

void launch_extract(const double2* M, int64_t ldm, int64_t N, const int* row_of, int no, const int* col_of,
                    int ni, double2* S, int64_t ldS, const int* pairs, int npairs, cudaStream_t s) {
  int64_t tot = (int64_t)no * ni;
  if (tot > 0) k_extract<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(M, ldm, N, row_of, no, col_of, ni, S, ldS);
  if (npairs > 0) k_delta<<<(npairs + 255) / 256, 256, 0, s>>>(S, ldS, pairs, npairs);
}

// ---------------------------------------------------------------------------
// probe columns of the first slice: p1 = v, p2 = M_1 v (top-left block of the
// assembled matrix times v), rows [N, R) zero.  One warp per row.
// ---------------------------------------------------------------------------
__global__ void k_probe_init(double2* M, int64_t ldm, int64_t N, int64_t R, int64_t pc1) {
  const int64_t i = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= R) return;
  double2 acc = cmk(0.0, 0.0);
  if (i < N)
    for (int64_t j = lane; j < N; j += 32) acc = cadd(acc, cmul(M[i * ldm + j], probe_v(j)));
  for (int off = 16; off > 0; off >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
  }
  if (lane == 0) {
    M[i * ldm + pc1] = (i < N) ? probe_v(i) : cmk(0.0, 0.0);
    M[i * ldm + pc1 + 1] = (i < N) ? acc : cmk(0.0, 0.0);
  }
}

void launch_probe_init(double2* M, int64_t ldm, int64_t N, int64_t R, int64_t pc1, cudaStream_t s) {
  k_probe_init<<<(unsigned)((R + 7) / 8), 256, 0, s>>>(M, ldm, N, R, pc1);
}

// ---------------------------------------------------------------------------
// misc
// ---------------------------------------------------------------------------
__global__ void k_check_finite(const double2* x, int64_t n, int* status) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool bad = false;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 v = x[i];
    if (!isfinite(v.x) || !isfinite(v.y)) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatusNonfinite);
}

void launch_check_finite(const double2* x, int64_t n, int* status, cudaStream_t s) {
  if (n <= 0) return;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  k_check_finite<<<(unsigned)blocks, 256, 0, s>>>(x, n, status);
}

// dst[r*ldd + c] = src[r*lds + c] * diag[c]  (phi * diag(exp(1i*kx)) for G0)
__global__ void k_scale_cols(const double2* src, int64_t lds, const double2* diag, double2* dst, int64_t ldd,
                             int64_t rows, int64_t cols) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t r = blockIdx.y; r < rows; r += gridDim.y)
    if (c < cols) dst[r * ldd + c] = cmul(src[r * lds + c], diag[c]);
}

void launch_scale_cols(const double2* src, int64_t lds, const double2* diag, double2* dst, int64_t ldd,
                       int64_t rows, int64_t cols, cudaStream_t s) {
  dim3 grid((unsigned)((cols + 127) / 128), (unsigned)(rows < 8192 ? rows : 8192));
  k_scale_cols<<<grid, 128, 0, s>>>(src, lds, diag, dst, ldd, rows, cols);
}

// ---------------------------------------------------------------------------
// permittivity gradient
// ---------------------------------------------------------------------------
// g[m] = coef * sum_a Phi[a][m] sum_b D[a][b] Psi[m][b]  (Phi: n_out x N, Psi:
// N x n_in, D: n_out x n_in, all row-major), for small n_out * n_in (D staged
// in shared memory)
__global__ void k_grad_fused(const double2* Phi, const double2* Psi, const double2* D, int64_t N, int n_out,
                             int n_in, double2 coef, double2* g) {
  extern __shared__ double2 Ds[];
  for (int e = threadIdx.x; e < n_out * n_in; e += blockDim.x) Ds[e] = D[e];
  __syncthreads();
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= N) return;
  double2 acc = cmk(0.0, 0.0);
  for (int a = 0; a < n_out; a++) {
    double2 e = cmk(0.0, 0.0);
    for (int b = 0; b < n_in; b++) e = cadd(e, cmul(Ds[a * n_in + b], Psi[m * n_in + b]));
    acc = cadd(acc, cmul(Phi[a * N + m], e));
  }
  g[m] = cmul(coef, acc);
}

void launch_grad_fused(const double2* Phi, const double2* Psi, const double2* D, int64_t N, int n_out, int n_in,
                       double2 coef, double2* g, cudaStream_t s) {
  k_grad_fused<<<(unsigned)((N + 127) / 128), 128, sizeof(double2) * n_out * n_in, s>>>(Phi, Psi, D, N, n_out,
                                                                                        n_in, coef, g);
}

// One slice of the backward recursions and the gradient contraction in one
// launch, for few channels (n_in, n_out <= kGradFusedMax):
//   Psi_out = g_j Psi_in + [X_j, 0]      (N x n_in)
//   Phi_out = Phi_in g_j + [Z_j; 0]      (n_out x N)
//   g[m]    = coef sum_a Phi_out[a][m] sum_b D[a][b] Psi_out[m][b]
// with g_j = W(0:N, 0:N), X_j = W(0:N, N:N+ni_s), Z_j = W(N:N+no_s, 0:N)
// (W row-major, leading dimension ld).  CTA c owns sites [16c, 16c+16):
// those rows of Psi_out and columns of Phi_out, accumulated over K in chunks
// of up to 128 staged in (dynamic) shared memory, then their contraction.
constexpr int kGradFusedMax = 32;
constexpr int kGTM = 16, kGKC = 128;

__host__ __device__ inline size_t grad_step_smem(int n_in, int n_out) {
  // sPsi[KC][n_in], sPhi[n_out][KC], sWr[16][KC+1], sWc[KC][17], oPsi[16][n_in], oPhi[n_out][16]
  return sizeof(double2) * ((size_t)kGKC * n_in + (size_t)n_out * kGKC + kGTM * (kGKC + 1) + kGKC * (kGTM + 1) +
                            kGTM * n_in + (size_t)n_out * kGTM);
}

__global__ void __launch_bounds__(256) k_grad_step(const double2* __restrict__ W, int64_t ld, int64_t N, int n_in,
                                                   int n_out, int ni_s, int no_s, const double2* __restrict__ Psi_in,
                                                   const double2* __restrict__ Phi_in, const double2* __restrict__ D,
                                                   double2 coef, double2* __restrict__ Psi_out,
                                                   double2* __restrict__ Phi_out, double2* __restrict__ g) {
  extern __shared__ double2 gsm[];
  double2* sPsi = gsm;                               // [KC][n_in]
  double2* sPhi = sPsi + kGKC * n_in;                // [n_out][KC]
  double2* sWr = sPhi + n_out * kGKC;                // [16][KC + 1]
  double2* sWc = sWr + kGTM * (kGKC + 1);            // [KC][17]
  double2* oPsi = sWc + kGKC * (kGTM + 1);           // [16][n_in]
  double2* oPhi = oPsi + kGTM * n_in;                // [n_out][16]
  const int t = threadIdx.x;
  const int64_t m0 = (int64_t)blockIdx.x * kGTM;
  const int tm = (int)min((int64_t)kGTM, N - m0);
  const int nP = kGTM * n_in, nF = n_out * kGTM;  // outputs of this CTA (<= 512 each)
  double2 accP[2] = {cmk(0, 0), cmk(0, 0)}, accF[2] = {cmk(0, 0), cmk(0, 0)};
  for (int64_t k0 = 0; k0 < N; k0 += kGKC) {
    const int kc = (int)min((int64_t)kGKC, N - k0);
    for (int e = t; e < kc * n_in; e += 256) sPsi[e] = Psi_in[k0 * n_in + e];  // rows k0.. of Psi_in, contiguous
    for (int e = t; e < n_out * kc; e += 256) {
      const int a = e / kc, k = e % kc;
      sPhi[a * kGKC + k] = Phi_in[(int64_t)a * N + k0 + k];
    }
    for (int e = t; e < kGTM * kc; e += 256) {
      const int r = e / kc, k = e % kc;
      sWr[r * (kGKC + 1) + k] = (r < tm) ? W[(m0 + r) * ld + k0 + k] : cmk(0, 0);
    }
    for (int e = t; e < kc * kGTM; e += 256) {
      const int k = e / kGTM, c = e % kGTM;
      sWc[k * (kGTM + 1) + c] = (c < tm) ? W[(k0 + k) * ld + m0 + c] : cmk(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int o = t + 256 * q;
      if (o < nP) {
        const int r = o / n_in, b = o % n_in;
        double2 sp = accP[q];
        for (int k = 0; k < kc; k++) sp = cadd(sp, cmul(sWr[r * (kGKC + 1) + k], sPsi[k * n_in + b]));
        accP[q] = sp;
      }
      if (o < nF) {
        const int a = o / kGTM, c = o % kGTM;
        double2 sf = accF[q];
        for (int k = 0; k < kc; k++) sf = cadd(sf, cmul(sPhi[a * kGKC + k], sWc[k * (kGTM + 1) + c]));
        accF[q] = sf;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int o = t + 256 * q;
    if (o < nP) {
      const int r = o / n_in, b = o % n_in;
      if (r < tm) {
        double2 v = accP[q];
        if (b < ni_s) v = cadd(v, W[(m0 + r) * ld + N + b]);
        Psi_out[(m0 + r) * n_in + b] = v;
        oPsi[r * n_in + b] = v;
      }
    }
    if (o < nF) {
      const int a = o / kGTM, c = o % kGTM;
      if (c < tm) {
        double2 v = accF[q];
        if (a < no_s) v = cadd(v, W[(N + a) * ld + m0 + c]);
        Phi_out[(int64_t)a * N + m0 + c] = v;
        oPhi[a * kGTM + c] = v;
      }
    }
  }
  if (!g) return;
  __syncthreads();
  // g[m] = coef sum_a Phi[a][m] (D Psi^T)[a][m]: warp w handles sites w, w + 8
  const int lane = t & 31, warp = t >> 5;
  for (int r = warp; r < tm; r += 8) {
    double2 acc = cmk(0, 0);
    for (int a = lane; a < n_out; a += 32) {
      double2 e = cmk(0, 0);
      for (int b = 0; b < n_in; b++) e = cadd(e, cmul(D[a * n_in + b], oPsi[r * n_in + b]));
      acc = cadd(acc, cmul(oPhi[a * kGTM + r], e));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
    }
    if (lane == 0) g[m0 + r] = cmul(coef, acc);
  }
}

bool grad_step_fits(int n_in, int n_out) { return n_in <= kGradFusedMax && n_out <= kGradFusedMax; }

void launch_grad_step(const double2* W, int64_t ld, int64_t N, int n_in, int n_out, int ni_s, int no_s,
                      const double2* Psi_in, const double2* Phi_in, const double2* D, double2 coef, double2* Psi_out,
                      double2* Phi_out, double2* g, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_grad_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)grad_step_smem(kGradFusedMax, kGradFusedMax));
    attr = true;
  }
  k_grad_step<<<(unsigned)((N + kGTM - 1) / kGTM), 256, grad_step_smem(n_in, n_out), s>>>(
      W, ld, N, n_in, n_out, ni_s, no_s, Psi_in, Phi_in, D, coef, Psi_out, Phi_out, g);
}

// g[m] = coef * sum_a Phi[a][m] Et[a][m]  (Phi, Et: n_out x N row-major)
__global__ void k_grad_slice(const double2* Phi, const double2* Et, int64_t N, int64_t n_out, double2 coef,
                             double2* g) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= N) return;
  double2 acc = cmk(0.0, 0.0);
  for (int64_t a = 0; a < n_out; a++) acc = cadd(acc, cmul(Phi[a * N + m], Et[a * N + m]));
  g[m] = cmul(coef, acc);
}

// dst[r*ldd + c] = scale * src[r*lds + c] (src == nullptr: zero), rows x cols
__global__ void k_block_copy(double2* dst, int64_t ldd, const double2* src, int64_t lds, int64_t rows, int64_t cols,
                             double scale) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= cols) return;
  for (int64_t r = blockIdx.y; r < rows; r += gridDim.y)
    dst[r * ldd + c] = src ? cscale(src[r * lds + c], scale) : cmk(0.0, 0.0);
}

void launch_block_copy(double2* dst, int64_t ldd, const double2* src, int64_t lds, int64_t rows, int64_t cols,
                       double scale, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  dim3 grid((unsigned)((cols + 127) / 128), (unsigned)(rows < 8192 ? rows : 8192));
  k_block_copy<<<grid, 128, 0, s>>>(dst, ldd, src, lds, rows, cols, scale);
}

__global__ void k_add_identity(double2* M, int64_t ldm, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) M[i * ldm + i].x += 1.0;
}

void launch_add_identity(double2* M, int64_t ldm, int64_t n, cudaStream_t s) {
  if (n > 0) k_add_identity<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(M, ldm, n);
}

// out[m + i*ld] = Psi[m][col_of[i]] (Psi: N x n_in row-major, augmented column order)
__global__ void k_store_field(const double2* Psi, const int* col_of, int64_t N, int n_in, double2* out, int64_t ld) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= N * n_in) return;
  const int i = (int)(e / N);
  const int64_t m = e % N;
  out[m + i * ld] = Psi[m * n_in + col_of[i]];
}

void launch_store_field(const double2* Psi, const int* col_of, int64_t N, int n_in, double2* out, int64_t ld,
                        cudaStream_t s) {
  const int64_t tot = N * n_in;
  if (tot > 0) k_store_field<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Psi, col_of, N, n_in, out, ld);
}

void launch_grad_slice(const double2* Phi, const double2* Et, int64_t N, int64_t n_out, double2 coef, double2* g,
                       cudaStream_t s) {
  k_grad_slice<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(Phi, Et, N, n_out, coef, g);
}

}  // namespace rgf

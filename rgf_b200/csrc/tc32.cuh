// Split-precision (3xTF32) real GEMM on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, FP32 accumulators in TMEM), operands staged in
// shared memory by TMA tensor copies (cp.async.bulk.tensor, 128-byte swizzle).
//
//   D[m][n] = sum_k A[m][k] * B[n][k]          (both operands K-major, fp32)
//
// Each operand comes as two arrays, hi = round-to-tf32(x) and lo = x - hi,
// and the product is formed as A_lo B_hi + A_hi B_lo + A_hi B_hi (the lo*lo
// term is dropped): about 21 bits of each product survive instead of the 11
// of one TF32 product (the "3xTF32" split of Ootomo & Yokota, "Recovering
// single precision accuracy from Tensor Cores while surpassing the FP32
// theoretical peak performance", IJHPCA 2022).
//
// Complex products are real GEMMs over a realified layout: a complex matrix P
// (rows x K) stored row-major interleaved (re, im) is the real K-major A
// operand [rows x 2K] as it lies in memory; the right factor Q (K x cols) is
// given as the real K-major B operand Bt[2 cols x 2K] with
//   Bt[2l][2j] = Re Q[j][l], Bt[2l][2j+1] = -Im Q[j][l],
//   Bt[2l+1][2j] = Im Q[j][l], Bt[2l+1][2j+1] = Re Q[j][l],
// so that D[m][2l] + i D[m][2l+1] = (P Q)[m][l] with the flop count of the
// complex product (8 real flops per complex multiply-add).
//
// One CTA computes one BM x BN tile of D over its share of K (K-split over
// blockIdx.z).  128 threads: warp 0 lane 0 issues the TMA copies, warp 1 owns
// the TMEM allocation and its lane 0 issues the MMAs, then all four warps read
// the accumulator back (warp w reads TMEM lanes 32w..32w+31 = tile rows) and
// run the epilogue.  Every wait is bounded and reports through g.err.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace rgf {
namespace tc32 {

constexpr int BM = 128;  // tile rows = TMEM lanes
constexpr int BK = 32;   // real K per pipeline stage: one 128-byte swizzle row of fp32
constexpr int kThreads = 128;

enum : int {
  kStore = 0,    // out[m*ldo + n] = D
  kPartial = 1,  // out[z*split_stride + m*ldo + n] = D  (K-split partial sums)
  kGJ = 2,       // Gauss-Jordan step: out = W' - D, W' = out with the pivot column block
                 // [gj_c0, gj_c0 + gj_nb) (complex columns) replaced by the identity's
};

enum : int { kErrTimeout = 4 };

struct GemmArgs {
  int M, Nr;               // rows of D, real columns of D
  int k_chunks;            // BK-chunks of K per CTA (one K-split)
  int k_total;             // > 0: ragged K-split instead, split z of Z taking the chunks
                           // [z k_total / Z, (z + 1) k_total / Z) (k_chunks unused)
  int a_z, b_z;            // batch coordinate (3rd tensor-map dimension) of A and B
  int mode;
  float* out;              // row-major fp32
  int64_t ldo;             // floats
  int64_t split_stride;    // floats between K-split partials (kPartial)
  int gj_c0, gj_nb;        // kGJ: pivot block (complex columns)
  int* err;                // error word (kErrTimeout)
  long long timeout;       // spin limit in SM clock cycles
  const int* az_dev;       // non-null: a_z is added to *az_dev (read after the grid before has finished)
};

// tile width BN: any multiple of 16 in [64, 256] (the M = 128 MMA shape);
// every stage buffer starts on a 1024-byte boundary (the swizzle atom)
template <int BN>
struct Cfg {
  static_assert(BN % 16 == 0 && BN >= 64 && BN <= 256, "BN");
  static constexpr uint32_t A_BYTES = BM * BK * 4;
  static constexpr uint32_t B_BYTES = BN * BK * 4;
  static constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES = (int)((224u * 1024u) / STAGE_BYTES);
  static_assert(STAGES >= 2 && B_BYTES % 1024 == 0, "stages");
  static constexpr uint32_t SMEM = STAGES * STAGE_BYTES + 1024;  // + alignment slack
  static constexpr uint32_t TMEM_COLS = BN <= 64 ? 64 : (BN <= 128 ? 128 : 256);  // a power of two
  // instruction descriptor: D f32 (bits 4-5 = 1), A/B tf32 (bits 7-9, 10-12 = 2),
  // both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
  static constexpr uint32_t IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, 128-byte swizzle: 8-row groups
// 1024 bytes apart (SBO), LBO unused (1), descriptor version 1 (bits 46-47),
// layout SWIZZLE_128B (2 at bits 61-63)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: false (and the error word set) after `timeout` cycles
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const GemmArgs& g) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > g.timeout) {
      atomicOr(g.err, kErrTimeout);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc32_gemm(const __grid_constant__ CUtensorMap ta_hi, const __grid_constant__ CUtensorMap ta_lo,
                const __grid_constant__ CUtensorMap tb_hi, const __grid_constant__ CUtensorMap tb_lo,
                GemmArgs g) {
  using C = Cfg<BN>;
  constexpr int S = C::STAGES;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[S];
  __shared__ __align__(8) uint64_t empty_bar[S];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;

  // programmatic dependent launch: the next kernel in the stream may start its
  // prologue now; it waits (griddepcontrol.wait) for this grid before reading
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t base = (su32(smem_raw) + 1023u) & ~1023u;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  int kc0 = blockIdx.z * g.k_chunks, nk = g.k_chunks;
  if (g.k_total > 0) {
    kc0 = (int)((int64_t)blockIdx.z * g.k_total / gridDim.z);
    nk = (int)((int64_t)(blockIdx.z + 1) * g.k_total / gridDim.z) - kc0;
  }
  int a_z = g.a_z;
  auto sA_hi = [&](int s) { return base + (uint32_t)s * C::STAGE_BYTES; };
  auto sA_lo = [&](int s) { return sA_hi(s) + C::A_BYTES; };
  auto sB_hi = [&](int s) { return sA_hi(s) + 2 * C::A_BYTES; };
  auto sB_lo = [&](int s) { return sA_hi(s) + 2 * C::A_BYTES + C::B_BYTES; };

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(su32(&full_bar[s]), 1);
      mbar_init(su32(&empty_bar[s]), 1);
    }
    mbar_init(su32(&done_bar), 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_sh)),
                 "r"(C::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;
  asm volatile("griddepcontrol.wait;" ::: "memory");  // the operands and `out` of the grid before
  if (g.az_dev) a_z += *g.az_dev;

  if (warp == 0 && lane == 0) {
    // producer: one stage = A_hi, A_lo (BM rows) and B_hi, B_lo (BN rows) of BK floats
    for (int kt = 0; kt < nk; kt++) {
      const int s = kt % S;
      if (kt >= S && !mbar_wait(su32(&empty_bar[s]), ((kt / S) - 1) & 1, g)) {
        abort_sh = 1;
        break;
      }
      const uint32_t fb = su32(&full_bar[s]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(C::STAGE_BYTES)
                   : "memory");
      const int kx = (kc0 + kt) * BK;
      tma_load_3d(sA_hi(s), &ta_hi, kx, m0, a_z, fb);
      tma_load_3d(sA_lo(s), &ta_lo, kx, m0, a_z, fb);
      tma_load_3d(sB_hi(s), &tb_hi, kx, n0, g.b_z, fb);
      tma_load_3d(sB_lo(s), &tb_lo, kx, n0, g.b_z, fb);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: 4 K-steps of 8 per stage, 3 products each
    for (int kt = 0; kt < nk; kt++) {
      const int s = kt % S;
      if (!mbar_wait(su32(&full_bar[s]), (kt / S) & 1, g)) {
        abort_sh = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint64_t ah = sw128_desc(sA_hi(s)), al = sw128_desc(sA_lo(s));
      const uint64_t bh = sw128_desc(sB_hi(s)), bl = sw128_desc(sB_lo(s));
#pragma unroll
      for (int kk = 0; kk < BK / 8; kk++) {
        const uint64_t o = (uint64_t)(kk * 32 / 16);  // 8 fp32 = 32 bytes along the swizzled row
        mma_tf32(tmem, al + o, bh + o, C::IDESC, (kt | kk) != 0);
        mma_tf32(tmem, ah + o, bl + o, C::IDESC, 1);
        mma_tf32(tmem, ah + o, bh + o, C::IDESC, 1);
      }
      mma_commit(su32(&empty_bar[s]));
    }
    mma_commit(su32(&done_bar));
  }
  __syncwarp();

  // epilogue: TMEM -> shared-memory tile (the drained pipeline buffers; thread
  // (warp, lane) moves tile row 32*warp + lane) -> global, one warp per row so
  // that every access is a contiguous 512-byte run
  const bool ok = mbar_wait(su32(&done_bar), 0, g);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  constexpr int TP = BN + 4;  // tile pitch in floats (row shift of 4 banks: conflict-free float4 stores)
  static_assert(BM * TP * 4 <= S * C::STAGE_BYTES, "epilogue tile");
  float* tile = reinterpret_cast<float*>(smem_raw + (base - su32(smem_raw)));
  const bool run = ok && nk > 0;
  if (run) {
    const int row = warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      float4* t4 = reinterpret_cast<float4*>(tile + row * TP + c);
#pragma unroll
      for (int j = 0; j < 4; j++) t4[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
  }
  __syncthreads();
  if (run) {
    float* obase = g.out + (g.mode == kPartial ? (int64_t)blockIdx.z * g.split_stride : 0);
    const int jlo = 2 * g.gj_c0, jhi = 2 * (g.gj_c0 + g.gj_nb);  // real columns of the pivot block
#pragma unroll 2
    for (int r = warp; r < BM; r += 4) {
      const int m = m0 + r;
      if (m >= g.M) break;
      float* orow = obase + (int64_t)m * g.ldo;
      for (int cc = lane * 4; cc < BN; cc += 128) {
        const int n = n0 + cc;
        if (n >= g.Nr) break;
        const float4 d4 = *reinterpret_cast<const float4*>(tile + r * TP + cc);
        const float d[4] = {d4.x, d4.y, d4.z, d4.w};
        const bool vec = (n + 4 <= g.Nr) && ((reinterpret_cast<uintptr_t>(orow + n) & 15) == 0);
        if (g.mode == kGJ) {
          const bool plain = n + 4 <= jlo || n >= jhi;  // no pivot-block column among the four
          if (vec && plain) {
            float4 w = *reinterpret_cast<const float4*>(orow + n);
            *reinterpret_cast<float4*>(orow + n) = make_float4(w.x - d[0], w.y - d[1], w.z - d[2], w.w - d[3]);
          } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int nn = n + j;
              if (nn >= g.Nr) break;
              const float w = (nn >= jlo && nn < jhi) ? (((nn & 1) == 0 && (nn >> 1) == m) ? 1.f : 0.f) : orow[nn];
              orow[nn] = w - d[j];
            }
          }
        } else if (vec) {
          *reinterpret_cast<float4*>(orow + n) = d4;
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (n + j < g.Nr) orow[n + j] = d[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS)
                 : "memory");
  }
}

#endif  // __CUDACC__

// ---------------------------------------------------------------------------
// host side: tensor maps (3D: K floats x rows x batch, box 32 x box_rows x 1,
// 128-byte swizzle, zero fill outside the tensor)
// ---------------------------------------------------------------------------
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// A K-major operand: element (row r, k) of batch z at base[z*batch_stride + r*ld + k]
// (floats).  ld and batch_stride must be multiples of 4 floats (16 bytes), base
// 16-byte aligned, kdim a multiple of BK.  Returns false if the map is refused.
inline bool make_map(CUtensorMap* map, const float* base, int64_t kdim, int64_t rows, int64_t batch, int64_t ld,
                     int64_t batch_stride, int box_rows,
                     CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_128B) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn || kdim % BK || ld % 4 || batch_stride % 4 || (reinterpret_cast<uintptr_t>(base) & 15) || rows < 1 ||
      batch < 1 || box_rows < 1 || box_rows > 256)
    return false;
  cuuint64_t dims[3] = {(cuuint64_t)kdim, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)(batch > 1 ? batch_stride : ld * rows) * 4};
  cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace tc32
}  // namespace rgf

// Persistent slice-recursion kernel (FP64 plain form).
//
// One cooperative launch runs the L slice sweeps of cal_smatrix_RGF.m:263-269
// (any of the five branches, projected on the requested channels; sweep.cu
// explains the augmented-matrix formulation).  The active augmented matrix W
// (R x C) is cut into TR x TC tiles of BM x BN; CTA (I, Cq) keeps its tile in
// FP64 DMMA accumulator registers for the whole recursion, so W goes back to
// memory only once per slice (for the slice assembly).
//
// Pivot step s (block J_s = [j0, j0+jn), jn <= 32) of the Gauss-Jordan sweep:
//     W <- W_mod + Pc * U,  Pc = [-W(i,J) (i not in J) ; +I (i in J)]
//                           U  = T_s * [W(J,c) (c not in J) | I (c in J)],  T_s = W(J,J)^{-1}
// where W_mod is W with the rows and columns of J zeroed.  Roles:
//  * tile CTA, 2 math warpgroups: wait for Pc(I) and U(Cq) of step s, stage
//    them in shared memory with TMA bulk copies (cp.async.bulk + mbarrier) and
//    update the whole register tile with mma.sync.m8n8k4.f64.  Then the warps
//    holding them publish pieces of later steps: the blocks (J_x, J_x) and
//    (J_x, J_{x-1}) of x = s+3 for the prep CTA, the pivot columns
//    W(I, J_{s+1}) of step s+1, and the rows W(J_{s+2}, Cq) for the panels.
//  * tile CTA, 1 panel warpgroup: its ceil(BN/TR)-column share of U_s(Cq)
//    as soon as T_s is out, then one step ahead the pivot rows of step s+1
//    in its share (the rows J_{s+1} published after step s-1, updated by
//    step s), both on the FP64 tensor cores.
//  * prep CTA (SM of its own): for step x, once U_{x-2} is out, the blocks
//        y0 = W^{(x-2)}(J_x,J_x),  y1 = W^{(x-2)}(J_x,J_{x-1})
//    (W^{(s)} = W after step s) from the blocks published after step x-3.
//  * T-server CTA (SM of its own, so its FP64 pipe is not shared with the
//    bulk update): its fourth warpgroup stages y0, y1 and
//    a3 = W^{(x-2)}(J_{x-1},J_x) (from the panels' pivot rows) in shared
//    memory; its 8 math warps form the next pivot block by the Schur update
//        W^{(s-1)}(J_s,J_s) = y0 - y1 (T_{s-1} a3)
//    and invert it by register-resident Gauss-Jordan with partial pivoting
//    (owner warps run ahead with per-row release counters, redux.sync pivot
//    search, implicit row interchanges, rows scaled once at the end); the
//    first pivot block of every slice comes straight from the slice assembly.
// setmaxnreg moves registers from the panel warpgroup (88) to the math
// warpgroups (208) so the 96x96 complex tile (144 registers/thread) fits.
// Exchange buffers are double-buffered by step parity; each has a publication
// flag (release/acquire, holds the step number) and a consumption counter the
// next writer of that parity waits on.  Every wait is bounded by a clock
// budget; on expiry the kernel sets kStatusTimeout, raises a global abort word
// that all other waits poll, and every role returns uniformly.
//
// A probe pair of columns (p1 = v, p2 = M_n v) rides along: after slice n, p2
// holds G_n M_n v, and max |G_n M_n v - v| bounds the error of every slice
// inverse a posteriori.
#include <math.h>

#include "persist.cuh"
#include "recip.cuh"

namespace rgf {

namespace {

constexpr int kPB = 32;  // pivot block width
constexpr int kPanelWarps = 4, kPanelThreads = kPanelWarps * 32;  // one warpgroup
constexpr int kBarMath = 1, kBarPanel = 2, kBarPub = 3, kBarDjj = 4, kBarSrv = 5, kBarPre0 = 6,
              kBarPre1 = 7, kBarSrv2 = 8, kBarGang = 9;  // named barriers
constexpr int kMaxTile = 96;
constexpr int kServerThreads = 256;  // the math warpgroups of the T-server CTA
constexpr unsigned kFull = 0xffffffffu;

template <int BM, int BN>
struct Cfg {
  static constexpr int WM = 2, WN = 4;  // math warp grid
  static constexpr int MathWarps = WM * WN, MathThreads = MathWarps * 32;
  static constexpr int Threads = MathThreads + kPanelThreads;
  static constexpr int MathRegs = 208, PanelRegs = 88;  // 256*208 + 128*88 = 384*168
};

// Named barriers in their non-.aligned form (per-thread arrival), preceded
// by a warp reconvergence, so that no barrier depends on the compiler having
// reconverged a warp after lane-divergent code.
__device__ __forceinline__ void bar_sync(int id, int n) {
  __syncwarp();
  asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
// CTA-uniform OR over the threads of a named barrier
__device__ __forceinline__ int bar_or(int id, int n, int pred) {
  int r;
  __syncwarp();
  asm volatile(
      "{ .reg .pred p, q; setp.ne.s32 p, %3, 0; barrier.red.or.pred q, %1, %2, p; selp.s32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"(id), "r"(n), "r"(pred)
      : "memory");
  return r;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ int ld_acquire_cta(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared.s32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(int* p, int v) {
  asm volatile("st.release.cta.shared.s32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}
// volatile keeps predicated products from being if-converted into
// unconditional ones; callers order the issue so that the two dependent
// DMMAs of each complex product are far apart
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// swizzled element positions of the staged operand tiles (conflict-free
// m8n8k4 fragment loads): A is [BM][32], B is [32][BN]
__device__ __forceinline__ int swzA(int r, int k) { return r * kPB + (k ^ ((r & 1) << 2)); }
template <int BN>
__device__ __forceinline__ int swzB(int k, int c) { return k * BN + (c ^ ((k & 3) << 1)); }

typedef double2 Blk[kPB][kPB + 1];  // padded 32x32 block in shared memory

struct Shared {
  union {
    struct {  // tile CTAs, math role: staged operands of the current step
      alignas(128) double2 A[kMaxTile * kPB];
      alignas(128) double2 B[kPB * kMaxTile];
    } op;
    struct {  // T-server CTA: next pivot block, T_{s-1}, scratch, per step
              // parity the blocks a3 and (J_s, J_s), (J_s, J_{s-1}) staged by
              // the prep warps, and a prep operand
      Blk a1, tprev, v;
      Blk a3[2];
      Blk y[2][2];
    } srv;
  };
  alignas(8) unsigned long long mbar;
  int math_abort;
  int panel_abort;
  Blk T;   // panel role: T_s
  Blk Mr;  // panel role: my columns of the pivot rows
  // T-server Gauss-Jordan: pivot q's multipliers are in srv.v[q][r]; per row r
  // its pivot index copy, release counter, and the reciprocal of the pivot
  // it became
  int gpiv[kPB][kPB];
  int gflag[kPB];
  double2 drow[kPB];
  int gj_fail;  // a Gauss-Jordan wait gave up
  int asig[2];  // T-server: step whose a3[parity] block is staged (prep -> server)
  int ysig[2];  // T-server: step whose y[parity] blocks are ready (prep -> server)
  int ycons;    // T-server: last step whose y blocks the server has read
  int perm[kPB], pinv[kPB];
};

__device__ __forceinline__ void trace_ev(const PersistParams& p, int s, int ev) {
  if (p.trace && s >= 0 && s < p.trace_steps)
    p.trace[((size_t)blockIdx.x * p.trace_steps + s) * kTraceEvents + ev] = gtimer();
}

__device__ __forceinline__ bool give_up(const PersistParams& p, long long t0) {
  if (*(volatile const int*)p.abort) return true;
  if (clock64() - t0 > p.timeout_cycles) {
    atomicOr(p.status, kStatusTimeout);
    atomicExch(p.abort, 1);
    return true;
  }
  return false;
}

// bounded wait on a flag word; false = gave up (timeout here or abort raised elsewhere)
__device__ bool wait_ge(const PersistParams& p, const int* flag, int target) {
  if (ld_acquire(flag) >= target) return true;
  const long long t0 = clock64();
  for (int spins = 1;; spins++) {
    if (spins > 64) __nanosleep(32);
    if (ld_acquire(flag) >= target) return true;
    if ((spins & 63) == 0 && give_up(p, t0)) return false;
  }
}

// the same on a shared-memory flag (other warps of this CTA)
__device__ bool wait_cta_ge(const PersistParams& p, const int* flag, int target) {
  if (ld_acquire_cta(flag) >= target) return true;
  const long long t0 = clock64();
  for (int spins = 1;; spins++) {
    if (spins > 64) __nanosleep(32);
    if (ld_acquire_cta(flag) >= target) return true;
    if ((spins & 63) == 0 && give_up(p, t0)) return false;
  }
}

// one warp waits until flags[0..count) >= target and, if extra != nullptr,
// *extra >= target; the flags are polled in parallel, one per lane.  Returns
// the same verdict in every lane.
__device__ bool warp_wait_all(const PersistParams& p, const int* flags, int count, const int* extra, int target) {
  const int lane = threadIdx.x & 31;
  const long long t0 = clock64();
  for (int spins = 0;; spins++) {
    bool mine = true;
    for (int r = lane; r < count; r += 32) mine = mine && (ld_acquire(flags + r) >= target);
    if (lane == 0 && extra) mine = mine && (ld_acquire(extra) >= target);
    if (__all_sync(kFull, mine)) return true;
    if (spins > 64) __nanosleep(32);
    if ((spins & 63) == 63) {
      const int bad = (lane == 0) ? (int)give_up(p, t0) : 0;
      if (__shfl_sync(kFull, bad, 0)) return false;
    }
  }
}

// Flag words.  A flag of a buffer with several writers (the server blocks)
// is kept per step parity: the same-parity value can only advance after the
// server consumed the previous one, so "flag >= s" means "published for s".
struct Sync {
  int *pc_flag, *pre_flag, *t_flag, *u_flag, *d_flag, *srv_flag, *d_used, *rowp_flag, *srv2_flag, *y_flag, *y_used;
  int *pc_cons, *pre_cons, *t_cons, *u_cons, *srv_cons, *pcp_cons;
  __device__ explicit Sync(const PersistParams& p) {
    pc_flag = p.flags;
    pre_flag = pc_flag + p.TR;  // [2][TC]: per parity (a slice start publishes two steps at once)
    t_flag = pre_flag + 2 * p.TC;
    u_flag = t_flag + 1;
    d_flag = u_flag + p.TR * p.TC;
    srv_flag = d_flag + 1;
    d_used = srv_flag + 2;
    rowp_flag = d_used + 1;  // [TC][TR]: rows of the step in panel I's share of tile column Cq
    srv2_flag = rowp_flag + p.TR * p.TC;  // [2]: block (J_s2, J_s1), possibly from another tile column
    y_flag = srv2_flag + 2;               // [2]: ybuf of a step parity written (prep CTA)
    y_used = y_flag + 2;                  // last step whose ybuf the T-server CTA has loaded
    pc_cons = p.cons;
    pre_cons = pc_cons + 2 * p.TR;
    t_cons = pre_cons + 2 * p.TC;
    u_cons = t_cons + 2;
    srv_cons = u_cons + 2 * p.TC;
    pcp_cons = srv_cons + 2;  // [2]: panels done reading the pivot columns of a step
  }
};

// ---------------------------------------------------------------------------
// tile CTA, math warpgroups
// ---------------------------------------------------------------------------
template <int BM, int BN>
struct MathTile {
  static constexpr int WR = BM / Cfg<BM, BN>::WM, WC = BN / Cfg<BM, BN>::WN;  // warp tile
  static constexpr int MI = WR / 8, NI = WC / 8;
  double acc[MI][NI][4];  // {re(c), re(c+1), im(c), im(c+1)}
  int lane, wr, wc;
  int r_base, c_base;
  __device__ int row(int mi) const { return r_base + mi * 8 + (lane >> 2); }
  __device__ int col(int ni, int h) const { return c_base + ni * 8 + (lane & 3) * 2 + h; }
};

template <int BM, int BN>
__device__ void math_role(const PersistParams& p, Shared& sh, const Sync& sy, int I, int Cq) {
  using Tile = MathTile<BM, BN>;
  constexpr int MI = Tile::MI, NI = Tile::NI;
  constexpr int kMathWarps = Cfg<BM, BN>::MathWarps, kMathThreads = Cfg<BM, BN>::MathThreads;
  Tile t;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  t.lane = tid & 31;
  t.wr = warp >> 2;
  t.wc = warp & 3;
  t.r_base = I * BM + t.wr * Tile::WR;
  t.c_base = Cq * BN + t.wc * Tile::WC;
  const int S = p.L * p.NB;
  const int tr0 = I * BM, tc0 = Cq * BN;  // tile origin

  // Publication sets.  After the update of step s the warps holding pieces
  // of later steps publish them: the pivot columns of s1 = s+1 (pc), the
  // rows J_{s1+1} (pre: the panels update them by step s1 into the pivot
  // rows of s1+1), at a slice start also the rows J_{s1} and the first pivot
  // block (djj), and, when s2 = s1+1 is in the same slice, the 32x32 blocks
  // (J_s2, J_s2) and (J_s2, J_s1) of W for the T-server (srv).  Membership depends only on
  // the warp's row / column range, so every warp evaluates it for every warp
  // of the CTA (barrier counts, flag-releasing lead).
  enum { kSetPc, kSetPre, kSetDjj, kSetSrv };
  auto in_set = [&](int kind, int w, int s1) {
    const int w1 = (s1 % p.NB) * kPB, w2 = w1 + kPB;
    const int rb = tr0 + (w >> 2) * Tile::WR, cb = tc0 + (w & 3) * Tile::WC;
    const bool r1 = (w1 + kPB > rb) && (w1 < rb + Tile::WR);
    const bool c1 = (w1 + kPB > cb) && (w1 < cb + Tile::WC);
    const bool r2 = (w2 + kPB > rb) && (w2 < rb + Tile::WR);
    const bool c2 = (w2 + kPB > cb) && (w2 < cb + Tile::WC);
    return kind == kSetPc ? c1 : kind == kSetPre ? r1 : kind == kSetDjj ? (r1 && c1) : (r2 && (c1 || c2));
  };
  auto pub_set = [&](int kind, int s1, int* lead) {
    int n = 0;
    *lead = -1;
    for (int w = kMathWarps - 1; w >= 0; w--)
      if (in_set(kind, w, s1)) {
        n++;
        *lead = w;
      }
    return n;
  };
  // does subtile row mi / column ni of this warp lie in the 32-wide window at w
  auto row_in = [&](int mi, int w) { return (unsigned)(t.r_base + mi * 8 - w) < (unsigned)kPB; };
  auto col_in = [&](int ni, int w) { return (unsigned)(t.c_base + ni * 8 - w) < (unsigned)kPB; };
  const int lr = t.lane >> 2, lc = (t.lane & 3) * 2;  // this thread's row / column within a subtile
  const int sw = (lr & 1) << 2;                       // swzA swizzle of this thread's rows
  auto load_tile = [&]() {
#pragma unroll
    for (int mi = 0; mi < MI; mi++)
#pragma unroll
      for (int ni = 0; ni < NI; ni++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = t.row(mi), j = t.col(ni, h);
          const double2 v = (i < p.R && j < p.C) ? __ldcg(p.M + (int64_t)i * p.ldm + j) : cmk(0.0, 0.0);
          t.acc[mi][ni][h] = v.x;
          t.acc[mi][ni][2 + h] = v.y;
        }
  };
  auto store_tile = [&]() {
#pragma unroll
    for (int mi = 0; mi < MI; mi++)
#pragma unroll
      for (int ni = 0; ni < NI; ni++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = t.row(mi), j = t.col(ni, h);
          if (i < p.R && j < p.C) __stcg(p.M + (int64_t)i * p.ldm + j, cmk(t.acc[mi][ni][h], t.acc[mi][ni][2 + h]));
        }
  };
  // Slice boundary on the register tile: probe check (p2 = G_n M_n v against
  // v), the snapshot of W after the slice when `snap` is given (layout of W,
  // probe columns excepted) and, when eps_next is given, the next slice
  // matrix in place: top-left A_{n+1} - G_n, -Z rows, X columns and the Y
  // block unchanged, probe pair p1 = v, p2 = A_{n+1} v - G_n v.  Each thread
  // works on its own accumulators only.  The probe pair is the column pair
  // (pc1, pc1 + 1), pc1 even, so one thread holds both as h = 0, 1.
  // Returns the largest probe residual this thread saw.
  auto boundary_regs = [&](const double2* eps_next, double2* snap) {
    double pmax = 0.0;
    // the probe pair of each row goes through a small local array, so that
    // its (long) arithmetic is instantiated once, not once per accumulator
    double2 pr[MI][2];
    unsigned has = 0;
#pragma unroll
    for (int mi = 0; mi < MI; mi++) {
      const int i = t.row(mi);
      if (i >= p.R) continue;
      const bool top = i < p.N;
      const double2 ke = (eps_next && top) ? cmul(p.k2, __ldg(eps_next + i)) : cmk(0.0, 0.0);
#pragma unroll
      for (int ni = 0; ni < NI; ni++) {
        const int j0c = t.col(ni, 0);  // even; j0c + 1 is the h = 1 column
        if (j0c >= p.C) continue;
        double* a = t.acc[mi][ni];
        if (j0c == p.pc1) {
          pr[mi][0] = cmk(a[0], a[2]);
          pr[mi][1] = cmk(a[1], a[3]);
          has |= 1u << mi;
          continue;
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int j = j0c + h;
          if (j >= p.C) continue;
          if (snap) __stcg(snap + (int64_t)i * p.ldm + j, cmk(a[h], a[2 + h]));
          if (!eps_next || j >= p.N) continue;  // X columns and the Y block are carried unchanged
          a[h] = -a[h];  // -G_n, or the -Z rows
          a[2 + h] = -a[2 + h];
          if (i == j) {
            a[h] -= ke.x;
            a[2 + h] -= ke.y;
          }
        }
      }
      // + A0 (stencil entries of row i), one entry at a time
      if (!eps_next || !top) continue;
#pragma unroll 1
      for (int q = 0; q < kMaxStencil; q++) {
        const int cq = __ldg(p.st_col + (int64_t)i * kMaxStencil + q);
        if (cq < 0) continue;
        const double2 v = __ldg(p.st_val + (int64_t)i * kMaxStencil + q);
#pragma unroll
        for (int ni = 0; ni < NI; ni++)
#pragma unroll
          for (int h = 0; h < 2; h++)
            if (cq == t.col(ni, h) && cq != p.pc1 && cq != p.pc1 + 1) {
              t.acc[mi][ni][h] += v.x;
              t.acc[mi][ni][2 + h] += v.y;
            }
      }
    }
    if (has == 0u) return pmax;
#pragma unroll 1
    for (int mi = 0; mi < MI; mi++) {
      if (!((has >> mi) & 1u)) continue;
      const int i = t.row(mi);
      if (i < p.N) {
        const double2 v = probe_v(i);
        const double2 d = csub(pr[mi][1], v);
        const double rr = sqrt(cabs2(d));
        pmax = (rr == rr) ? fmax(pmax, rr) : INFINITY;  // fmax would drop a NaN
        if (eps_next) {
          double2 Av = csub(cmk(0.0, 0.0), cmul(cmul(p.k2, __ldg(eps_next + i)), v));
          for (int q = 0; q < kMaxStencil; q++) {
            const int cq = __ldg(p.st_col + (int64_t)i * kMaxStencil + q);
            if (cq >= 0) Av = cadd(Av, cmul(__ldg(p.st_val + (int64_t)i * kMaxStencil + q), probe_v(cq)));
          }
          pr[mi][1] = csub(Av, pr[mi][0]);
          pr[mi][0] = v;
        }
      } else if (eps_next) {
        pr[mi][0] = pr[mi][1] = cmk(0.0, 0.0);
      }
    }
#pragma unroll
    for (int mi = 0; mi < MI; mi++)
#pragma unroll
      for (int ni = 0; ni < NI; ni++)
        if (((has >> mi) & 1u) && t.col(ni, 0) == p.pc1) {
          t.acc[mi][ni][0] = pr[mi][0].x;
          t.acc[mi][ni][2] = pr[mi][0].y;
          t.acc[mi][ni][1] = pr[mi][1].x;
          t.acc[mi][ni][3] = pr[mi][1].y;
        }
    return pmax;
  };
  // rank-32 update of the whole warp tile: first halves of every complex
  // product, then the dependent second halves
  auto mma_pass = [&]() {
#pragma unroll
    for (int kk = 0; kk < kPB / 4; kk++) {
      double2 b[NI];
#pragma unroll
      for (int ni = 0; ni < NI; ni++)
        b[ni] = sh.op.B[swzB<BN>(kk * 4 + (t.lane & 3), t.wc * Tile::WC + ni * 8 + lr)];
#pragma unroll
      for (int mi = 0; mi < MI; mi++) {
        const double ax = sh.op.A[swzA(t.wr * Tile::WR + mi * 8 + lr, kk * 4 + (t.lane & 3))].x;
#pragma unroll
        for (int ni = 0; ni < NI; ni++) {
          dmma(t.acc[mi][ni][0], t.acc[mi][ni][1], ax, b[ni].x);
          dmma(t.acc[mi][ni][2], t.acc[mi][ni][3], ax, b[ni].y);
        }
      }
#pragma unroll
      for (int mi = 0; mi < MI; mi++) {
        const double ay = sh.op.A[swzA(t.wr * Tile::WR + mi * 8 + lr, kk * 4 + (t.lane & 3))].y;
#pragma unroll
        for (int ni = 0; ni < NI; ni++) {
          dmma(t.acc[mi][ni][0], t.acc[mi][ni][1], -ay, b[ni].y);
          dmma(t.acc[mi][ni][2], t.acc[mi][ni][3], ay, b[ni].x);
        }
      }
    }
  };
  // 32x32 block (rows in window wr_, columns in window wc_) of W into a
  // row-major [32][32] buffer; rows / columns at or beyond `lim` are padded
  // with the identity (pad_id) or zeros
  auto store_block = [&](double2* dst, int wr_, int wc_, int lim_r, int lim_c, bool pad_id) {
#pragma unroll
    for (int mi = 0; mi < MI; mi++) {
      if (!row_in(mi, wr_)) continue;
      const int r = t.r_base + mi * 8 + lr - wr_;
#pragma unroll
      for (int ni = 0; ni < NI; ni++) {
        if (!col_in(ni, wc_)) continue;
        const int c0 = t.c_base + ni * 8 + lc - wc_;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c = c0 + h;
          const bool in = r < lim_r && c < lim_c;
          const double2 v = in ? cmk(t.acc[mi][ni][h], t.acc[mi][ni][2 + h])
                               : cmk((pad_id && r == c) ? 1.0 : 0.0, 0.0);
          __stcg(dst + r * kPB + c, v);
        }
      }
    }
  };
  // the first pivot block of a slice -> djjbuf for the T-server
  auto publish_djj = [&](int s1) {
    const int w0 = (s1 % p.NB) * kPB;
    const int jnn = min(kPB, p.N - w0);
    int ok = 1;
    if (t.lane == 0 && s1 >= p.NB) ok = wait_ge(p, sy.d_used, s1 - p.NB);  // previous slice's was loaded
    ok = __shfl_sync(kFull, ok, 0);
    if (ok) store_block(p.djjbuf, w0, w0, jnn, jnn, true);
    int lead;
    const int n = pub_set(kSetDjj, s1, &lead);
    const int all_ok = !bar_or(kBarDjj, n * 32, !ok);
    if (warp == lead && t.lane == 0 && all_ok) {
      st_release(sy.d_flag, s1);
    }
  };
  // the pivot columns (pcbuf) of step s1; the lead warp releases the flag
  // after every publishing warp wrote
  auto publish_pc = [&](int s1) {
    const int w0 = (s1 % p.NB) * kPB;
    const int jnn = min(kPB, p.N - w0);
    const int par = s1 & 1;
    int lead;
    const int n = pub_set(kSetPc, s1, &lead);
    if (warp == lead && t.lane == 0) trace_ev(p, s1 - 1, kTrGlobEnter);
    int ok = 1;
    if (t.lane == 0 && s1 >= 2) {  // the math warps and every panel are done with step s1-2's
      ok = wait_ge(p, sy.pc_cons + par * p.TR + I, p.TC * (s1 >> 1));
      ok = ok && wait_ge(p, sy.pcp_cons + par, (p.TR * p.TC + 1) * (s1 >> 1));  // panels + prep CTA
    }
    ok = __shfl_sync(kFull, ok, 0);
    if (ok) {
      // Pc = [-W(i, J) ; +I on the pivot rows], zero beyond the last pivot
      // column and below row R, stored in the swizzled [BM][32] layout
      double2* pcb = p.pcbuf + ((size_t)par * p.TR + I) * (BM * kPB) + (t.r_base - tr0 + lr) * kPB;
#pragma unroll
      for (int ni = 0; ni < NI; ni++) {
        if (!col_in(ni, w0)) continue;
        const int kc = t.c_base + ni * 8 - w0;  // multiple of 8: the swizzle acts on lc + h only
#pragma unroll
        for (int mi = 0; mi < MI; mi++) {
          const int i = t.r_base + mi * 8 + lr;
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int k = kc + lc + h;
            double2 wv;
            if (k >= jnn || i >= p.R) wv = cmk(0.0, 0.0);
            else if (i >= w0 && i < w0 + jnn) wv = cmk((i - w0 == k) ? 1.0 : 0.0, 0.0);
            else wv = cmk(-t.acc[mi][ni][h], -t.acc[mi][ni][2 + h]);
            __stcg(pcb + mi * 8 * kPB + kc + ((lc + h) ^ sw), wv);
          }
        }
      }
    }
    if (warp == lead && t.lane == 0) trace_ev(p, s1 - 1, kTrGlobStored);
    const int all_ok = !bar_or(kBarPub, n * 32, !ok);
    if (warp == lead && t.lane == 0 && all_ok) {  // an aborted publish never releases anything
      st_release(sy.pc_flag + I, s1);
      trace_ev(p, s1 - 1, kTrMathPublished);
    }
  };
  // rows J_x of the current W (prebuf[x & 1][Cq][k][c - tc0], zero beyond the
  // last pivot row) for the panels of tile column Cq
  auto publish_pre = [&](int x, int bar_id) {
    const int w0 = (x % p.NB) * kPB;
    const int jnn = min(kPB, p.N - w0);
    const int par = x & 1;
    int lead;
    const int n = pub_set(kSetPre, x, &lead);
    int ok = 1;
    if (t.lane == 0 && x >= 2) ok = wait_ge(p, sy.pre_cons + par * p.TC + Cq, p.TR * (x >> 1));
    ok = __shfl_sync(kFull, ok, 0);
    if (ok) {
      double2* rowb = p.prebuf + ((size_t)par * p.TC + Cq) * (kPB * BN) + (t.c_base - tc0 + lc);
#pragma unroll
      for (int mi = 0; mi < MI; mi++) {
        if (!row_in(mi, w0)) continue;
        const int kr = t.r_base + mi * 8 + lr - w0;
        const bool valid = kr < jnn;
        double2* q = rowb + kr * BN;
#pragma unroll
        for (int ni = 0; ni < NI; ni++)
#pragma unroll
          for (int h = 0; h < 2; h++)
            __stcg(q + ni * 8 + h, valid ? cmk(t.acc[mi][ni][h], t.acc[mi][ni][2 + h]) : cmk(0.0, 0.0));
      }
    }
    const int all_ok = !bar_or(bar_id, n * 32, !ok);
    if (warp == lead && t.lane == 0 && all_ok) st_release(sy.pre_flag + par * p.TC + Cq, x);
  };
  // blocks (J_s2, J_s2) (padded with the identity beyond the last pivot row)
  // and (J_s2, J_s1) (zero rows there) of the current W, s2 = s1+1, for the
  // T-server's prep warps, which update them by step s2-2 (unless s2 is the
  // second step of its slice) into the blocks of the Schur update of step s2
  auto publish_srv = [&](int s1, int bar_id) {
    const int s2 = s1 + 1;
    const int w1 = (s1 % p.NB) * kPB, w2 = w1 + kPB;
    const int jn2 = min(kPB, p.N - w2);
    const int par = s2 & 1;
    int lead;
    const int n = pub_set(kSetSrv, s1, &lead);
    if (warp == lead && t.lane == 0) trace_ev(p, s1 - 1, kTrSrvPubEnter);
    int ok = 1;
    if (t.lane == 0 && s2 >= 2) ok = wait_ge(p, sy.srv_cons + par, s2 >> 1);
    ok = __shfl_sync(kFull, ok, 0);
    if (ok) {
      store_block(p.srvbuf + (size_t)par * 2 * kPB * kPB, w2, w2, jn2, jn2, true);
      store_block(p.srvbuf + ((size_t)par * 2 + 1) * kPB * kPB, w2, w1, jn2, kPB, false);
    }
    if (warp == lead && t.lane == 0) trace_ev(p, s1 - 1, kTrSrvPubStored);
    const int all_ok = !bar_or(bar_id, n * 32, !ok);
    if (warp == lead && t.lane == 0 && all_ok) {
      if (w2 >= tc0 && w2 < tc0 + BN) st_release(sy.srv_flag + par, s2);
      if (w1 >= tc0 && w1 < tc0 + BN) st_release(sy.srv2_flag + par, s2);
      trace_ev(p, s1 - 1, kTrSrvPubDone);
    }
  };
  // every piece of later steps this warp holds after the update of step
  // s1 - 1: the server blocks of step s1 + 2, the pivot columns of s1, the
  // rows J_{s1+1}; at a slice start (kernel start or after the slice
  // assembly) also the server blocks of step s1 + 1, the rows J_{s1} and the
  // first pivot block
  auto publish = [&](int s1, bool slice_start) {
    const int k1 = s1 % p.NB;
    const bool next_in_slice = k1 + 1 < p.NB;  // step s1 + 1 is in the same slice
    if (slice_start && in_set(kSetDjj, warp, s1)) publish_djj(s1);
    if (slice_start && next_in_slice && in_set(kSetSrv, warp, s1)) publish_srv(s1, kBarSrv);
    if (k1 + 2 < p.NB && in_set(kSetSrv, warp, s1 + 1)) publish_srv(s1 + 1, kBarSrv2);
    if (in_set(kSetPc, warp, s1)) publish_pc(s1);
    if (slice_start && in_set(kSetPre, warp, s1)) publish_pre(s1, kBarPre0);
    if (next_in_slice && in_set(kSetPre, warp, s1 + 1)) publish_pre(s1 + 1, kBarPre1);
  };

  load_tile();
  bar_sync(kBarMath, kMathThreads);
  publish(0, true);

  double probe_max = 0.0;
  for (int s = 0; s < S; s++) {
    const int n = s / p.NB, k = s % p.NB;
    const int j0 = k * kPB, jn = min(kPB, p.N - j0);
    const int par = s & 1;
    // ---- operands of step s -> shared memory (TMA bulk copies) ----
    bar_sync(kBarMath, kMathThreads);  // all warps are done with the previous tiles
    if (warp == 0) {
      if (t.lane == 0) trace_ev(p, s, kTrMathStart);
      const bool ok = warp_wait_all(p, sy.u_flag + Cq * p.TR, p.TR, sy.pc_flag + I, s);
      if (t.lane == 0) {
        sh.math_abort = !ok;
        trace_ev(p, s, kTrMathOperands);
        if (ok) {
          asm volatile("fence.proxy.async.global;" ::: "memory");
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          const uint32_t bytesA = BM * kPB * sizeof(double2), bytesB = kPB * BN * sizeof(double2);
          const uint32_t mb = smem_u32(&sh.mbar);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytesA + bytesB)
                       : "memory");
          const double2* srcA = p.pcbuf + ((size_t)par * p.TR + I) * (BM * kPB);
          const double2* srcB = p.ubuf + ((size_t)par * p.TC + Cq) * (kPB * BN);
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  smem_u32(sh.op.A)),
              "l"(srcA), "r"(bytesA), "r"(mb)
              : "memory");
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  smem_u32(sh.op.B)),
              "l"(srcB), "r"(bytesB), "r"(mb)
              : "memory");
        }
      }
    }
    bar_sync(kBarMath, kMathThreads);
    if (sh.math_abort) return;
    {
      const uint32_t mb = smem_u32(&sh.mbar);
      uint32_t done = 0;
      const long long t0 = clock64();
      int timed_out = 0;
      while (!done && !timed_out) {
        asm volatile(
            "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
            : "=r"(done)
            : "r"(mb), "r"((uint32_t)par)
            : "memory");
        if (!done && clock64() - t0 > p.timeout_cycles) timed_out = 1;
      }
      if (bar_or(kBarMath, kMathThreads, timed_out)) {
        // the copies of this step may still be in flight: give them the same
        // budget once more before the shared memory is abandoned
        if (!done) {
          const long long t1 = clock64();
          while (!done && clock64() - t1 <= p.timeout_cycles)
            asm volatile(
                "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
                : "=r"(done)
                : "r"(mb), "r"((uint32_t)par)
                : "memory");
        }
        if (tid == 0) {
          atomicOr(p.status, kStatusTimeout);
          atomicExch(p.abort, 1);
        }
        return;
      }
    }
    if (tid == 0) {
      trace_ev(p, s, kTrMathCopied);
      atomicAdd(sy.pc_cons + par * p.TR + I, 1);
      atomicAdd(sy.u_cons + par * p.TC + Cq, 1);
    }
    // ---- W_mod: rows and columns of the pivot block J read as zero ----
#pragma unroll
    for (int mi = 0; mi < MI; mi++)
#pragma unroll
      for (int ni = 0; ni < NI; ni++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = t.row(mi), j = t.col(ni, h);
          if ((unsigned)(i - j0) < (unsigned)jn || (unsigned)(j - j0) < (unsigned)jn) {
            t.acc[mi][ni][h] = 0.0;
            t.acc[mi][ni][2 + h] = 0.0;
          }
        }
    // ---- rank-32 update, then the pieces of step s+1 ----
    const int s1 = s + 1;
    const bool last_block = (k == p.NB - 1);
    const bool slice_end = last_block && (s1 < S);
    mma_pass();
    if (!last_block) publish(s1, false);
    if (tid == 0) trace_ev(p, s, kTrMathDone);
    if (last_block) {
      // slice boundary: probe check and the next slice matrix A_{n+1} - G_n
      // in the registers, then the first pieces of slice n+1 published; after
      // the last slice the tile goes to its home in W
      const double2* eps_next = slice_end ? p.eps + (p.eps_first + (int64_t)(n + 1) * p.eps_step) * p.N : nullptr;
      double2* snap = (p.snap && (n % p.snap_mod) == p.snap_mod - 1) ? p.snap + (int64_t)(n / p.snap_mod) * p.snap_ld
                                                                     : nullptr;
      probe_max = fmax(probe_max, boundary_regs(eps_next, snap));
      if (slice_end) publish(s1, true);
      else store_tile();
    }
  }
  for (int off = 16; off > 0; off >>= 1) probe_max = fmax(probe_max, __shfl_xor_sync(kFull, probe_max, off));
  if (t.lane == 0 && probe_max > 0.0)
    atomicMax(p.probe_max, (unsigned long long)__double_as_longlong(probe_max));
}

// ---------------------------------------------------------------------------
// tile CTA, panel warpgroup: U_s(:, my columns) = T_s * W(J_s, my columns),
// then the pivot rows of step s+1 in my columns one step ahead
// ---------------------------------------------------------------------------
// The pivot rows of step s+1 after the update of step s are
//     W^(s)(J_{s+1}, c) = P_{s+1}(c) [c not in J_s] + Pc_s(J_{s+1}, :) U_s(:, c)
// with P_{s+1} = W^(s-1)(J_{s+1}, :), published by the math warps holding
// those rows after step s-1, and Pc_s = -W^(s-1)(:, J_s) the pivot columns
// of step s: the same update the math warps apply to their registers (whose
// rows J_{s+1} are then never read again).  Computing them here, right after
// U_s, takes the math pass of step s off the path from T_s to U_{s+1}.
// The share of panel I is columns [cs, cs + w) of tile column Cq.
template <int BM, int BN>
__device__ void panel_role(const PersistParams& p, Shared& sh, const Sync& sy, int I, int Cq) {
  const int t = threadIdx.x - Cfg<BM, BN>::MathThreads;
  const int lane = t & 31, warp = t >> 5;
  const int S = p.L * p.NB;
  const int per = (BN + p.TR - 1) / p.TR;
  const int cs = I * per;
  const int w = max(0, min(per, BN - cs));
  constexpr int kPer = kPB * kPB / kPanelThreads;
  const int r = warp * 8 + (lane >> 2);  // warp w computes rows [8w, 8w+8), one 8-column tile at a time

  // rows of step s1 = s+1 in my columns -> rowbuf[s1 & 1]: P_{s1} updated by
  // step s, or P_{s1} itself when s1 starts a slice (s = -1: the first step)
  auto lookahead = [&](int s) -> bool {
    const int s1 = s + 1;
    const bool upd = s >= 0 && (s % p.NB) + 1 < p.NB;
    const int par = s & 1, par1 = s1 & 1;
    const int w1 = (s1 % p.NB) * kPB, jn1 = min(kPB, p.N - w1);
    const int I1 = w1 / BM;
    const int j0 = upd ? (s % p.NB) * kPB : 0, jn = upd ? min(kPB, p.N - j0) : 0;
    if (t == 0) {
      int ok = wait_ge(p, sy.pre_flag + par1 * p.TC + Cq, s1);
      if (ok && upd) ok = wait_ge(p, sy.pc_flag + I1, s);
      sh.panel_abort = !ok;
    }
    bar_sync(kBarPanel, kPanelThreads);
    if (sh.panel_abort) return false;
    double2 v[kPer];
    if (upd && w > 0) {  // Pc_s(J_{s1}, :) -> sh.T (T_s is not needed any more)
      const double2* pcb = p.pcbuf + ((size_t)par * p.TR + I1) * (BM * kPB) + (size_t)(w1 - I1 * BM) * kPB;
#pragma unroll
      for (int u = 0; u < kPer; u++) {
        const int e = t + u * kPanelThreads, q = e / kPB, c = e % kPB;
        v[u] = __ldcg(pcb + q * kPB + (c ^ ((q & 1) << 2)));
      }
#pragma unroll
      for (int u = 0; u < kPer; u++) sh.T[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
    }
    const double2* pre = p.prebuf + ((size_t)par1 * p.TC + Cq) * (kPB * BN);
    const double2* ub = p.ubuf + ((size_t)(par & 1) * p.TC + Cq) * (kPB * BN);
    double2* rowo = p.rowbuf + ((size_t)par1 * p.TC + Cq) * (kPB * BN);
    for (int cc = 0; cc < w; cc += kPB) {
      const int wc = min(kPB, w - cc);
      if (upd) {  // U_s(:, this chunk), as stored for the math warps, -> sh.Mr
#pragma unroll
        for (int u = 0; u < kPer; u++) {
          const int e = t + u * kPanelThreads, q = e / kPB, c = e % kPB;
          v[u] = (c < wc) ? __ldcg(ub + swzB<BN>(q, cs + cc + c)) : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < kPer; u++) sh.Mr[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
      }
      bar_sync(kBarPanel, kPanelThreads);
      for (int nt = 0; nt * 8 < wc; nt++) {
        double acc[4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c = nt * 8 + (lane & 3) * 2 + h;
          const int64_t gc = (int64_t)Cq * BN + cs + cc + c;
          double2 pv = (c < wc) ? __ldcg(pre + r * BN + cs + cc + c) : cmk(0.0, 0.0);
          if (gc >= j0 && gc < j0 + jn) pv = cmk(0.0, 0.0);  // columns J_s read as zero
          acc[h] = pv.x;
          acc[2 + h] = pv.y;
        }
        if (upd) {
#pragma unroll
          for (int kk = 0; kk < kPB / 4; kk++) {
            const double2 a = sh.T[r][kk * 4 + (lane & 3)];
            const double2 bb = sh.Mr[kk * 4 + (lane & 3)][nt * 8 + (lane >> 2)];
            dmma(acc[0], acc[1], a.x, bb.x);
            dmma(acc[2], acc[3], a.x, bb.y);
            dmma(acc[0], acc[1], -a.y, bb.y);
            dmma(acc[2], acc[3], a.y, bb.x);
          }
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int c = nt * 8 + (lane & 3) * 2 + h;
          if (c >= wc) continue;
          const int64_t gc = (int64_t)Cq * BN + cs + cc + c;
          const double2 o = (r >= jn1 || gc >= p.C) ? cmk(0.0, 0.0) : cmk(acc[h], acc[2 + h]);
          __stcg(rowo + r * BN + cs + cc + c, o);
        }
      }
      bar_sync(kBarPanel, kPanelThreads);
    }
    if (t == 0) {
      atomicAdd(sy.pre_cons + par1 * p.TC + Cq, 1);
      if (s >= 0) atomicAdd(sy.pcp_cons + par, 1);
      st_release(sy.rowp_flag + Cq * p.TR + I, s1);
    }
    return true;
  };

  for (int s = -1; s < S; s++) {  // s = -1: only the pivot rows of the first step
    if (s >= 0) {
      const int k = s % p.NB;
      const int j0 = k * kPB, jn = min(kPB, p.N - j0);
      const int par = s & 1;
      const double2* tb = p.tbuf + (size_t)par * kPB * kPB;
      const double2* rows = p.rowbuf + ((size_t)par * p.TC + Cq) * (kPB * BN);
      double2* ub = p.ubuf + ((size_t)par * p.TC + Cq) * (kPB * BN);
      // chunk 0 of my pivot rows (written by this warpgroup one step earlier)
      // goes to shared memory before T_s is awaited
      double2 v[kPer];
      if (w > 0) {
#pragma unroll
        for (int u = 0; u < kPer; u++) {
          const int e = t + u * kPanelThreads, q = e / kPB, c = e % kPB;
          v[u] = (c < min(kPB, w)) ? __ldcg(rows + q * BN + cs + c) : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < kPer; u++) sh.Mr[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
      }
      if (t == 0) {
        // the math warps of tile column Cq have copied U of step s-2 (checked
        // before T_s comes, so that it costs nothing on the path from T_s)
        trace_ev(p, s, kTrPanelStart);
        int ok = (w > 0 && s >= 2) ? wait_ge(p, sy.u_cons + par * p.TC + Cq, p.TR * (s >> 1)) : 1;
        ok = ok && wait_ge(p, sy.t_flag, s);
        sh.panel_abort = !ok;
        trace_ev(p, s, kTrPanelUin);
      }
      bar_sync(kBarPanel, kPanelThreads);
      if (sh.panel_abort) return;
      for (int cc = 0; cc < w; cc += kPB) {
        const int wc = min(kPB, w - cc);
        if (cc == 0) {
#pragma unroll
          for (int u = 0; u < kPer; u++) v[u] = __ldcg(tb + t + u * kPanelThreads);
#pragma unroll
          for (int u = 0; u < kPer; u++) sh.T[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
        } else {
#pragma unroll
          for (int u = 0; u < kPer; u++) {
            const int e = t + u * kPanelThreads, q = e / kPB, c = e % kPB;
            v[u] = (c < wc) ? __ldcg(rows + q * BN + cs + cc + c) : cmk(0.0, 0.0);
          }
#pragma unroll
          for (int u = 0; u < kPer; u++) sh.Mr[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
        }
        bar_sync(kBarPanel, kPanelThreads);
        // T_s is padded with the identity and the pivot rows with zeros beyond jn
        for (int nt = 0; nt * 8 < wc; nt++) {
          double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int kk = 0; kk < kPB / 4; kk++) {
            const double2 a = sh.T[r][kk * 4 + (lane & 3)];
            const double2 bb = sh.Mr[kk * 4 + (lane & 3)][nt * 8 + (lane >> 2)];
            dmma(acc[0], acc[1], a.x, bb.x);
            dmma(acc[2], acc[3], a.x, bb.y);
            dmma(acc[0], acc[1], -a.y, bb.y);
            dmma(acc[2], acc[3], a.y, bb.x);
          }
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int c = nt * 8 + (lane & 3) * 2 + h;
            if (c >= wc) continue;
            const int64_t gc = (int64_t)Cq * BN + cs + cc + c;
            double2 o = cmk(acc[h], acc[2 + h]);
            if (r >= jn || gc >= p.C) o = cmk(0.0, 0.0);
            else if (gc >= j0 && gc < j0 + jn) o = sh.T[r][gc - j0];
            __stcg(ub + swzB<BN>(r, cs + cc + c), o);
          }
        }
        bar_sync(kBarPanel, kPanelThreads);
      }
      bar_sync(kBarPanel, kPanelThreads);  // every read of T is done
      if (t == 0) {
        atomicAdd(sy.t_cons + par, 1);
        st_release(sy.u_flag + Cq * p.TR + I, s);
        trace_ev(p, s, kTrPanelUout);
      }
    }
    if (s + 1 < S && !lookahead(s)) return;
  }
}

// ---------------------------------------------------------------------------
// T-server CTA
// ---------------------------------------------------------------------------
// Gauss-Jordan inversion of the 32x32 pivot block with partial pivoting,
// register resident: lane r of warp w holds row r, columns [4w, 4w+4).  The
// block is padded with the identity beyond its jn valid rows and columns, so
// all 32 pivots run (a padding column is a unit vector whose pivot is its
// own padding row; the result is the inverse padded with the identity).
//
// Rows are kept unscaled: after pivot q (row pv, reciprocal d of the pivot
// value, multipliers m(r) = a(r,q) d for r != pv, m(pv) = 0) every column c
// of every warp takes the one complex FMA  a(r,c) -= m(r) a(pv,c), the pivot
// column becomes (-m, with 1 in row pv), and row r is multiplied by the d of
// the pivot it became only at the end.
//
// Warp w chooses the pivots of its own four columns and runs ahead: for each
// one it publishes m(r), pv (and d in lane pv) with a release store of its
// own row's counter, lane by lane, and goes on at once; every warp applies
// the pivots in order, each lane waiting (bounded) on its own row's counter,
// so the chain from one pivot to the next crosses warps only at the
// four-column block boundaries.  Pivot search: one redux.sync over
// single-precision magnitudes packed with the lane index, the reciprocal
// formed speculatively by every lane meanwhile.  Row interchanges are
// implicit:  inv[pinv[r]][perm[c]] = a(r, c),  perm[q] = row chosen at q.
// Returns false in every lane if a wait gave up (abort or timeout).
__device__ __forceinline__ bool gj_ahead(const PersistParams& p, Shared& sh, double2 (&a)[4], int t) {
  constexpr int NC = 4;
  const int lane = t & 31, warp = t >> 5;
  unsigned used = 0;
  bool sing = false, ok = true;
  for (int b = 0; b < kPB / NC; b++) {
    if (warp == b) {
#pragma unroll
      for (int cq = 0; cq < NC; cq++) {
        const int q = b * NC + cq;
        const double2 vq = a[cq];
        const double2 dq = crecip_nr(vq);  // speculative: used only if this lane wins
        const float fx = (float)vq.x, fy = (float)vq.y;
        const float mag = fx * fx + fy * fy;
        const bool elig = !((used >> lane) & 1u);
        const unsigned key = elig ? ((__float_as_uint(mag) & ~63u) | (unsigned)(32 - lane)) : 0u;
        const unsigned best = __reduce_max_sync(kFull, key);
        const int pv = 32 - (int)(best & 63u);
        const double2 d = cmk(__shfl_sync(kFull, dq.x, pv), __shfl_sync(kFull, dq.y, pv));
        const bool me = lane == pv;
        const double2 m = me ? cmk(0.0, 0.0) : cmul(vq, d);
        sh.srv.v[q][lane] = m;
        sh.gpiv[q][lane] = pv;
        if (me) {
          sh.drow[lane] = d;
          sh.pinv[lane] = q;
        }
        if (lane == 0) sh.perm[q] = pv;
        st_release_cta(&sh.gflag[lane], q + 1);
        // a zero reciprocal of a nonzero pivot (|z|^2 beyond the range of
        // rcp.approx.ftz) is as unusable as a non-finite one
        sing = sing || (best >> 6) == 0u || !isfinite(d.x) || !isfinite(d.y) || (d.x == 0.0 && d.y == 0.0);
        used |= 1u << pv;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          if (c == cq) {
            a[c] = me ? cmk(1.0, 0.0) : cneg(m);
          } else {
            const double2 pr = cmk(__shfl_sync(kFull, a[c].x, pv), __shfl_sync(kFull, a[c].y, pv));
            a[c] = cmk(fma(-m.x, pr.x, fma(m.y, pr.y, a[c].x)), fma(-m.x, pr.y, fma(-m.y, pr.x, a[c].y)));
          }
        }
      }
    } else {
#pragma unroll
      for (int cq = 0; cq < NC; cq++) {
        const int q = b * NC + cq;
        if (ld_acquire_cta(&sh.gflag[lane]) <= q) {
          const long long t0 = clock64();
          for (int spins = 1;; spins++) {
            if (ld_acquire_cta(&sh.gflag[lane]) > q) break;
            if ((spins & 63) == 0 && give_up(p, t0)) {
              ok = false;
              break;
            }
          }
        }
        const double2 m = sh.srv.v[q][lane];
        const int pv = sh.gpiv[q][lane] & 31;
        used |= 1u << pv;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const double2 pr = cmk(__shfl_sync(kFull, a[c].x, pv), __shfl_sync(kFull, a[c].y, pv));
          a[c] = cmk(fma(-m.x, pr.x, fma(m.y, pr.y, a[c].x)), fma(-m.x, pr.y, fma(-m.y, pr.x, a[c].y)));
        }
      }
    }
  }
  // every lane has acquired its own row's counter for all 32 pivots, so the
  // reciprocal of the pivot its row became is visible to it
  const double2 dr = sh.drow[lane];
#pragma unroll
  for (int c = 0; c < NC; c++) a[c] = cmul(a[c], dr);
  if (sing && lane == 0) atomicOr(p.status, kStatusSingular);
  return __all_sync(kFull, ok);
}

// Cout = Cin + alpha * A B for padded 32x32 complex blocks in shared memory
// (Cin may be Cout: every element is read and written by the same thread),
// on the FP64 tensor cores; 8 warps, warp w computes rows [8 (w>>1), +8) and
// columns [16 (w&1), +16).
__device__ __forceinline__ void blk_gemm(const Blk& A, const Blk& B, const Blk* Cin, double alpha, Blk& Cout, int t) {
  const int lane = t & 31, warp = t >> 5;
  const int r = 8 * (warp >> 1) + (lane >> 2), cb = 16 * (warp & 1);
  double acc[2][4];
#pragma unroll
  for (int n = 0; n < 2; n++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const double2 c0 = Cin ? (*Cin)[r][cb + 8 * n + (lane & 3) * 2 + h] : cmk(0.0, 0.0);
      acc[n][h] = c0.x;
      acc[n][2 + h] = c0.y;
    }
#pragma unroll
  for (int kk = 0; kk < kPB / 4; kk++) {
    const double2 a = A[8 * (warp >> 1) + (lane >> 2)][kk * 4 + (lane & 3)];
    const double ax = alpha * a.x, ay = alpha * a.y;
    double2 b[2];
#pragma unroll
    for (int n = 0; n < 2; n++) b[n] = B[kk * 4 + (lane & 3)][cb + 8 * n + (lane >> 2)];
#pragma unroll
    for (int n = 0; n < 2; n++) {
      dmma(acc[n][0], acc[n][1], ax, b[n].x);
      dmma(acc[n][2], acc[n][3], ax, b[n].y);
    }
#pragma unroll
    for (int n = 0; n < 2; n++) {
      dmma(acc[n][0], acc[n][1], -ay, b[n].y);
      dmma(acc[n][2], acc[n][3], ay, b[n].x);
    }
  }
#pragma unroll
  for (int n = 0; n < 2; n++)
#pragma unroll
    for (int h = 0; h < 2; h++) Cout[r][cb + 8 * n + (lane & 3) * 2 + h] = cmk(acc[n][h], acc[n][2 + h]);
}

// the 8 math warps of the server CTA form and invert every pivot block one
// step ahead of the bulk update.  For step s (not the first of its slice):
//   a3 = W^{(s-2)}(J_{s-1}, J_s)  = pivot rows of step s-1, columns J_s  } staged by the
//   y0 = W^{(s-2)}(J_s, J_s)                                             } prep warps of
//   y1 = W^{(s-2)}(J_s, J_{s-1})                                         } this CTA
// and W^{(s-1)}(J_s, J_s) = y0 - y1 (T_{s-1} a3); the product V = T_{s-1} a3
// is formed while the prep warps finish y0 and y1.
template <int BM, int BN>
__device__ void server_role(const PersistParams& p, Shared& sh, const Sync& sy, int t) {
  const int lane = t & 31, warp = t >> 5;
  const int S = p.L * p.NB;
  const int ntiles = p.TR * p.TC;
  for (int s = 0; s < S; s++) {
    const int k = s % p.NB;
    const int jn = min(kPB, p.N - k * kPB);
    const int par = s & 1;
    // thread 0: is the T buffer of this parity already free (read by every panel)?
    bool tcons_ok = true;
    if (t == 0) {
      trace_ev(p, s, kTrPanelStart);
      tcons_ok = s < 2 || ld_acquire(sy.t_cons + par) >= ntiles * (s >> 1);
    }
    if (k != 0) {  // V = T_{s-1} a3 while y0 and y1 are formed
      if (bar_or(kBarMath, kServerThreads, (t == 0) ? !wait_cta_ge(p, &sh.asig[par], s) : 0)) return;
      blk_gemm(sh.srv.tprev, sh.srv.a3[par], nullptr, 1.0, sh.srv.v, t);
    }
    int bad = 0;
    if (t == 0) {
      bad = !wait_cta_ge(p, &sh.ysig[par], s);
      trace_ev(p, s, kTrPanelTin);
    }
    if (t < kPB) sh.gflag[t] = 0;
    if (t == 0) sh.gj_fail = 0;
    if (bar_or(kBarMath, kServerThreads, bad)) return;
    if (t == 0) trace_ev(p, s, kTrSrvLoaded);
    if (k != 0) {  // W^{(s-1)}(J_s,J_s) = y0 - y1 V
      blk_gemm(sh.srv.y[par][1], sh.srv.v, &sh.srv.y[par][0], -1.0, sh.srv.a1, t);
      bar_sync(kBarMath, kServerThreads);
    }
    if (t == 0) trace_ev(p, s, kTrSrvSchur);
    double2 a[4];
    const Blk& a0 = (k != 0) ? sh.srv.a1 : sh.srv.y[par][0];
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] = a0[lane][warp * 4 + c];
    if (!gj_ahead(p, sh, a, t)) sh.gj_fail = 1;
    if (t == 0) {
      trace_ev(p, s, kTrSrvGJ);
      sh.panel_abort = tcons_ok ? 0 : !wait_ge(p, sy.t_cons + par, ntiles * (s >> 1));
      st_release_cta(&sh.ycons, s);  // y[par] was read before the Gauss-Jordan started
    }
    bar_sync(kBarMath, kServerThreads);
    if (sh.panel_abort || sh.gj_fail) return;
    double2* tb = p.tbuf + (size_t)par * kPB * kPB;
    const int rr = sh.pinv[lane];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int cc = sh.perm[warp * 4 + c];
      __stcg(tb + rr * kPB + cc, a[c]);
      sh.srv.tprev[rr][cc] = a[c];
    }
    bar_sync(kBarMath, kServerThreads);
    if (t == 0) {
      if (!p.withhold_t) st_release(sy.t_flag, s);
      trace_ev(p, s, kTrPanelTout);
    }
  }
}

// ---------------------------------------------------------------------------
// prep CTA (math warpgroups): for every step x the blocks
//   y0 = W^{(x-2)}(J_x, J_x),  y1 = W^{(x-2)}(J_x, J_{x-1})
// the T-server's Schur update of step x starts from, into ybuf[x & 1].  For
// the second step of a slice they are the blocks the math warps published
// after the slice assembly; from the third step on the published blocks are
// W^{(x-3)} and get the update of step x-2 here,
//   y = B + Pc_{x-2}(J_x, :) U_{x-2}(:, J_x or J_{x-1}),
// from the pivot columns and U rows of step x-2 as stored for the math
// warps.  The first step of a slice passes the first pivot block on.  This
// keeps the math pass of step x-2 off the server's chain, and the products
// off the server's SM, whose Gauss-Jordan they would slow down.
// ---------------------------------------------------------------------------
template <int BM, int BN>
__device__ void yprep_role(const PersistParams& p, Shared& sh, const Sync& sy, int t) {
  const int lane = t & 31, warp = t >> 5;
  const int S = p.L * p.NB;
  constexpr int kPer = kPB * kPB / kServerThreads;
  // bounded load of a 32x32 block (row stride ld; entries outside rows x cols
  // zero; column c read at col_of(c)) into a padded shared block
  auto load_blk = [&](Blk& dst, const double2* src, int ld, int rows, int cols, auto col_of) {
    double2 v[kPer];
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = t + u * kServerThreads, q = e / kPB, c = e % kPB;
      v[u] = (q < rows && c < cols) ? __ldcg(src + (size_t)q * ld + col_of(q, c)) : cmk(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < kPer; u++) dst[(t + u * kServerThreads) / kPB][(t + u * kServerThreads) % kPB] = v[u];
  };
  auto plain = [](int, int c) { return c; };
  Blk& y0 = sh.srv.y[0][0];
  Blk& y1 = sh.srv.y[0][1];
  for (int x = 0; x < S; x++) {
    const int k = x % p.NB, par = x & 1;
    const int w = k * kPB, jn = min(kPB, p.N - w);
    if (warp == 0) {
      int ok = 1;
      if (lane == 0) {
        trace_ev(p, x, kTrMathStart);
        if (x >= 2) ok = wait_ge(p, sy.y_used, x - 2);  // ybuf[par] of step x-2 was loaded
        if (ok) {
          ok = (k == 0) ? wait_ge(p, sy.d_flag, x)
                        : (wait_ge(p, sy.srv_flag + par, x) && wait_ge(p, sy.srv2_flag + par, x));
        }
        if (ok && k >= 2) ok = wait_ge(p, sy.pc_flag + w / BM, x - 2);
      }
      ok = __shfl_sync(kFull, ok, 0);
      if (ok && k >= 2) {  // U_{x-2} of the tile columns holding J_x and J_{x-1}
        ok = warp_wait_all(p, sy.u_flag + (w / BN) * p.TR, p.TR, nullptr, x - 2);
        if (ok) ok = warp_wait_all(p, sy.u_flag + ((w - kPB) / BN) * p.TR, p.TR, nullptr, x - 2);
      }
      sh.panel_abort = !ok;  // every lane writes the same value
    }
    bar_sync(kBarMath, kServerThreads);
    if (sh.panel_abort) return;
    if (k == 0) {
      load_blk(y0, p.djjbuf, kPB, kPB, kPB, plain);
    } else {
      const double2* sb = p.srvbuf + (size_t)par * 2 * kPB * kPB;
      load_blk(y0, sb, kPB, kPB, kPB, plain);
      load_blk(y1, sb + kPB * kPB, kPB, kPB, kPB, plain);
    }
    if (k >= 2) {
      // Pc_{x-2}(J_x, :), rows beyond jn zero -> sh.T; U_{x-2}(:, J_x), columns
      // beyond jn zero -> sh.Mr; U_{x-2}(:, J_{x-1}) -> srv.v
      const int I1 = w / BM, C0 = w / BN, C1 = (w - kPB) / BN;
      load_blk(sh.T, p.pcbuf + ((size_t)par * p.TR + I1) * (BM * kPB) + (size_t)(w - I1 * BM) * kPB, kPB, jn, kPB,
               [](int q, int c) { return c ^ ((q & 1) << 2); });
      const int o0 = w - C0 * BN, o1 = w - kPB - C1 * BN;
      load_blk(sh.Mr, p.ubuf + ((size_t)par * p.TC + C0) * (kPB * BN), 0, kPB, jn,
               [o0](int q, int c) { return swzB<BN>(q, o0 + c); });
      load_blk(sh.srv.v, p.ubuf + ((size_t)par * p.TC + C1) * (kPB * BN), 0, kPB, kPB,
               [o1](int q, int c) { return swzB<BN>(q, o1 + c); });
    }
    bar_sync(kBarMath, kServerThreads);
    if (t == 0) {  // every input is in shared memory: its buffers may be reused
      if (k == 0) st_release(sy.d_used, x);
      atomicAdd(sy.srv_cons + par, 1);
      if (x >= 2) atomicAdd(sy.pcp_cons + par, 1);  // done with the pivot columns of step x-2
    }
    if (k >= 2) {  // the update by step x-2
      blk_gemm(sh.T, sh.Mr, &y0, 1.0, y0, t);
      blk_gemm(sh.T, sh.srv.v, &y1, 1.0, y1, t);
      bar_sync(kBarMath, kServerThreads);
    }
    double2* yb = p.ybuf + (size_t)par * 2 * kPB * kPB;
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = t + u * kServerThreads;
      __stcg(yb + e, y0[e / kPB][e % kPB]);
      if (k != 0) __stcg(yb + kPB * kPB + e, y1[e / kPB][e % kPB]);
    }
    bar_sync(kBarMath, kServerThreads);
    if (t == 0) {
      st_release(sy.y_flag + par, x);
      trace_ev(p, x, kTrMathDone);
    }
  }
}

// T-server CTA, stage warpgroup: copies each step's a3 (the pivot rows of
// step x-1 in columns J_x, from the panels) and y blocks (from the prep CTA)
// into shared memory ahead of the server warps, which find them there.
template <int BM, int BN>
__device__ void stage_role(const PersistParams& p, Shared& sh, const Sync& sy) {
  const int t = threadIdx.x - Cfg<BM, BN>::MathThreads;
  const int lane = t & 31, warp = t >> 5;
  const int S = p.L * p.NB;
  constexpr int kPer = kPB * kPB / kPanelThreads;
  auto copy_blk = [&](Blk& dst, const double2* src, int ld, int cols) {
    double2 v[kPer];
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = t + u * kPanelThreads, q = e / kPB, c = e % kPB;
      v[u] = c < cols ? __ldcg(src + (size_t)q * ld + c) : cmk(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < kPer; u++) dst[(t + u * kPanelThreads) / kPB][(t + u * kPanelThreads) % kPB] = v[u];
  };
  for (int x = 0; x < S; x++) {
    const int k = x % p.NB, par = x & 1;
    const int w = k * kPB, jn = min(kPB, p.N - w);
    // the server warps are done with [par] of step x-2
    if (x >= 2 && bar_or(kBarPanel, kPanelThreads, (t == 0) ? !wait_cta_ge(p, &sh.ycons, x - 2) : 0)) return;
    if (k != 0) {  // a3 comes in shares from the TR panels of its tile column
      int bad = 0;
      if (warp == 0) {
        const bool ok = warp_wait_all(p, sy.rowp_flag + (w / BN) * p.TR, p.TR, nullptr, x - 1);
        bad = (lane == 0) && !ok;
      }
      if (bar_or(kBarPanel, kPanelThreads, bad)) return;
      const int C2 = w / BN;
      copy_blk(sh.srv.a3[par], p.rowbuf + ((size_t)(par ^ 1) * p.TC + C2) * (kPB * BN) + (w - C2 * BN), BN, jn);
      bar_sync(kBarPanel, kPanelThreads);
      if (t == 0) st_release_cta(&sh.asig[par], x);
    }
    if (bar_or(kBarPanel, kPanelThreads, (t == 0) ? !wait_ge(p, sy.y_flag + par, x) : 0)) return;
    const double2* yb = p.ybuf + (size_t)par * 2 * kPB * kPB;
    copy_blk(sh.srv.y[par][0], yb, kPB, kPB);
    if (k != 0) copy_blk(sh.srv.y[par][1], yb + kPB * kPB, kPB, kPB);
    bar_sync(kBarPanel, kPanelThreads);
    if (t == 0) {
      st_release_cta(&sh.ysig[par], x);
      st_release(sy.y_used, x);
    }
  }
}

template <int BM, int BN>
__global__ void __launch_bounds__(Cfg<BM, BN>::Threads, 1) k_persist(PersistParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Shared& sh = *reinterpret_cast<Shared*>(smem_raw);
  const int I = blockIdx.x / p.TC, Cq = blockIdx.x % p.TC;
  Sync sy(p);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sh.mbar)) : "memory");
    sh.math_abort = 0;
    sh.panel_abort = 0;
    sh.ysig[0] = sh.ysig[1] = -1;
    sh.asig[0] = sh.asig[1] = -1;
    sh.ycons = -1;
  }
  __syncthreads();
  const bool server = blockIdx.x == (unsigned)(p.TR * p.TC);
  const bool yprep = blockIdx.x == (unsigned)(p.TR * p.TC + 1);
  static_assert(Cfg<BM, BN>::MathThreads == kServerThreads, "the server uses the math warpgroups");
  if (threadIdx.x < Cfg<BM, BN>::MathThreads) {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(Cfg<BM, BN>::MathRegs));
    if (server) server_role<BM, BN>(p, sh, sy, threadIdx.x);
    else if (yprep) yprep_role<BM, BN>(p, sh, sy, threadIdx.x);
    else math_role<BM, BN>(p, sh, sy, I, Cq);
  } else {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(Cfg<BM, BN>::PanelRegs));
    if (server) stage_role<BM, BN>(p, sh, sy);
    else if (!yprep) panel_role<BM, BN>(p, sh, sy, I, Cq);
  }
}

// ---------------------------------------------------------------------------
// Many structures in one launch: gangs of CTAs sized to each structure, handed
// out by a work queue in device memory.
// ---------------------------------------------------------------------------
// The grid holds one CTA per SM.  A CTA that is free takes the queue's lock,
// joins the pool of free CTAs and, while a structure not yet dispatched fits
// the pool (the items are ordered by cost, largest first: the first that
// fits among the kGangWindow next ones), hands it a gang: each gang member gets
// the item and its place in the item's grid (tile CTA, T-server or prep CTA)
// through its mailbox.  Every member then runs the role the single-structure kernel would
// give it, with the item's own exchange buffers and flags; when it returns,
// the CTA is free again.  Once the queue is empty every CTA in the pool is
// told to stop.  The head of the queue always fits the grid, so when all
// gangs have finished it is dispatched: no deadlock.  Waits for the lock and
// for a mailbox are bounded by `sched_timeout` cycles (they may span the run
// of a whole structure) and poll the queue's abort word.
__device__ __forceinline__ int ldcg_i(const int* p) { return __ldcg(p); }
__device__ __forceinline__ void stcg_i(int* p, int v) { __stcg(p, v); }

// Parameters of the structures of a gang launch: constant memory, read by
// every role as the single-structure kernel reads its launch parameters
// (kept in constant banks, so the roles' register use stays as it is there).
__constant__ PersistParams c_gang_p[kGangMaxItems];
static_assert(sizeof(c_gang_p) <= 60 * 1024, "gang parameters must fit the constant bank");

__device__ bool gang_lock(GangState* gs, long long timeout) {
  const long long t0 = clock64();
  while (atomicCAS(&gs->lock, 0, 1) != 0) {
    if (ldcg_i(&gs->abort)) return false;
    if (clock64() - t0 > timeout) {
      atomicExch(&gs->abort, 1);
      return false;
    }
    __nanosleep(64);
  }
  __threadfence();
  return true;
}

__device__ void gang_unlock(GangState* gs) {
  __threadfence();
  atomicExch(&gs->lock, 0);
}

__device__ void gang_mail(GangState* gs, int cta, int item, int local) {
  stcg_i(&gs->mail_item[cta], item);
  stcg_i(&gs->mail_local[cta], local);
  __threadfence();
  atomicAdd(&gs->mail_seq[cta], 1);
}

// thread 0 of CTA `me`: the next assignment (item, place), item < 0 = stop
__device__ void gang_next(const int* __restrict__ ctas, int count, GangState* gs, int me, int seq, long long timeout,
                          int* item, int* local) {
  *item = -1;
  *local = 0;
  if (!gang_lock(gs, timeout)) return;
  int nfree = ldcg_i(&gs->nfree);
  int next = ldcg_i(&gs->next);
  stcg_i(&gs->pool[nfree++], me);
  // dispatch, as long as something fits the pool: the first structure, in
  // queue order, among the kGangWindow next ones not yet dispatched that fits
  // (the head whenever it fits; smaller ones behind it fill CTAs the head
  // cannot use yet).  A dispatched structure is marked taken; the head moves
  // past taken ones.
  for (;;) {
    int pick = -1;
    for (int q = next, seen = 0; q < count && seen < kGangWindow; q++) {
      if (ldcg_i(&gs->taken[q])) continue;
      seen++;
      if (ctas[q] <= nfree) {
        pick = q;
        break;
      }
    }
    if (pick < 0) break;
    stcg_i(&gs->taken[pick], 1);
    const int need = ctas[pick];
    for (int l = 0; l < need; l++) gang_mail(gs, ldcg_i(&gs->pool[--nfree]), pick, l);
    while (next < count && ldcg_i(&gs->taken[next])) next++;
  }
  if (next >= count) {
    while (nfree > 0) gang_mail(gs, ldcg_i(&gs->pool[--nfree]), -1, 0);
  }
  stcg_i(&gs->nfree, nfree);
  stcg_i(&gs->next, next);
  gang_unlock(gs);
  const long long t0 = clock64();
  for (int spins = 0;; spins++) {
    if (ld_acquire(&gs->mail_seq[me]) > seq) break;
    if (ldcg_i(&gs->abort)) return;
    if ((spins & 63) == 63 && clock64() - t0 > timeout) {
      atomicExch(&gs->abort, 1);
      return;
    }
    __nanosleep(128);
  }
  *item = ldcg_i(&gs->mail_item[me]);
  *local = ldcg_i(&gs->mail_local[me]);
}

template <int BM, int BN>
__global__ void __launch_bounds__(Cfg<BM, BN>::Threads, 1)
    k_persist_gang(const int* __restrict__ ctas, int count, GangState* gs, long long sched_timeout) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Shared& sh = *reinterpret_cast<Shared*>(smem_raw);
  __shared__ int s_item, s_local;
  constexpr int kAll = Cfg<BM, BN>::Threads;
  const uint32_t mb = smem_u32(&sh.mbar);
  // The two warpgroup kinds keep their own loops (their register budgets
  // differ after setmaxnreg) and meet only at the named barrier kBarGang.
  if (threadIdx.x < Cfg<BM, BN>::MathThreads) {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(Cfg<BM, BN>::MathRegs));
    if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    for (int seq = 0;; seq++) {
      if (threadIdx.x == 0) {
        int item, local;
        gang_next(ctas, count, gs, (int)blockIdx.x, seq, sched_timeout, &item, &local);
        s_item = item;
        s_local = local;
        if (item >= 0) {
          // the mbarrier's phase restarts with the structure's step count
          asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
          asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
          sh.math_abort = 0;
          sh.panel_abort = 0;
          sh.ysig[0] = sh.ysig[1] = -1;
          sh.asig[0] = sh.asig[1] = -1;
          sh.ycons = -1;
        }
      }
      bar_sync(kBarGang, kAll);
      const int item = s_item, local = s_local;
      if (item < 0) break;
      const PersistParams& p = c_gang_p[item];
      Sync sy(p);
      const int ntiles = p.TR * p.TC;
      if (local == ntiles) server_role<BM, BN>(p, sh, sy, threadIdx.x);
      else if (local == ntiles + 1) yprep_role<BM, BN>(p, sh, sy, threadIdx.x);
      else math_role<BM, BN>(p, sh, sy, local / p.TC, local % p.TC);
      bar_sync(kBarGang, kAll);  // the whole CTA is done with the item
    }
  } else {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(Cfg<BM, BN>::PanelRegs));
    for (;;) {
      bar_sync(kBarGang, kAll);
      const int item = s_item, local = s_local;
      if (item < 0) break;
      const PersistParams& p = c_gang_p[item];
      Sync sy(p);
      const int ntiles = p.TR * p.TC;
      if (local == ntiles) stage_role<BM, BN>(p, sh, sy);
      else if (local != ntiles + 1) panel_role<BM, BN>(p, sh, sy, local / p.TC, local % p.TC);
      bar_sync(kBarGang, kAll);
    }
  }
}

}  // namespace

size_t persist_smem_bytes() { return sizeof(Shared); }

cudaError_t launch_persist_gang(const PersistParams* params, const int* ctas, int count, GangState* state, int grid,
                                long long sched_timeout, int BM, int BN, cudaStream_t s) {
  if (count > kGangMaxItems) return cudaErrorInvalidValue;
  const void* fn = nullptr;
  if (BM == 96 && BN == 96) fn = (const void*)k_persist_gang<96, 96>;
  else if (BM == 64 && BN == 64) fn = (const void*)k_persist_gang<64, 64>;
  else if (BM == 32 && BN == 32) fn = (const void*)k_persist_gang<32, 32>;
  else return cudaErrorInvalidValue;
  const size_t smem = sizeof(Shared);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyToSymbolAsync(c_gang_p, params, sizeof(PersistParams) * count, 0, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&ctas, (void*)&count, (void*)&state, (void*)&sched_timeout};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(persist_threads(BM, BN)), args, smem, s);
}

int persist_threads(int BM, int BN) {
  if (BM == 96) return Cfg<96, 96>::Threads;
  if (BM == 64) return Cfg<64, 64>::Threads;
  return Cfg<32, 32>::Threads;
}

// tile shape: the largest that keeps >= 60% of the SMs busy, else the one
// with the most CTAs; two SMs always stay free for the T-server and prep CTAs.  With
// prefer_large (several sweeps sharing the GPU) simply the largest tile whose
// grid fits in `sms`.
bool persist_choose_tile(int64_t R, int64_t C, int sms, int* BM, int* BN, bool prefer_large) {
  const int cand[3] = {96, 64, 32};
  const int avail = sms - kPersistExtraCtas;
  for (int q = 0; q < 3 && prefer_large; q++) {
    const int64_t tiles = ((R + cand[q] - 1) / cand[q]) * ((C + cand[q] - 1) / cand[q]);
    if (tiles <= avail) {
      *BM = *BN = cand[q];
      return true;
    }
  }
  for (int q = 0; q < 3; q++) {
    const int64_t tiles = ((R + cand[q] - 1) / cand[q]) * ((C + cand[q] - 1) / cand[q]);
    if (tiles <= avail && tiles * 10 >= (int64_t)avail * 6) {
      *BM = *BN = cand[q];
      return true;
    }
  }
  for (int q = 2; q >= 0; q--) {
    const int64_t tiles = ((R + cand[q] - 1) / cand[q]) * ((C + cand[q] - 1) / cand[q]);
    if (tiles <= avail) {
      *BM = *BN = cand[q];
      return true;
    }
  }
  return false;
}

cudaError_t launch_persist(const PersistParams& p, int BM, int BN, cudaStream_t s) {
  PersistParams pp = p;
  void* args[] = {(void*)&pp};
  const size_t smem = sizeof(Shared);
  const void* fn = nullptr;
  if (BM == 96 && BN == 96) fn = (const void*)k_persist<96, 96>;
  else if (BM == 64 && BN == 64) fn = (const void*)k_persist<64, 64>;
  else if (BM == 32 && BN == 32) fn = (const void*)k_persist<32, 32>;
  else return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaLaunchCooperativeKernel(fn, dim3(p.TR * p.TC + kPersistExtraCtas), dim3(persist_threads(BM, BN)), args,
                                     smem, s);
}

}  // namespace rgf

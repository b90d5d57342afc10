// Persistent slice-recursion kernel (see persist.cu).
#pragma once
#include "rgf_internal.cuh"

namespace rgf {

struct PersistParams {
  int N, R, C;           // pivot dimension, active rows, active columns of the augmented matrix
  int TR, TC;            // tile grid (TR x TC CTAs)
  int NB;                // pivot blocks per slice = ceil(N / 32)
  int L;                 // slices swept by this launch
  double2* M;            // augmented matrix (row-major, leading dimension ldm): in and out
  int64_t ldm;
  const double2* eps;    // slice n (recursion order) is eps + (eps_first + n * eps_step) * N
  int64_t eps_first, eps_step;
  double2 k2;            // k0dx^2
  const int* st_col;     // A0 stencil, kMaxStencil entries per row
  const double2* st_val;
  int pc1;               // probe columns pc1, pc1 + 1 (pc1 even), -1 = none
  double2* pcbuf;        // [2][TR][BM][32]
  double2* rowbuf;       // [2][TC][32][BN] pivot rows of a step (written by the panels)
  double2* prebuf;       // [2][TC][32][BN] the same rows one step earlier (written by the math warps)
  double2* tbuf;         // [2][32][32]
  double2* ubuf;         // [2][TC][32][BN]
  double2* djjbuf;       // [32][32] first pivot block of a slice, for the T-server CTA
  double2* srvbuf;       // [2][2][32][32] blocks the prep CTA updates into the T-server's blocks
  double2* ybuf;         // [2][2][32][32] the T-server's blocks (J_s, J_s), (J_s, J_{s-1}) of a step
  int* flags;  // pc[TR], pre[2][TC], t[1], u[TC*TR], d[1], srv[2], d_used[1], rowp[TC*TR], srv2[2],
               // y[2], y_used[1] (init -1)
  int* cons;   // pc[2][TR], pre[2][TC], t[2], u[2][TC], srv[2], pcp[2]                              (init 0)
  // optional snapshots of W after slice n (launch-relative) for every n with
  // n % snap_mod == snap_mod - 1, at snap + (n / snap_mod) * snap_ld, laid
  // out as M (probe columns excepted)
  double2* snap;
  int snap_mod;
  int64_t snap_ld;
  int* status;           // kStatus* bits
  int* abort;            // raised by the first wait that times out
  unsigned long long* probe_max;  // bits of max |G_n M_n v - v| (non-negative double)
  long long timeout_cycles;
  int withhold_t;        // test hook: the T-server never releases its T flag
  // optional per-step event timestamps (%globaltimer, ns) for the first
  // trace_steps steps: trace[(cta * trace_steps + s) * kTraceEvents + e]
  unsigned long long* trace;
  int trace_steps;
};

// trace events: math role
enum { kTrMathStart = 0, kTrMathOperands, kTrMathCopied, kTrMathPublished, kTrMathDone,
       // panel role
       kTrPanelStart, kTrPanelTin, kTrPanelTout, kTrPanelUin, kTrPanelUout,
       // finer grain: server pieces loaded / next pivot block formed / GJ done
       kTrSrvLoaded, kTrSrvSchur, kTrSrvGJ,
       // publication of the pivot rows / columns and of the server blocks (lead warp)
       kTrGlobEnter, kTrGlobStored, kTrSrvPubEnter, kTrSrvPubStored, kTrSrvPubDone,
       // T-server: end of the factorization of each 4-pivot group
       kTrSrvGroup0, kTraceEvents = kTrSrvGroup0 + 8 };

inline int persist_flag_words(int TR, int TC) { return TR + 2 * TC + 1 + TR * TC + 1 + 2 + 1 + TR * TC + 2 + 3; }
// CTAs beyond the TR x TC tiles: the T-server and the prep CTA
constexpr int kPersistExtraCtas = 2;
inline int persist_cons_words(int TR, int TC) { return 2 * TR + 2 * TC + 2 + 2 * TC + 2 + 2; }

// Several structures in one cooperative launch (gangs of CTAs from a device
// work queue, see persist.cu).  params / ctas (host) are ordered by cost,
// largest first; ctas[i] = TR * TC + kPersistExtraCtas <= grid; at most
// kGangMaxItems structures.  Launches that share a device must not overlap
// (the parameters live in one constant-memory array).
constexpr int kGangMaxCtas = 1024;
constexpr int kGangMaxItems = 160;  // structures per launch (constant memory)
constexpr int kGangWindow = 16;     // queue positions a free pool may look ahead
struct GangState {  // zero-initialised before the launch
  int lock, next, nfree, abort;
  int pool[kGangMaxCtas];
  int mail_seq[kGangMaxCtas], mail_item[kGangMaxCtas], mail_local[kGangMaxCtas];
  int taken[kGangMaxItems];
};
cudaError_t launch_persist_gang(const PersistParams* params, const int* ctas, int count, GangState* state, int grid,
                                long long sched_timeout, int BM, int BN, cudaStream_t s);

size_t persist_smem_bytes();
int persist_threads(int BM, int BN);
bool persist_choose_tile(int64_t R, int64_t C, int sms, int* BM, int* BN, bool prefer_large = false);
cudaError_t launch_persist(const PersistParams& p, int BM, int BN, cudaStream_t s);

}  // namespace rgf

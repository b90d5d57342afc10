// C ABI of librgf (include/rgf.h): handle, workspace and the host-side
// orchestration of the device pipeline
//
//   channels -> transverse profiles phi -> lead G0 (complex GEMM) ->
//   initial augmented slice matrix -> L sweeps (one per slice) ->
//   attach of the far lead -> Fisher-Lee extraction
//
// following cal_smatrix_RGF.m:95-289 (cal_smatrix_RGF_3D.m:93-304 in 3D).
// Input validation mirrors cal_smatrix_RGF.m:79-93 / 103-178; errors are
// returned as rgf_status with a message in rgf_last_error().
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <chrono>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "channels.cuh"
#include "persist.cuh"
#include "rgf_internal.cuh"
#include "mixed.cuh"
#include "sweep.cuh"

namespace rgf {

static thread_local std::string tl_err;
void set_error(const std::string& msg) { tl_err = msg; }

// Bump region of caller-independent device memory (the static scratch of
// rgf_smatrix_2d_noalloc); buffers carved from it are never freed.
struct Arena {
  unsigned char* base = nullptr;
  size_t cap = 0, used = 0;
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct GangBatch {
  std::mutex mu;
  std::condition_variable cv;
  int pending = 0;  // threads that have neither handed in a sweep nor left
  bool done = false;
  cudaError_t result = cudaSuccess;
  struct Sub {
    PersistParams p;
    int ctas;
    double cost;
  };
  std::vector<Sub> subs;
  int device = 0, sms = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
};


}  // namespace rgf

using namespace rgf;

struct rgf_handle_s {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the handle's own stream
  // sampled kernel timing (rgf_options.profile)
  std::vector<cudaEvent_t> ev;
  int64_t prof_n = 0;
  double prof_ms = 0.0, prof_flops = 0.0;
  // workspace (grow-only)
  DevBuf k0, k1, kx[2], lam[2], mu[2], isprop[2], prop[2], conj[2], nprop, status;
  DevBuf phi, tmp, g0s, g0e, st_col, st_val, eps, aug, pc, u, idx, sdev;
  DevBuf xpc, xrow, xt, xu, xsync, xprobe;  // persistent-kernel exchange buffers
  DevBuf gck, gseg, gm0, gpsi, gphi, get, gd, gg;   // permittivity gradient (checkpoints, carriers)
  DevBuf gf;                                        // fields staged for a host output
  DevBuf segs;                                      // segment states staged for a merge
  int sms = 0;
  // batched calls: one sub-handle per concurrent pipeline (own stream and
  // workspace, a share of the SMs for its persistent sweeps)
  std::vector<rgf_handle_s*> workers;
  std::atomic<int> sm_free{0};          // batch parent: SMs not held by a running sweep
  std::atomic<int>* sm_budget = nullptr;  // batch worker: the parent's counter
  int64_t launches = 0;
  std::string prof_kernel;
  double probe = 0.0;
  DevBuf gepp;  // scratch of the whole-column pivoting (per-step engine)
  // tuned tile table of the persistent engine: rows Rp <= tile_rmax[i] use
  // tile tile_bm[i] (first match) when its grid fits the GPU
  std::vector<int64_t> tile_rmax;
  std::vector<int> tile_bm;
  // batched call in one launch: the coordinator this worker hands its sweep to
  rgf::GangBatch* gang = nullptr;
  bool gang_submitted = false;
  int engine_used = 0;     // engine of the last call's final run
  int fallback = 0;        // 1: the persistent engine's result was rejected and recomputed
  double probe_first = 0;  // probe residual of the rejected run
  // non-null: every workspace buffer is carved from this arena and nothing is
  // ever allocated (the handle of rgf_smatrix_2d_noalloc)
  Arena* arena = nullptr;
  // split-precision form (RGF_TF32X3): workspace, and what the last call did
  DevBuf mx[kMxSlots];
  MixedStats mx_stats;
  int mx_form = RGF_FP64;  // form whose S the last call returned
  int mx_fallback = 0;     // 1: the refinement did not converge and S is the FP64 form's
};

namespace {

#define RGF_CUDA_TRY(call)                                                         \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call); \
      return e_ == cudaErrorMemoryAllocation ? RGF_ERR_OOM : RGF_ERR_CUDA;         \
    }                                                                              \
  } while (0)

rgf_status ensure(rgf_handle h, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return RGF_OK;
  if (h->arena) {  // never cudaMalloc on an allocation-free handle
    Arena* a = h->arena;
    const size_t need = (bytes + 255) & ~(size_t)255;
    if (a->used + need > a->cap) {
      set_error("problem too large for the static device scratch of rgf_smatrix_2d_noalloc (" +
                std::to_string(a->cap >> 20) + " MiB): its workspace needs more; use rgf_smatrix_2d");
      return RGF_ERR_ARG;
    }
    b.p = a->base + a->used;
    b.bytes = bytes;
    a->used += need;
    return RGF_OK;
  }
  // stream-ordered (re)allocation: cudaFree / cudaMalloc would synchronize the
  // whole device, stalling the concurrent pipelines of a batched call
  if (b.p) cudaFreeAsync(b.p, h->stream);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMallocAsync(&b.p, bytes, h->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
              cudaGetErrorString(e));
    return RGF_ERR_OOM;
  }
  b.bytes = bytes;
  return RGF_OK;
}

template <class T>
T* as(DevBuf& b) {
  return reinterpret_cast<T*>(b.p);
}

inline double2 d2(rgf_cplx c) { return make_double2(c.re, c.im); }
inline bool finite_c(rgf_cplx c) { return isfinite(c.re) && isfinite(c.im); }

rgf_status check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("CUDA launch failed: ") + cudaGetErrorString(e));
    return RGF_ERR_CUDA;
  }
  return RGF_OK;
}

// ---------------------------------------------------------------------------
// channels (setup_channels.m / setup_channels_3D.m)
// ---------------------------------------------------------------------------
struct ChanInfo {
  int64_t np[2] = {0, 0};
  bool same = false;   // R side aliases L (epsilon_R == epsilon_L, setup_channels.m:166)
  bool two_sided = true;
  bool has_conj = false;
  SideDev side[2];
};

SideDev side_of(rgf_handle h, int s) {
  SideDev d;
  d.kx = as<double2>(h->kx[s]);
  d.lam = as<double2>(h->lam[s]);
  d.sqrtmu = as<double2>(h->mu[s]);
  d.isprop = as<int>(h->isprop[s]);
  d.prop = as<int>(h->prop[s]);
  d.nprop = as<int>(h->nprop) + s;
  d.conj = as<int>(h->conj[s]);
  return d;
}

rgf_status run_channels(rgf_handle h, const Transverse& tr, double2 k2eL, double2 k2eR, bool two_sided,
                        ChanInfo* ci) {
  const int64_t N = tr.N;
  rgf_status st;
  if ((st = ensure(h, h->k0, sizeof(double) * tr.n0))) return st;
  if ((st = ensure(h, h->k1, sizeof(double) * tr.n1))) return st;
  for (int s = 0; s < 2; s++) {
    if ((st = ensure(h, h->kx[s], sizeof(double2) * N))) return st;
    if ((st = ensure(h, h->lam[s], sizeof(double2) * N))) return st;
    if ((st = ensure(h, h->mu[s], sizeof(double2) * N))) return st;
    if ((st = ensure(h, h->isprop[s], sizeof(int) * N))) return st;
    if ((st = ensure(h, h->prop[s], sizeof(int) * N))) return st;
    if ((st = ensure(h, h->conj[s], sizeof(int) * N))) return st;
  }
  if ((st = ensure(h, h->nprop, sizeof(int) * 2))) return st;
  ci->two_sided = two_sided;
  ci->same = !two_sided || (k2eL.x == k2eR.x && k2eL.y == k2eR.y);
  int conj_mode = 0;
  int64_t ind_zero0 = -1;
  if (tr.dim == 2) {
    if (tr.bc == RGF_BC_PERIODIC || (tr.bc == RGF_BC_BLOCH && tr.ka0 == 0.0)) {
      conj_mode = 2;
      ind_zero0 = ((tr.n0 % 2 == 1) ? (tr.n0 + 1) / 2 : tr.n0 / 2) - 1;
    } else if (tr.bc != RGF_BC_BLOCH) {
      conj_mode = 1;
    }
  }
  ci->has_conj = conj_mode != 0;
  launch_transverse(tr, as<double>(h->k0), as<double>(h->k1), h->stream);
  h->launches++;
  for (int s = 0; s < 2; s++) {
    ci->side[s] = side_of(h, s);
    if (s == 1 && ci->same) {
      ci->side[1] = ci->side[0];
      continue;
    }
    launch_longitudinal(tr, as<double>(h->k0), as<double>(h->k1), s == 0 ? k2eL : k2eR, ci->side[s], h->stream);
    launch_compact(N, ci->side[s], conj_mode, ind_zero0, h->stream);
    h->launches += 2;
  }
  if ((st = check_launch())) return st;
  int np[2] = {0, 0};
  RGF_CUDA_TRY(cudaMemcpyAsync(np, as<int>(h->nprop), sizeof(int) * 2, cudaMemcpyDeviceToHost, h->stream));
  RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
  ci->np[0] = np[0];
  ci->np[1] = ci->same ? np[0] : np[1];
  return RGF_OK;
}

rgf_status copy_channels_out(rgf_handle h, const Transverse& tr, const ChanInfo& ci, rgf_channels* ch) {
  if (!ch) return RGF_OK;
  const int64_t N = tr.N;
  std::vector<double> k0(tr.n0), k1(tr.n1);
  RGF_CUDA_TRY(cudaMemcpy(k0.data(), h->k0.p, sizeof(double) * tr.n0, cudaMemcpyDeviceToHost));
  if (tr.dim == 3) RGF_CUDA_TRY(cudaMemcpy(k1.data(), h->k1.p, sizeof(double) * tr.n1, cudaMemcpyDeviceToHost));
  if (ch->kydx) {
    for (int64_t a = 0; a < N; a++) ch->kydx[a] = (tr.dim == 2) ? k0[a] : k1[a / tr.n0];
  }
  if (ch->kxdx_t && tr.dim == 3) {
    for (int64_t a = 0; a < N; a++) ch->kxdx_t[a] = k0[a % tr.n0];
  }
  const int nsides = ci.two_sided ? 2 : 1;
  for (int s = 0; s < nsides; s++) {
    const SideDev& sd = ci.side[s];
    rgf_cplx* kx = s == 0 ? ch->kxdx_L : ch->kxdx_R;
    rgf_cplx* mu = s == 0 ? ch->sqrt_mu_L : ch->sqrt_mu_R;
    int64_t* ip = s == 0 ? ch->ind_prop_L : ch->ind_prop_R;
    int64_t* ic = s == 0 ? ch->ind_prop_conj_L : ch->ind_prop_conj_R;
    const int64_t np = ci.np[s];
    if (kx) RGF_CUDA_TRY(cudaMemcpy(kx, sd.kx, sizeof(double2) * N, cudaMemcpyDeviceToHost));
    std::vector<int> prop(np > 0 ? np : 1), conj(np > 0 ? np : 1);
    std::vector<double2> muall(N);
    if (np > 0) RGF_CUDA_TRY(cudaMemcpy(prop.data(), sd.prop, sizeof(int) * np, cudaMemcpyDeviceToHost));
    if (mu) {
      RGF_CUDA_TRY(cudaMemcpy(muall.data(), sd.sqrtmu, sizeof(double2) * N, cudaMemcpyDeviceToHost));
      for (int64_t p = 0; p < np; p++) mu[p] = rgf_cplx{muall[prop[p]].x, muall[prop[p]].y};
    }
    if (ip)
      for (int64_t p = 0; p < np; p++) ip[p] = prop[p];
    if (ic && ci.has_conj && np > 0) {
      RGF_CUDA_TRY(cudaMemcpy(conj.data(), sd.conj, sizeof(int) * np, cudaMemcpyDeviceToHost));
      for (int64_t p = 0; p < np; p++) ic[p] = conj[p];
    }
  }
  ch->N_prop_L = ci.np[0];
  ch->N_prop_R = ci.two_sided ? ci.np[1] : -1;
  ch->has_prop_conj = ci.has_conj ? 1 : 0;
  return RGF_OK;
}

// resolve one side's channel list (cal_smatrix_RGF.m:103-178)
rgf_status resolve_list(const int64_t* ind, int64_t n, int64_t np, const char* name, char side,
                        std::vector<int>* out) {
  out->clear();
  if (n == RGF_ALL) {
    for (int64_t p = 0; p < np; p++) out->push_back((int)p);
    return RGF_OK;
  }
  if (n < 0) {
    set_error(std::string(name) + ": negative channel count");
    return RGF_ERR_ARG;
  }
  if (n > 0 && !ind) {
    set_error(std::string(name) + ": NULL index list");
    return RGF_ERR_ARG;
  }
  for (int64_t k = 0; k < n; k++) {
    if (ind[k] < 0 || ind[k] >= np) {
      set_error(std::string(name) + ", when specified, must be an array of positive integers not exceeding N_prop_" +
                side + "=" + std::to_string(np));
      return RGF_ERR_ARG;
    }
    out->push_back((int)ind[k]);
  }
  return RGF_OK;
}

// MATLAB [~, io, ii] = intersect(out, in): first occurrences of common values
void intersect_pairs(const std::vector<int>& out, const std::vector<int>& in, int off_o, int off_i,
                     std::vector<int>* pairs) {
  std::vector<int> vals;
  for (int v : out)
    if (std::find(in.begin(), in.end(), v) != in.end() && std::find(vals.begin(), vals.end(), v) == vals.end())
      vals.push_back(v);
  for (int v : vals) {
    int io = (int)(std::find(out.begin(), out.end(), v) - out.begin());
    int ii = (int)(std::find(in.begin(), in.end(), v) - in.begin());
    pairs->push_back(off_o + io);
    pairs->push_back(off_i + ii);
  }
}

struct Request {
  std::vector<int> out[2], in[2];  // [L, R]
};

rgf_status resolve_request(const rgf_request* req, const ChanInfo& ci, Request* r) {
  rgf_status st;
  if ((st = resolve_list(req->ind_out_L, req->n_out_L, ci.np[0], "out.ind_out_L", 'L', &r->out[0]))) return st;
  if ((st = resolve_list(req->ind_out_R, req->n_out_R, ci.np[1], "out.ind_out_R", 'R', &r->out[1]))) return st;
  if ((st = resolve_list(req->ind_in_L, req->n_in_L, ci.np[0], "in.ind_in_L", 'L', &r->in[0]))) return st;
  if ((st = resolve_list(req->ind_in_R, req->n_in_R, ci.np[1], "in.ind_in_R", 'R', &r->in[1]))) return st;
  return RGF_OK;
}

// ---------------------------------------------------------------------------
// the S-matrix pipeline shared by 2D and 3D
// ---------------------------------------------------------------------------
struct Problem {
  Transverse tr;
  int64_t L;
  const rgf_cplx* eps;
  bool eps_dev;
  rgf_cplx epsL, epsR, k0dx;
};

rgf_status validate_problem(const Problem& p, const rgf_request* req) {
  if (!req) {
    set_error("request must not be NULL");
    return RGF_ERR_ARG;
  }
  if (p.tr.N <= 0 || p.tr.n0 <= 0 || p.tr.n1 <= 0) {
    set_error(p.tr.dim == 2 ? "need at least one site along the transverse (y) direction"
                            : "need at least one site along the transverse directions (x,y)");
    return RGF_ERR_ARG;
  }
  if (p.tr.N > (int64_t)1 << 30) {
    set_error("transverse size too large");
    return RGF_ERR_ARG;
  }
  if (p.L < 0) {
    set_error("number of slices must be >= 0");
    return RGF_ERR_ARG;
  }
  if (p.L > 0 && !p.eps) {
    set_error("syst.epsilon must be provided");
    return RGF_ERR_ARG;
  }
  if (!finite_c(p.k0dx) || !finite_c(p.epsL) || !finite_c(p.epsR)) {
    set_error("syst.k0dx, syst.epsilon_L and syst.epsilon_R must be finite");
    return RGF_ERR_NONFINITE;
  }
  if (p.tr.bc < 0 || p.tr.bc > RGF_BC_BLOCH || (p.tr.dim == 3 && p.tr.bc != RGF_BC_PERIODIC &&
                                                p.tr.bc != RGF_BC_DIRICHLET && p.tr.bc != RGF_BC_BLOCH)) {
    set_error("Boundary condition BC is not an eligible option");
    return RGF_ERR_ARG;
  }
  if (!isfinite(p.tr.ka0) || !isfinite(p.tr.ka1)) {
    set_error("Bloch phase must be finite and real");
    return RGF_ERR_ARG;
  }
  return RGF_OK;
}

void k2eps(rgf_cplx k0dx, rgf_cplx eps, double2* k2, double2* k2e) {
  double2 k = d2(k0dx);
  *k2 = cmul(k, k);
  *k2e = cmul(*k2, d2(eps));
}

rgf_status smatrix_sizes(rgf_handle h, const Problem& p, const rgf_request* req, int64_t* n_out,
                         int64_t* n_in) {
  rgf_status st;
  if ((st = validate_problem(p, req))) return st;
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  double2 k2, k2eL, k2eR;
  k2eps(p.k0dx, p.epsL, &k2, &k2eL);
  k2eps(p.k0dx, p.epsR, &k2, &k2eR);
  ChanInfo ci;
  if ((st = run_channels(h, p.tr, k2eL, k2eR, true, &ci))) return st;
  Request r;
  if ((st = resolve_request(req, ci, &r))) return st;
  *n_out = (int64_t)(r.out[0].size() + r.out[1].size());
  *n_in = (int64_t)(r.in[0].size() + r.in[1].size());
  return RGF_OK;
}

// Permittivity gradient request of smatrix(): g[m + n*N] = sum_ab D_ab dS_ab / d eps[m, n]
// for the weights D (n_out x n_in, column-major, leading dimension ldD, in the
// row/column order of S); D and g are device pointers when S is.
//
// The same backward pass also yields the fields inside the structure: with
// `psi`, psi[m + n*N + b*N*L] = (G_{n, ends} B)_{m b}, the response at site m
// of slice n to input channel b (the columns of S), written as each Psi_j
// is formed.  D == nullptr: fields only (no gradient).
struct GradReq {
  const rgf_cplx* D;
  int64_t ldD;
  rgf_cplx* g;
  int64_t checkpoint;  // slices per recomputed segment (<= 0: ceil(sqrt(L)))
  rgf_cplx* psi = nullptr;
};

// ---------------------------------------------------------------------------
// Batched call in one launch.  Every structure of the batch runs the usual
// pipeline on a host thread of its own (own handle, stream and workspace) up
// to its persistent sweep; there it hands the sweep's parameters to the
// coordinator and waits.  When every thread has either handed in its sweep or
// finished without one, the last to arrive runs all sweeps in ONE cooperative
// launch of k_persist_gang (gangs of CTAs sized to each structure from a work
// queue in device memory, largest first), and every thread goes on with its
// far lead and Fisher-Lee extraction.
// ---------------------------------------------------------------------------
// runs the gang launch over every sweep handed in (called by the last thread
// to arrive, with the lock held)
void gang_launch(GangBatch* g) {
  g->done = true;
  if (g->subs.empty()) return;
  std::vector<GangBatch::Sub>& v = g->subs;
  std::stable_sort(v.begin(), v.end(), [](const GangBatch::Sub& a, const GangBatch::Sub& b) { return a.cost > b.cost; });
  std::vector<PersistParams> params(v.size());
  std::vector<int> ctas(v.size());
  double est_s = 0.0;
  for (size_t i = 0; i < v.size(); i++) {
    params[i] = v[i].p;
    ctas[i] = v[i].ctas;
    est_s += v[i].cost;
  }
  // the launch's parameters live in one constant-memory array per device:
  // gang launches of the process do not overlap
  static std::mutex launch_mu;
  std::lock_guard<std::mutex> launch_lock(launch_mu);
  cudaError_t e = cudaSetDevice(g->device);
  int* d_ctas = nullptr;
  GangState* d_state = nullptr;
  if (e == cudaSuccess) e = cudaMallocAsync(&d_ctas, sizeof(int) * ctas.size(), g->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_state, sizeof(GangState), g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_ctas, ctas.data(), sizeof(int) * ctas.size(), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_state, 0, sizeof(GangState), g->stream);
  int clk_khz = 2000000;
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, g->device);
  // a free CTA may wait for a whole structure to finish: bound the scheduler's
  // waits by three times the batch's sequential estimate, at least 30 s
  const double sched_s = std::max(30.0, 3.0 * est_s);
  const long long sched_cycles = (long long)(sched_s * 1e3 * clk_khz);
  if (e == cudaSuccess)
    e = launch_persist_gang(params.data(), d_ctas, (int)ctas.size(), d_state, g->sms, sched_cycles, 96, 96,
                            g->stream);
  int abort_word = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&abort_word, &d_state->abort, sizeof(int), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (d_ctas) cudaFreeAsync(d_ctas, g->stream);
  if (d_state) cudaFreeAsync(d_state, g->stream);
  cudaStreamSynchronize(g->stream);
  g->launches++;
  if (e == cudaSuccess && abort_word) {
    // the scheduler gave up: no sweep of this launch can be trusted; every
    // structure raises its own timeout flag so that its call fails
    for (const GangBatch::Sub& sb : v) {
      const int bits = kStatusTimeout;
      cudaMemcpy(sb.p.abort, &bits, sizeof(int), cudaMemcpyHostToDevice);
      cudaMemcpy(sb.p.status, &bits, sizeof(int), cudaMemcpyHostToDevice);
    }
  }
  if (e != cudaSuccess) cudaGetLastError();
  g->result = e;
}

void gang_arrive_locked(GangBatch* g) {
  if (--g->pending == 0) {
    gang_launch(g);
    g->cv.notify_all();
  }
}

// a worker's sweep: wait until the gang launch has run it
cudaError_t gang_run(GangBatch* g, const PersistParams& pp, int BM, int ctas) {
  std::unique_lock<std::mutex> lock(g->mu);
  // cost estimate (seconds) for the queue order and the scheduler's bound:
  // steps x ~25 us per step on 96 x 96 tiles
  g->subs.push_back({pp, ctas, (double)pp.L * pp.NB * 25e-6});
  (void)BM;
  gang_arrive_locked(g);
  g->cv.wait(lock, [&] { return g->done; });
  return g->result;
}

// a worker that finished without handing in a sweep
void gang_leave(GangBatch* g) {
  std::lock_guard<std::mutex> lock(g->mu);
  gang_arrive_locked(g);
}

// Largest per-slice probe residual max|G_n M_n v - v| (|v_i| = 1) accepted
// from the persistent engine, whose pivot search stays inside each 32 x 32
// pivot block: above it (or on a zero / non-finite pivot) the S-matrix is
// recomputed by the per-step engine with partial pivoting over the whole
// column.  Above kProbeIllcond even that result is reported as
// RGF_ERR_ILLCOND (MATLAB's inv would warn "close to singular").
constexpr double kProbeRetry = 1e-10;
constexpr double kProbeIllcond = 1e-8;
// internal status of smatrix_run: recompute with engine 1
constexpr rgf_status kRetryWholeColumn = static_cast<rgf_status>(1000);

// Segment sweep of an L-split S-matrix: the slices [0, cut) swept from the
// left lead (side 0) or [cut, L) from the right lead (side 1), carrying only
// that side's requested channels, with no far lead; `state` receives W after
// the segment's last slice, [[g, X], [Z, Y]] row-major with leading dimension
// N + n_in(side) (g the lead-connected Green's function of the segment's last
// slice, X = g..g0 B, Z = C g0..g, Y = C G B at the lead).
struct SegReq {
  int side;
  int64_t cut;
  rgf_cplx* state;
};

rgf_status smatrix_run(rgf_handle h, const Problem& p, const rgf_request* req, const rgf_options* opt, rgf_cplx* S,
                       int64_t ldS, rgf_channels* ch, const GradReq* gr, int engine, const SegReq* seg) {
  rgf_status st;
  h->launches = 0;
  h->probe = 0.0;
  h->engine_used = engine;
  if ((st = validate_problem(p, req))) return st;
  const bool want_mixed = opt && opt->precision == RGF_TF32X3;
  if (opt && opt->precision != RGF_FP64 && !want_mixed) {
    set_error("unsupported precision form (rgf_precision: RGF_FP64 or RGF_TF32X3)");
    return RGF_ERR_ARG;
  }
  if (want_mixed && (gr || seg || h->gang || h->arena)) {
    set_error("the split-precision form (RGF_TF32X3) computes S-matrices only: gradients, fields, segments, the "
              "one-launch batch and rgf_smatrix_2d_noalloc take RGF_FP64");
    return RGF_ERR_ARG;
  }
  const bool S_dev = opt && opt->S_on_device;
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  const Transverse& tr = p.tr;
  const int64_t N = tr.N, L = p.L;
  double2 k2, k2eL, k2eR;
  k2eps(p.k0dx, p.epsL, &k2, &k2eL);
  k2eps(p.k0dx, p.epsR, &k2, &k2eR);

  // (1) channels, request resolution (cal_smatrix_RGF.m:98-178)
  ChanInfo ci;
  if ((st = run_channels(h, tr, k2eL, k2eR, true, &ci))) return st;
  Request rq;
  if ((st = resolve_request(req, ci, &rq))) return st;
  const int noL = (int)rq.out[0].size(), noR = (int)rq.out[1].size();
  const int niL = (int)rq.in[0].size(), niR = (int)rq.in[1].size();
  const int n_out = noL + noR, n_in = niL + niR;
  if (gr && gr->psi && n_in > 0 && n_out == 0) {
    set_error("the fields are computed with S: request at least one output channel");
    return RGF_ERR_ARG;
  }
  if (n_out == 0 || n_in == 0) {  // :181-184
    if (gr && gr->D && L > 0) {  // S is empty: so is its derivative
      if (S_dev) RGF_CUDA_TRY(cudaMemsetAsync(gr->g, 0, sizeof(rgf_cplx) * N * L, h->stream));
      else memset(gr->g, 0, sizeof(rgf_cplx) * N * L);
    }
    return copy_channels_out(h, tr, ci, ch);
  }
  if (gr && gr->D && gr->ldD < n_out) {
    set_error("ldD must be >= the number of requested output channels");
    return RGF_ERR_ARG;
  }
  if (seg && (seg->cut <= 0 || seg->cut >= L || !seg->state || (seg->side != 0 && seg->side != 1))) {
    set_error("segment: need 0 < cut < L (each part at least one slice), side 0 or 1 and a state buffer");
    return RGF_ERR_ARG;
  }
  if (!S && !seg) {
    set_error("S must not be NULL");
    return RGF_ERR_ARG;
  }
  if (!seg && ldS < n_out) {
    set_error("ldS must be >= the number of requested output channels");
    return RGF_ERR_ARG;
  }

  // (2) recursion direction: right-to-left when nothing enters from the
  // right (cal_smatrix_RGF.m:217-236), left-to-right otherwise (:237-280)
  // (a segment sweep goes from its own lead and carries that side only)
  const bool mirror = seg ? seg->side == 1 : (niR == 0);
  const int s = mirror ? 1 : 0, e = 1 - s;
  static const std::vector<int> kNone;
  const std::vector<int>& in_s = rq.in[s];
  const std::vector<int>& out_s = rq.out[s];
  const std::vector<int>& in_e = seg ? kNone : rq.in[e];
  const std::vector<int>& out_e = seg ? kNone : rq.out[e];
  // slices swept (in recursion order 0 .. Ls-1; slice k is physical slice
  // mirror ? L-1-k : k)
  const int64_t Ls = seg ? (seg->side == 0 ? seg->cut : L - seg->cut) : L;
  const int ni_s = (int)in_s.size(), no_s = (int)out_s.size(), ni_e = (int)in_e.size(), no_e = (int)out_e.size();
  const int64_t R = N + no_s + no_e, C = N + ni_s + ni_e;
  // persistent engine: active R_p x C_p with the probe pair at an even column
  const int64_t Rp = N + no_s, pc1 = (N + ni_s + 1) & ~(int64_t)1, Cp = pc1 + 2;
  const int64_t ldm = (std::max(C, Cp) + 1) & ~(int64_t)1;
  const int kSwW = sweep_block_width();

  // (3) workspace
  if ((st = ensure(h, h->phi, sizeof(double2) * N * N))) return st;
  if ((st = ensure(h, h->tmp, sizeof(double2) * N * N))) return st;
  if ((st = ensure(h, h->g0s, sizeof(double2) * N * N))) return st;
  if (!ci.same && (st = ensure(h, h->g0e, sizeof(double2) * N * N))) return st;
  if ((st = ensure(h, h->st_col, sizeof(int) * N * kMaxStencil))) return st;
  if ((st = ensure(h, h->st_val, sizeof(double2) * N * kMaxStencil))) return st;
  if ((st = ensure(h, h->aug, sizeof(double2) * R * ldm))) return st;
  if ((st = ensure(h, h->pc, sizeof(double2) * std::max(R, Cp) * kSwW))) return st;
  if ((st = ensure(h, h->u, sizeof(double2) * kSwW * ldm))) return st;
  if ((st = ensure(h, h->status, sizeof(int)))) return st;
  if (!S_dev && (st = ensure(h, h->sdev, sizeof(double2) * (int64_t)n_out * n_in))) return st;
  // index arrays: in_s, out_s, in_e, out_e, row_of, col_of, delta pairs
  std::vector<int> row_of(n_out), col_of(n_in), pairs;
  for (int o = 0; o < n_out; o++) {
    // reference row order [out_L; out_R]; augmented order [out_s; out_e]
    bool isL = o < noL;
    int k = isL ? o : o - noL;
    bool is_s = (isL && s == 0) || (!isL && s == 1);
    row_of[o] = is_s ? k : no_s + k;
  }
  for (int i = 0; i < n_in; i++) {
    bool isL = i < niL;
    int k = isL ? i : i - niL;
    bool is_s = (isL && s == 0) || (!isL && s == 1);
    col_of[i] = is_s ? k : ni_s + k;
  }
  intersect_pairs(rq.out[0], rq.in[0], 0, 0, &pairs);        // cal_smatrix_RGF.m:286
  intersect_pairs(rq.out[1], rq.in[1], noL, niL, &pairs);    // :287
  const int npairs = (int)pairs.size() / 2;
  std::vector<int> idx;
  auto push = [&](const std::vector<int>& v) {
    size_t o = idx.size();
    idx.insert(idx.end(), v.begin(), v.end());
    return o;
  };
  size_t o_in_s = push(in_s), o_out_s = push(out_s), o_in_e = push(in_e), o_out_e = push(out_e);
  size_t o_row = push(row_of), o_col = push(col_of), o_pairs = push(pairs);
  // S order [in_L; in_R] / [out_L; out_R] channel lists (split-precision form)
  std::vector<int> in_lr(rq.in[0]), out_lr(rq.out[0]);
  in_lr.insert(in_lr.end(), rq.in[1].begin(), rq.in[1].end());
  out_lr.insert(out_lr.end(), rq.out[1].begin(), rq.out[1].end());
  size_t o_in_lr = push(in_lr), o_out_lr = push(out_lr);
  if ((st = ensure(h, h->idx, sizeof(int) * (idx.size() + 1)))) return st;
  int* idx_d = as<int>(h->idx);
  RGF_CUDA_TRY(cudaMemcpyAsync(idx_d, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, h->stream));
  int* status = as<int>(h->status);
  RGF_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), h->stream));

  // (4) epsilon on the device, checked for NaN/Inf
  const double2* eps_d = nullptr;
  if (L > 0) {
    if (p.eps_dev) {
      eps_d = reinterpret_cast<const double2*>(p.eps);
    } else {
      if ((st = ensure(h, h->eps, sizeof(double2) * N * L))) return st;
      RGF_CUDA_TRY(cudaMemcpyAsync(h->eps.p, p.eps, sizeof(double2) * N * L, cudaMemcpyHostToDevice, h->stream));
      eps_d = as<double2>(h->eps);
    }
    launch_check_finite(eps_d, N * L, status, h->stream);
    h->launches++;
  }

  // (5) transverse profiles, slice stencil, lead surface Green's functions
  //     G0 = phi diag(exp(1i kx)) phi'  (cal_smatrix_RGF.m:187-209)
  double2* phi = as<double2>(h->phi);
  launch_phi(tr, as<double>(h->k0), as<double>(h->k1), phi, N, h->stream);
  launch_stencil(tr, as<int>(h->st_col), as<double2>(h->st_val), h->stream);
  h->launches += 2;
  const SideDev& sd_s = ci.side[s];
  const SideDev& sd_e = ci.side[e];
  double2* g0s = as<double2>(h->g0s);
  double2* g0e = ci.same ? g0s : as<double2>(h->g0e);
  launch_scale_cols(phi, N, sd_s.lam, as<double2>(h->tmp), N, N, N, h->stream);
  launch_zgemm(N, N, N, cmk(1.0, 0.0), ZOp{as<double2>(h->tmp), N, 0}, ZOp{phi, N, 2}, cmk(0.0, 0.0), g0s, N,
               h->stream);
  h->launches += 2;
  if (!ci.same) {
    launch_scale_cols(phi, N, sd_e.lam, as<double2>(h->tmp), N, N, N, h->stream);
    launch_zgemm(N, N, N, cmk(1.0, 0.0), ZOp{as<double2>(h->tmp), N, 0}, ZOp{phi, N, 2}, cmk(0.0, 0.0), g0e, N,
                 h->stream);
    h->launches += 2;
  }
  if ((st = check_launch())) return st;

  // (5b) the split-precision form: low-precision factorization + FP64
  //      refinement of the whole solve; S written here unless the
  //      refinement does not converge, in which case the FP64 form below runs
  if (want_mixed && L > 0) {
    MixedProblem mp;
    mp.N = N;
    mp.L = L;
    mp.niL = niL;
    mp.niR = niR;
    mp.noL = noL;
    mp.noR = noR;
    mp.phi = phi;
    for (int q = 0; q < 2; q++) {
      mp.prop[q] = ci.side[q].prop;
      mp.sqrtmu[q] = ci.side[q].sqrtmu;
    }
    mp.in_idx = idx_d + o_in_lr;
    mp.out_idx = idx_d + o_out_lr;
    mp.pairs = idx_d + o_pairs;
    mp.npairs = npairs;
    mp.G0[0] = s == 0 ? g0s : g0e;
    mp.G0[1] = s == 0 ? g0e : g0s;
    mp.st_col = as<int>(h->st_col);
    mp.st_val = as<double2>(h->st_val);
    mp.k2 = k2;
    mp.eps = eps_d;
    double2* Sd = S_dev ? reinterpret_cast<double2*>(S) : as<double2>(h->sdev);
    mp.S = Sd;
    mp.ldS = S_dev ? ldS : n_out;
    MixedAlloc alloc = [&](int slot, size_t bytes, void** pp) -> rgf_status {
      rgf_status e2 = ensure(h, h->mx[slot], bytes);
      *pp = h->mx[slot].p;
      return e2;
    };
    h->mx_stats = MixedStats();
    st = smatrix_mixed(mp, alloc, h->stream, &h->mx_stats, &h->launches);
    if (st == RGF_OK) {
      if (!S_dev)
        RGF_CUDA_TRY(cudaMemcpy2DAsync(S, sizeof(rgf_cplx) * ldS, Sd, sizeof(double2) * n_out,
                                       sizeof(double2) * n_out, n_in, cudaMemcpyDeviceToHost, h->stream));
      int hstatus = 0;
      RGF_CUDA_TRY(cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
      if (hstatus & kStatusNonfinite) {
        set_error("syst.epsilon contains NaN or Inf");
        return RGF_ERR_NONFINITE;
      }
      h->mx_form = RGF_TF32X3;
      return copy_channels_out(h, tr, ci, ch);
    }
    if (st == RGF_ERR_OOM) {
      // the factor store does not fit: give its buffers back and take the
      // FP64 form, which needs a small fraction of the memory
      cudaGetLastError();
      for (DevBuf& b : h->mx) {
        if (b.p) cudaFreeAsync(b.p, h->stream);
        b.p = nullptr;
        b.bytes = 0;
      }
    } else if (st != kMixedNotConverged) {
      return st;
    }
    h->mx_fallback = 1;  // S from the FP64 form
  }

  // (6) initial augmented matrix
  double2* M = as<double2>(h->aug);
  const int* st_col = as<int>(h->st_col);
  const double2* st_val = as<double2>(h->st_val);
  const double2 eps_e = d2(e == 0 ? p.epsL : p.epsR);
  launch_fill_init(M, ldm, N, phi, N, sd_s.prop, sd_s.lam, sd_s.sqrtmu, idx_d + o_in_s, ni_s, idx_d + o_out_s,
                   no_s, h->stream);
  h->launches++;
  auto slice_eps = [&](int64_t k) {  // k-th slice in recursion order
    int64_t n = mirror ? (L - 1 - k) : k;
    return eps_d + n * N;
  };
  auto attach = [&](bool first) {
    // top-left: A0 - k0dx^2 eps_e - G0_e - G ; Z rows negated; B_e / C_e blocks
    launch_assemble(M, ldm, N, first ? N : N + no_s, first ? g0s : M, first ? N : ldm, g0e, N, st_col, st_val,
                    k2, nullptr, eps_e, h->stream);
    launch_fill_attach(M, ldm, N, ni_s, no_s, phi, N, sd_e.prop, sd_e.sqrtmu, idx_d + o_in_e, ni_e,
                       idx_d + o_out_e, no_e, h->stream);
    h->launches += 2;
  };
  if (Ls > 0) {
    launch_assemble(M, ldm, N, N, g0s, N, nullptr, 0, st_col, st_val, k2, slice_eps(0), cmk(0, 0), h->stream);
    h->launches++;
  } else {
    attach(true);
  }

  // (7) slices (cal_smatrix_RGF.m:263-269), then the far lead (:272-275)
  const int prof_every = (opt && opt->profile > 0) ? opt->profile : 0;
  size_t ev_used = 0;
  double prof_flops = 0.0;
  // One sweep (per-step engine) of the active Ract x Cact matrix.  Per pivot
  // block: the rows of the whole remaining column are pivoted into place
  // (partial pivoting as in LAPACK zgetrf), the block is inverted and the
  // rank-32 update applied; at the end the column exchanges are undone.
  if ((st = ensure(h, h->gepp, gepp_scratch_bytes(N)))) return st;
  auto sweep = [&](int64_t Ract, int64_t Cact, bool timed) -> rgf_status {
    for (int64_t j0 = 0; j0 < N; j0 += kSwW) {
      int jn = (int)std::min<int64_t>(kSwW, N - j0);
      launch_gepp_step(M, ldm, N, Cact, j0, jn, h->gepp.p, status, h->stream);
      h->launches += 2;
      launch_sweep_panel(M, ldm, Ract, Cact, j0, jn, as<double2>(h->pc), as<double2>(h->u), ldm, status,
                         h->stream);
      if (timed) {
        while (h->ev.size() < ev_used + 2) {
          cudaEvent_t ev;
          RGF_CUDA_TRY(cudaEventCreate(&ev));
          h->ev.push_back(ev);
        }
        RGF_CUDA_TRY(cudaEventRecord(h->ev[ev_used], h->stream));
      }
      launch_sweep_update(M, ldm, Ract, Cact, j0, jn, as<double2>(h->pc), as<double2>(h->u), ldm, h->stream);
      if (timed) {
        RGF_CUDA_TRY(cudaEventRecord(h->ev[ev_used + 1], h->stream));
        ev_used += 2;
        prof_flops += 8.0 * (double)Ract * (double)Cact * (double)jn;
      }
      h->launches += 2;
    }
    RGF_CUDA_TRY(launch_gepp_unpermute(M, ldm, Ract, N, h->gepp.p, h->stream));
    h->launches += 2;
    return RGF_OK;
  };
  int BMp = 0, BNp = 0;
  auto choose_tile = [&]() {
    // batched call in one launch: the largest tile that fits (fewest SMs per structure)
    if (h->gang) return persist_choose_tile(Rp, Cp, h->sms, &BMp, &BNp, true);
    for (size_t q = 0; q < h->tile_rmax.size(); q++) {
      if (Rp > h->tile_rmax[q]) continue;
      const int t = h->tile_bm[q];
      if (((Rp + t - 1) / t) * ((Cp + t - 1) / t) + kPersistExtraCtas <= h->sms) {
        BMp = BNp = t;
        return true;
      }
      break;
    }
    return persist_choose_tile(Rp, Cp, h->sms, &BMp, &BNp, h->sm_budget != nullptr);
  };
  bool use_persist = L > 0 && engine == 0 && choose_tile();
  bool ran_persist = false;
  // per-slice probe residual (both engines)
  unsigned long long* probe_d = nullptr;
  h->prof_kernel = sweep_update_kernel_name();
  if (L > 0) {
    if ((st = ensure(h, h->xprobe, sizeof(unsigned long long)))) return st;
    probe_d = as<unsigned long long>(h->xprobe);
    RGF_CUDA_TRY(cudaMemsetAsync(probe_d, 0, sizeof(unsigned long long), h->stream));
  }
  // Sweeps the slices [k_lo, k_hi) of the recursion order.  On entry M holds
  // the assembled matrix of slice k_lo, on return W after slice k_hi - 1 (not
  // assembled).  With `snap`, W after every slice k with
  // (k - k_lo) % snap_mod == snap_mod - 1 is also copied to
  // snap + ((k - k_lo) / snap_mod) * Rp * ldm.
  auto run_slices = [&](int64_t k_lo, int64_t k_hi, double2* snap, int snap_mod) -> rgf_status {
    const int64_t nsl = k_hi - k_lo;
    if (use_persist) {
      const int TR = (int)((Rp + BMp - 1) / BMp), TC = (int)((Cp + BNp - 1) / BNp);
      const int nflags = persist_flag_words(TR, TC), ncons = persist_cons_words(TR, TC);
      if ((st = ensure(h, h->xpc, sizeof(double2) * 2 * TR * BMp * 32))) return st;
      if ((st = ensure(h, h->xrow, sizeof(double2) * 4 * TC * 32 * BNp))) return st;  // rowbuf, prebuf
      if ((st = ensure(h, h->xt, sizeof(double2) * 11 * 32 * 32))) return st;  // tbuf[2], djjbuf, srvbuf[2][2], ybuf[2][2]
      if ((st = ensure(h, h->xu, sizeof(double2) * 2 * TC * 32 * BNp))) return st;
      if ((st = ensure(h, h->xsync, sizeof(int) * (nflags + ncons + 4)))) return st;
      int* flags = as<int>(h->xsync);
      RGF_CUDA_TRY(cudaMemsetAsync(flags, 0xFF, sizeof(int) * nflags, h->stream));
      RGF_CUDA_TRY(cudaMemsetAsync(flags + nflags, 0, sizeof(int) * (ncons + 4), h->stream));
      launch_probe_init(M, ldm, N, Rp, pc1, h->stream);
      h->launches++;
      PersistParams pp;
      pp.N = (int)N;
      pp.R = (int)Rp;
      pp.C = (int)Cp;
      pp.TR = TR;
      pp.TC = TC;
      pp.NB = (int)((N + kSwW - 1) / kSwW);
      pp.L = (int)nsl;
      pp.M = M;
      pp.ldm = ldm;
      pp.eps = eps_d;
      pp.eps_first = mirror ? L - 1 - k_lo : k_lo;
      pp.eps_step = mirror ? -1 : 1;
      pp.k2 = k2;
      pp.st_col = st_col;
      pp.st_val = st_val;
      pp.pc1 = (int)pc1;
      pp.pcbuf = as<double2>(h->xpc);
      pp.rowbuf = as<double2>(h->xrow);
      pp.prebuf = as<double2>(h->xrow) + (size_t)2 * TC * 32 * BNp;
      pp.tbuf = as<double2>(h->xt);
      pp.djjbuf = as<double2>(h->xt) + 2 * 32 * 32;
      pp.srvbuf = as<double2>(h->xt) + 3 * 32 * 32;
      pp.ybuf = as<double2>(h->xt) + 7 * 32 * 32;
      pp.ubuf = as<double2>(h->xu);
      pp.flags = flags;
      pp.cons = flags + nflags;
      pp.abort = flags + nflags + ncons;
      pp.snap = snap;
      pp.snap_mod = snap ? snap_mod : 1;
      pp.snap_ld = Rp * ldm;
      pp.status = status;
      pp.probe_max = probe_d;
      int clk_khz = 2000000;
      cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, h->device);
      // bound of every device-side wait: ~4 s, or RGF_WAIT_TIMEOUT_MS
      const char* tmo_env = getenv("RGF_WAIT_TIMEOUT_MS");
      const double tmo_ms = (tmo_env && atof(tmo_env) > 0) ? atof(tmo_env) : 4000.0;
      pp.timeout_cycles = (long long)(clk_khz * tmo_ms);
      // RGF_TEST_WITHHOLD_T=1 (failure-detection tests): the T-server never
      // releases its T flag, so every dependent wait runs out
      const char* wh_env = getenv("RGF_TEST_WITHHOLD_T");
      pp.withhold_t = (wh_env && atoi(wh_env) == 1) ? 1 : 0;
      pp.trace = nullptr;  // per-step event timestamps: a development aid, off in the library
      pp.trace_steps = 0;
      const bool timed = prof_every > 0;
      if (timed) {
        while (h->ev.size() < ev_used + 2) {
          cudaEvent_t ev;
          RGF_CUDA_TRY(cudaEventCreate(&ev));
          h->ev.push_back(ev);
        }
        RGF_CUDA_TRY(cudaEventRecord(h->ev[ev_used], h->stream));
      }
      // in a batch, hold SMs for the whole cooperative grid while it runs, so
      // that the grids of concurrent pipelines always fit on the GPU together
      const int need = TR * TC + kPersistExtraCtas;
      if (h->sm_budget) {
        for (;;) {
          int cur = h->sm_budget->load();
          if (cur >= need && h->sm_budget->compare_exchange_weak(cur, cur - need)) break;
          std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
      }
      cudaError_t e;
      if (h->gang && !h->gang_submitted && BMp == 96) {
        // one launch for the whole batch (96 x 96 tiles): hand the sweep to
        // the gang launch and wait until it has run; a structure that needs
        // smaller tiles sweeps on its own before the gang launch
        RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->gang_submitted = true;
        e = gang_run(h->gang, pp, BMp, need);
      } else {
        e = launch_persist(pp, BMp, BNp, h->stream);
      }
      if (h->sm_budget) {
        const cudaError_t se = cudaStreamSynchronize(h->stream);
        h->sm_budget->fetch_add(need);
        RGF_CUDA_TRY(se);
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        use_persist = false;  // e.g. the cooperative launch does not fit: per-step engine below
      } else {
        h->launches++;
        ran_persist = true;
        if (timed) {
          RGF_CUDA_TRY(cudaEventRecord(h->ev[ev_used + 1], h->stream));
          ev_used += 2;
          for (int64_t j0 = 0; j0 < N; j0 += kSwW)
            prof_flops +=
                (double)nsl * 8.0 * (double)Rp * (double)(N + ni_s) * (double)std::min<int64_t>(kSwW, N - j0);
        }
        char nm[64];
        snprintf(nm, sizeof(nm), "k_persist<%d,%d> (FP64 DMMA sweep, all slices)", BMp, BNp);
        h->prof_kernel = nm;
        return RGF_OK;
      }
    }
    // per-step engine: the probe pair rides along as in the persistent one
    launch_probe_init(M, ldm, N, Rp, pc1, h->stream);
    h->launches++;
    for (int64_t k = k_lo; k < k_hi; k++) {
      if ((st = sweep(N + no_s, Cp, prof_every && (k % prof_every) == 0))) return st;
      launch_probe_check(M, ldm, N, pc1, probe_d, h->stream);
      h->launches++;
      if (snap && (k - k_lo) % snap_mod == snap_mod - 1)
        RGF_CUDA_TRY(cudaMemcpyAsync(snap + ((k - k_lo) / snap_mod) * Rp * ldm, M, sizeof(double2) * Rp * ldm,
                                     cudaMemcpyDeviceToDevice, h->stream));
      if (k + 1 < k_hi) {
        launch_assemble(M, ldm, N, N + no_s, M, ldm, nullptr, 0, st_col, st_val, k2, slice_eps(k + 1), cmk(0, 0),
                        h->stream);
        launch_probe_init(M, ldm, N, Rp, pc1, h->stream);
        h->launches += 2;
      }
      if (((k + 1) & 63) == 0 && (st = check_launch())) return st;
    }
    return RGF_OK;
  };
  // gradient: checkpoints of the forward sweep (W after every K-th slice) and
  // the assembled first slice
  // checkpoint interval: the caller's, else every slice when those snapshots
  // take at most 2 GiB (no recomputation), else ceil(sqrt(L))
  const int64_t gK =
      !gr ? 0
          : gr->checkpoint > 0 ? std::min<int64_t>(gr->checkpoint, std::max<int64_t>(L, 1))
          : (double)L * Rp * ldm * sizeof(double2) <= 2.0 * (1 << 30)
              ? 1
              : std::max<int64_t>(1, (int64_t)ceil(sqrt((double)L)));
  if (gr && L > 0) {
    if ((st = ensure(h, h->gck, sizeof(double2) * Rp * ldm * std::max<int64_t>(1, L / gK)))) return st;
    if ((st = ensure(h, h->gm0, sizeof(double2) * Rp * ldm))) return st;
    RGF_CUDA_TRY(cudaMemcpyAsync(h->gm0.p, M, sizeof(double2) * Rp * ldm, cudaMemcpyDeviceToDevice, h->stream));
  }
  if (Ls > 0) {
    if ((st = run_slices(0, Ls, gr ? as<double2>(h->gck) : nullptr, (int)gK))) return st;
    if (!seg) attach(false);
  }
  if (seg) {
    // the segment's state: W after its last slice (probe columns excluded)
    const int64_t Cs = N + ni_s;
    RGF_CUDA_TRY(cudaMemcpy2DAsync(seg->state, sizeof(rgf_cplx) * Cs, M, sizeof(double2) * ldm,
                                   sizeof(double2) * Cs, Rp, S_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                   h->stream));
  } else {
    if ((st = sweep(R, C, false))) return st;

    // (8) Fisher-Lee (cal_smatrix_RGF.m:279-289)
    double2* Sd = S_dev ? reinterpret_cast<double2*>(S) : as<double2>(h->sdev);
    const int64_t ldSd = S_dev ? ldS : n_out;
    launch_extract(M, ldm, N, idx_d + o_row, n_out, idx_d + o_col, n_in, Sd, ldSd, idx_d + o_pairs, npairs,
                   h->stream);
    h->launches += 1 + (npairs > 0 ? 1 : 0);
    if ((st = check_launch())) return st;
    if (!S_dev) {
      RGF_CUDA_TRY(cudaMemcpy2DAsync(S, sizeof(rgf_cplx) * ldS, Sd, sizeof(double2) * n_out,
                                     sizeof(double2) * n_out, n_in, cudaMemcpyDeviceToHost, h->stream));
    }
  }
  // (9) permittivity gradient: the backward recursions
  //     Psi_j = [X_j, 0] + g_j Psi_{j+1},  Phi_j = [Z_j; 0] + Phi_{j+1} g_j
  //     dS_ab/d eps(m, slice j) = -2i k0dx^2 Phi_j[a][m] Psi_j[m][b]
  //     over the start-connected blocks g_j and carriers X_j, Z_j of the
  //     sweep, segment by segment from the last: each segment's slices are
  //     recomputed from its checkpoint with a snapshot after every slice.
  if (gr && L > 0) {
    const int64_t nI = n_in, nO = n_out;
    const bool want_g = gr->D != nullptr, want_f = gr->psi != nullptr;
    std::vector<rgf_cplx> Du((size_t)nO * nI), Da((size_t)nO * nI);
    if (!want_g) {
      // fields only: no weights
    } else if (S_dev) {
      RGF_CUDA_TRY(cudaMemcpy2DAsync(Du.data(), sizeof(rgf_cplx) * nO, gr->D, sizeof(rgf_cplx) * gr->ldD,
                                     sizeof(rgf_cplx) * nO, nI, cudaMemcpyDeviceToHost, h->stream));
      RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    } else {
      for (int64_t i = 0; i < nI; i++)
        for (int64_t o = 0; o < nO; o++) Du[o + i * nO] = gr->D[o + i * gr->ldD];
    }
    for (int64_t i = 0; i < nI; i++)
      for (int64_t o = 0; o < nO; o++) Da[(size_t)row_of[o] * nI + col_of[i]] = Du[o + i * nO];
    if ((st = ensure(h, h->gd, sizeof(double2) * nO * nI))) return st;
    if ((st = ensure(h, h->gpsi, sizeof(double2) * 2 * N * nI))) return st;
    if ((st = ensure(h, h->gphi, sizeof(double2) * 2 * nO * N))) return st;
    if ((st = ensure(h, h->get, sizeof(double2) * nO * N))) return st;
    if (gK > 1 && (st = ensure(h, h->gseg, sizeof(double2) * gK * Rp * ldm))) return st;
    if (want_g && !S_dev && (st = ensure(h, h->gg, sizeof(double2) * N * L))) return st;
    if (want_f && !S_dev && (st = ensure(h, h->gf, sizeof(double2) * N * L * nI))) return st;
    double2* Dd = as<double2>(h->gd);
    if (want_g)
      RGF_CUDA_TRY(cudaMemcpyAsync(Dd, Da.data(), sizeof(double2) * nO * nI, cudaMemcpyHostToDevice, h->stream));
    double2* fout = !want_f ? nullptr : S_dev ? reinterpret_cast<double2*>(gr->psi) : as<double2>(h->gf);
    double2* psi[2] = {as<double2>(h->gpsi), as<double2>(h->gpsi) + N * nI};
    double2* phv[2] = {as<double2>(h->gphi), as<double2>(h->gphi) + nO * N};
    double2* Et = as<double2>(h->get);
    double2* seg = as<double2>(h->gseg);
    double2* gout = !want_g ? nullptr : S_dev ? reinterpret_cast<double2*>(gr->g) : as<double2>(h->gg);
    // Psi_{L+1} = W(0:N, N:N+n_in) and Phi_{L+1} = W(N:N+n_out, 0:N) after the far lead
    RGF_CUDA_TRY(cudaMemcpy2DAsync(psi[0], sizeof(double2) * nI, M + N, sizeof(double2) * ldm, sizeof(double2) * nI,
                                   N, cudaMemcpyDeviceToDevice, h->stream));
    RGF_CUDA_TRY(cudaMemcpy2DAsync(phv[0], sizeof(double2) * N, M + N * ldm, sizeof(double2) * ldm,
                                   sizeof(double2) * N, nO, cudaMemcpyDeviceToDevice, h->stream));
    const double2 coef = cmul(cmk(0.0, -2.0), k2);
    const double2 one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
    int cur = 0;
    const int64_t nseg = (L + gK - 1) / gK;
    for (int64_t sg = nseg - 1; sg >= 0; sg--) {
      const int64_t k_lo = sg * gK, k_hi = std::min(L, k_lo + gK);
      // with a snapshot of every slice (gK == 1) nothing is recomputed
      const double2* segW = gK == 1 ? as<double2>(h->gck) + k_lo * Rp * ldm : seg;
      if (gK > 1) {
        if (sg == 0) {
          RGF_CUDA_TRY(
              cudaMemcpyAsync(M, h->gm0.p, sizeof(double2) * Rp * ldm, cudaMemcpyDeviceToDevice, h->stream));
        } else {
          RGF_CUDA_TRY(cudaMemcpyAsync(M, as<double2>(h->gck) + (sg - 1) * Rp * ldm, sizeof(double2) * Rp * ldm,
                                       cudaMemcpyDeviceToDevice, h->stream));
          launch_assemble(M, ldm, N, N + no_s, M, ldm, nullptr, 0, st_col, st_val, k2, slice_eps(k_lo), cmk(0, 0),
                          h->stream);
          h->launches++;
        }
        if ((st = run_slices(k_lo, k_hi, seg, 1))) return st;
      }
      for (int64_t j = k_hi - 1; j >= k_lo; j--) {
        const double2* Wj = segW + (j - k_lo) * Rp * ldm;
        const int nx_ = cur ^ 1;
        const int64_t n_phys = mirror ? L - 1 - j : j;
        if (grad_step_fits((int)nI, (int)nO)) {
          // few channels: both recursions and the contraction in one launch
          launch_grad_step(Wj, ldm, N, (int)nI, (int)nO, ni_s, no_s, psi[cur], phv[cur], Dd, coef, psi[nx_], phv[nx_],
                           want_g ? gout + n_phys * N : nullptr, h->stream);
          h->launches++;
          if (want_f) {
            launch_store_field(psi[nx_], idx_d + o_col, N, (int)nI, fout + n_phys * N, N * L, h->stream);
            h->launches++;
          }
          cur = nx_;
          continue;
        }
        launch_zgemm_add(N, nI, N, ZOp{Wj, ldm, 0}, ZOp{psi[cur], nI, 0}, ZAdd{Wj + N, ldm, N, ni_s}, psi[nx_],
                         nI, h->stream);
        h->launches++;
        if (want_f) {
          launch_store_field(psi[nx_], idx_d + o_col, N, (int)nI, fout + n_phys * N, N * L, h->stream);
          h->launches++;
        }
        if (!want_g) {
          cur = nx_;
          continue;
        }
        launch_zgemm_add(nO, N, N, ZOp{phv[cur], N, 0}, ZOp{Wj, ldm, 0}, ZAdd{Wj + N * ldm, ldm, no_s, N},
                         phv[nx_], N, h->stream);
        if (nO * nI <= 1024) {
          launch_grad_fused(phv[nx_], psi[nx_], Dd, N, (int)nO, (int)nI, coef, gout + n_phys * N, h->stream);
          h->launches += 2;
        } else {
          launch_zgemm(nO, N, nI, one, ZOp{Dd, nI, 0}, ZOp{psi[nx_], nI, 1}, zero, Et, N, h->stream);
          launch_grad_slice(phv[nx_], Et, N, nO, coef, gout + n_phys * N, h->stream);
          h->launches += 3;
        }
        cur = nx_;
      }
      if ((st = check_launch())) return st;
    }
    if (want_g && !S_dev)
      RGF_CUDA_TRY(cudaMemcpyAsync(gr->g, gout, sizeof(double2) * N * L, cudaMemcpyDeviceToHost, h->stream));
    if (want_f && !S_dev)
      RGF_CUDA_TRY(cudaMemcpyAsync(gr->psi, fout, sizeof(double2) * N * L * nI, cudaMemcpyDeviceToHost, h->stream));
  } else if (gr) {
    // no slices: nothing depends on epsilon
  }

  int hstatus = 0;
  unsigned long long probe_bits = 0;
  RGF_CUDA_TRY(cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (probe_d)
    RGF_CUDA_TRY(cudaMemcpyAsync(&probe_bits, probe_d, sizeof(probe_bits), cudaMemcpyDeviceToHost, h->stream));
  RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
  memcpy(&h->probe, &probe_bits, sizeof(double));
  h->prof_n = (int64_t)(ev_used / 2);
  h->prof_ms = 0.0;
  h->prof_flops = prof_flops;
  for (size_t q = 0; q < ev_used; q += 2) {
    float ms = 0.f;
    RGF_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[q], h->ev[q + 1]));
    h->prof_ms += ms;
  }
  if (hstatus & kStatusNonfinite) {
    set_error("syst.epsilon contains NaN or Inf");
    return RGF_ERR_NONFINITE;
  }
  if (hstatus & kStatusTimeout) {  // before singular: what follows a timed-out sweep works on garbage
    set_error("a device-side wait timed out");
    return RGF_ERR_TIMEOUT;
  }
  // the persistent engine pivots inside each 32 x 32 block only: a zero or
  // non-finite pivot there, or a slice inverse whose probe residual is not
  // at round-off level, sends the whole call to the per-step engine
  if (ran_persist && ((hstatus & kStatusSingular) || !(h->probe <= kProbeRetry))) return kRetryWholeColumn;
  if (hstatus & kStatusSingular) {
    set_error("a slice matrix is singular (zero pivot under partial pivoting)");
    return RGF_ERR_SINGULAR;
  }
  if ((st = copy_channels_out(h, tr, ci, ch))) return st;
  if (!(h->probe <= kProbeIllcond)) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "a slice matrix is ill-conditioned: slice-inverse probe residual %.3g (> %.0e); S holds the result "
             "of partial pivoting, which may be inaccurate",
             h->probe, kProbeIllcond);
    set_error(msg);
    return RGF_ERR_ILLCOND;
  }
  return RGF_OK;
}

// smatrix_run with the engine of opt (default: persistent), recomputed by the
// per-step engine with whole-column pivoting when the persistent engine's
// in-block pivoting proves inadequate.
rgf_status smatrix(rgf_handle h, const Problem& p, const rgf_request* req, const rgf_options* opt, rgf_cplx* S,
                   int64_t ldS, rgf_channels* ch, const GradReq* gr = nullptr, const SegReq* seg = nullptr) {
  const int engine = (opt && opt->engine == 1) ? 1 : 0;
  h->fallback = 0;
  h->mx_form = RGF_FP64;
  h->mx_fallback = 0;
  rgf_status st = smatrix_run(h, p, req, opt, S, ldS, ch, gr, engine, seg);
  if (st == kRetryWholeColumn) {
    const double probe0 = h->probe;
    rgf_options o2 = opt ? *opt : rgf_options{};
    o2.precision = RGF_FP64;  // a split-precision attempt, if any, has already been made
    st = smatrix_run(h, p, req, &o2, S, ldS, ch, gr, 1, seg);
    h->fallback = 1;
    h->probe_first = probe0;
  }
  return st;
}

// Joins the two segment states of an L-split S-matrix (SegReq) across the
// cut by one Dyson step.  With the coupling -I between the left part's last
// slice b and the right part's first slice a = b + 1, and the states
// (g_L, X_L, Z_L, Y_L), (g_R, X_R, Z_R, Y_R), sweeping the pivot block
// P = I - g_R g_L of
//     [[ P,          g_R X_L,  X_R ],
//      [ -Z_L,       Y_L,      0   ],
//      [ -Z_R g_L,   Z_R X_L,  Y_R ]]
// leaves, in its corner, the four blocks C G B between the two lead surfaces:
//     C_L G_00 B_L = Y_L + Z_L (I - g_R g_L)^{-1} g_R X_L,
//     C_L G_0e B_R = Z_L (I - g_R g_L)^{-1} X_R,
//     C_R G_e0 B_L = Z_R X_L + Z_R g_L (I - g_R g_L)^{-1} g_R X_L,
//     C_R G_ee B_R = Y_R + Z_R g_L (I - g_R g_L)^{-1} X_R,
// (the Dyson equation for two coupled Green's functions; the same blocks the
// far-lead attachment of cal_smatrix_RGF.m:272-289 produces), from which S
// follows by the Fisher-Lee relation.  The sweep pivots over the whole
// column.
rgf_status segment_merge(rgf_handle h, const Problem& p, const rgf_request* req, const rgf_options* opt,
                         const rgf_cplx* stL, const rgf_cplx* stR, rgf_cplx* S, int64_t ldS) {
  rgf_status st;
  h->launches = 0;
  h->probe = 0.0;
  h->engine_used = 1;
  h->fallback = 0;
  if ((st = validate_problem(p, req))) return st;
  if (opt && opt->precision != RGF_FP64) {
    set_error("unsupported precision form");
    return RGF_ERR_ARG;
  }
  const bool S_dev = opt && opt->S_on_device;
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t N = p.tr.N;
  double2 k2, k2eL, k2eR;
  k2eps(p.k0dx, p.epsL, &k2, &k2eL);
  k2eps(p.k0dx, p.epsR, &k2, &k2eR);
  ChanInfo ci;
  if ((st = run_channels(h, p.tr, k2eL, k2eR, true, &ci))) return st;
  Request rq;
  if ((st = resolve_request(req, ci, &rq))) return st;
  const int noL = (int)rq.out[0].size(), noR = (int)rq.out[1].size();
  const int niL = (int)rq.in[0].size(), niR = (int)rq.in[1].size();
  const int n_out = noL + noR, n_in = niL + niR;
  if (n_out == 0 || n_in == 0) return RGF_OK;
  if (!S || !stL || !stR || ldS < n_out) {
    set_error("segment merge: S, both states and ldS >= n_out are needed");
    return RGF_ERR_ARG;
  }
  const int64_t CL = N + niL, CR = N + niR, RL = N + noL, RR = N + noR;
  const double2 *dL = reinterpret_cast<const double2*>(stL), *dR = reinterpret_cast<const double2*>(stR);
  if (!S_dev) {
    if ((st = ensure(h, h->segs, sizeof(double2) * (RL * CL + RR * CR)))) return st;
    RGF_CUDA_TRY(cudaMemcpyAsync(h->segs.p, stL, sizeof(double2) * RL * CL, cudaMemcpyHostToDevice, h->stream));
    RGF_CUDA_TRY(cudaMemcpyAsync(as<double2>(h->segs) + RL * CL, stR, sizeof(double2) * RR * CR,
                                 cudaMemcpyHostToDevice, h->stream));
    dL = as<double2>(h->segs);
    dR = dL + RL * CL;
  }
  const int kSwW = sweep_block_width();
  const int64_t R = N + n_out, C = N + n_in, ldm = (C + 1) & ~(int64_t)1;
  if ((st = ensure(h, h->aug, sizeof(double2) * R * ldm))) return st;
  if ((st = ensure(h, h->pc, sizeof(double2) * std::max(R, C) * kSwW))) return st;
  if ((st = ensure(h, h->u, sizeof(double2) * kSwW * ldm))) return st;
  if ((st = ensure(h, h->gepp, gepp_scratch_bytes(N)))) return st;
  if ((st = ensure(h, h->status, sizeof(int)))) return st;
  if (!S_dev && (st = ensure(h, h->sdev, sizeof(double2) * (int64_t)n_out * n_in))) return st;
  std::vector<int> idx;
  for (int o = 0; o < n_out; o++) idx.push_back(o);
  for (int i = 0; i < n_in; i++) idx.push_back(i);
  std::vector<int> pairs;
  intersect_pairs(rq.out[0], rq.in[0], 0, 0, &pairs);        // cal_smatrix_RGF.m:286
  intersect_pairs(rq.out[1], rq.in[1], noL, niL, &pairs);    // :287
  const size_t o_pairs = idx.size();
  idx.insert(idx.end(), pairs.begin(), pairs.end());
  if ((st = ensure(h, h->idx, sizeof(int) * (idx.size() + 1)))) return st;
  int* idx_d = as<int>(h->idx);
  RGF_CUDA_TRY(cudaMemcpyAsync(idx_d, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, h->stream));
  int* status = as<int>(h->status);
  RGF_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), h->stream));
  double2* M = as<double2>(h->aug);
  const double2 one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  const double2 *gL = dL, *XL = dL + N, *ZL = dL + N * CL, *YL = dL + N * CL + N;
  const double2 *gR = dR, *XR = dR + N, *ZR = dR + N * CR, *YR = dR + N * CR + N;
  launch_zgemm(N, N, N, mone, ZOp{gR, CR, 0}, ZOp{gL, CL, 0}, zero, M, ldm, h->stream);  // P = I - g_R g_L
  launch_add_identity(M, ldm, N, h->stream);
  if (niL) launch_zgemm(N, niL, N, one, ZOp{gR, CR, 0}, ZOp{XL, CL, 0}, zero, M + N, ldm, h->stream);
  launch_block_copy(M + N + niL, ldm, XR, CR, N, niR, 1.0, h->stream);
  launch_block_copy(M + N * ldm, ldm, ZL, CL, noL, N, -1.0, h->stream);
  if (noR) launch_zgemm(noR, N, N, mone, ZOp{ZR, CR, 0}, ZOp{gL, CL, 0}, zero, M + (N + noL) * ldm, ldm, h->stream);
  launch_block_copy(M + N * ldm + N, ldm, YL, CL, noL, niL, 1.0, h->stream);
  launch_block_copy(M + N * ldm + N + niL, ldm, nullptr, 0, noL, niR, 0.0, h->stream);
  if (noR && niL)
    launch_zgemm(noR, niL, N, one, ZOp{ZR, CR, 0}, ZOp{XL, CL, 0}, zero, M + (N + noL) * ldm + N, ldm, h->stream);
  launch_block_copy(M + (N + noL) * ldm + N + niL, ldm, YR, CR, noR, niR, 1.0, h->stream);
  h->launches += 9;
  for (int64_t j0 = 0; j0 < N; j0 += kSwW) {
    const int jn = (int)std::min<int64_t>(kSwW, N - j0);
    launch_gepp_step(M, ldm, N, C, j0, jn, h->gepp.p, status, h->stream);
    launch_sweep_panel(M, ldm, R, C, j0, jn, as<double2>(h->pc), as<double2>(h->u), ldm, status, h->stream);
    launch_sweep_update(M, ldm, R, C, j0, jn, as<double2>(h->pc), as<double2>(h->u), ldm, h->stream);
    h->launches += 4;
  }
  RGF_CUDA_TRY(launch_gepp_unpermute(M, ldm, R, N, h->gepp.p, h->stream));
  double2* Sd = S_dev ? reinterpret_cast<double2*>(S) : as<double2>(h->sdev);
  const int64_t ldSd = S_dev ? ldS : n_out;
  launch_extract(M, ldm, N, idx_d, n_out, idx_d + n_out, n_in, Sd, ldSd, idx_d + o_pairs, (int)pairs.size() / 2,
                 h->stream);
  h->launches += 4;
  if ((st = check_launch())) return st;
  if (!S_dev)
    RGF_CUDA_TRY(cudaMemcpy2DAsync(S, sizeof(rgf_cplx) * ldS, Sd, sizeof(double2) * n_out, sizeof(double2) * n_out,
                                   n_in, cudaMemcpyDeviceToHost, h->stream));
  int hstatus = 0;
  RGF_CUDA_TRY(cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (hstatus & kStatusSingular) {
    set_error("segment merge: the interface matrix I - g_R g_L is singular");
    return RGF_ERR_SINGULAR;
  }
  return RGF_OK;
}

Problem problem2d(const rgf_syst2d* s) {
  Problem p;
  p.tr.dim = 2;
  p.tr.n0 = s->ny;
  p.tr.n1 = 1;
  p.tr.N = s->ny;
  p.tr.bc = s->yBC;
  p.tr.ka0 = (s->yBC == RGF_BC_BLOCH) ? s->ka : 0.0;
  p.tr.ka1 = 0.0;
  p.L = s->nx;
  p.eps = s->epsilon;
  p.eps_dev = s->eps_on_device != 0;
  p.epsL = s->epsilon_L;
  p.epsR = s->epsilon_R;
  p.k0dx = s->k0dx;
  return p;
}

Problem problem3d(const rgf_syst3d* s) {
  Problem p;
  p.tr.dim = 3;
  p.tr.n0 = s->nx;
  p.tr.n1 = s->ny;
  p.tr.N = s->nx * s->ny;
  p.tr.bc = s->xyBC;
  p.tr.ka0 = (s->xyBC == RGF_BC_BLOCH) ? s->kxa : 0.0;
  p.tr.ka1 = (s->xyBC == RGF_BC_BLOCH) ? s->kya : 0.0;
  p.L = s->nz;
  p.eps = s->epsilon;
  p.eps_dev = s->eps_on_device != 0;
  p.epsL = s->epsilon_L;
  p.epsR = s->epsilon_R;
  p.k0dx = s->k0dx;
  return p;
}

rgf_status check_handle(rgf_handle h) {
  if (!h) {
    set_error("NULL handle");
    return RGF_ERR_ARG;
  }
  return RGF_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// static device scratch of rgf_smatrix_2d_noalloc
// ---------------------------------------------------------------------------
// Every GPU that loads this library holds this array until the process
// exits.  In host code the name only stands for the device symbol; its device
// address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[RGF_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of the scratch array in the current device's context.  It
// is looked up on every call (cudaGetSymbolAddress allocates nothing and is
// cheap), so a context the host application reset and recreated is seen.
// The first lookup on a device also loads this library's device code there.
rgf_status noalloc_scratch(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    set_error(std::string("rgf_smatrix_2d_noalloc: cudaGetSymbolAddress of the static scratch failed: ") +
              cudaGetErrorString(e));
    return RGF_ERR_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return RGF_OK;
}
}  // namespace

extern "C" {

rgf_status rgf_create(int device, rgf_handle* out) {
  if (!out) {
    set_error("NULL output pointer");
    return RGF_ERR_ARG;
  }
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return RGF_ERR_NODEVICE;
  }
  if (device < 0 || device >= n) {
    set_error("device index out of range");
    return RGF_ERR_ARG;
  }
  RGF_CUDA_TRY(cudaSetDevice(device));
  rgf_handle h = new rgf_handle_s();
  h->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    set_error(std::string("cudaStreamCreate failed: ") + cudaGetErrorString(e));
    return RGF_ERR_CUDA;
  }
  h->stream = h->own_stream;
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
  *out = h;
  return RGF_OK;
}

rgf_status rgf_destroy(rgf_handle h) {
  if (!h) return RGF_OK;
  cudaSetDevice(h->device);
  DevBuf* bufs[] = {&h->k0,     &h->k1,     &h->kx[0],     &h->kx[1],     &h->lam[0],  &h->lam[1],
                    &h->mu[0],  &h->mu[1],  &h->isprop[0], &h->isprop[1], &h->prop[0], &h->prop[1],
                    &h->conj[0], &h->conj[1], &h->nprop,   &h->status,    &h->phi,     &h->tmp,
                    &h->g0s,    &h->g0e,    &h->st_col,    &h->st_val,    &h->eps,     &h->aug,
                    &h->pc,     &h->u,      &h->idx,       &h->sdev,      &h->xpc,     &h->xrow,
                    &h->xt,     &h->xu,     &h->xsync,     &h->xprobe,    &h->gepp,    &h->gck,
                    &h->gseg,   &h->gm0,    &h->gpsi,      &h->gphi,      &h->get,     &h->gd,
                    &h->gg,     &h->gf,     &h->segs};
  for (DevBuf* b : bufs)
    if (b->p) cudaFree(b->p);
  for (DevBuf& b : h->mx)
    if (b.p) cudaFree(b.p);
  for (cudaEvent_t ev : h->ev) cudaEventDestroy(ev);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  for (rgf_handle_s* w : h->workers) rgf_destroy(w);
  delete h;
  return RGF_OK;
}

rgf_status rgf_smatrix_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req, const rgf_options* opt,
                          rgf_cplx* S, int64_t ldS, rgf_channels* ch) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst) {
    set_error("syst must be a structure");
    return RGF_ERR_ARG;
  }
  return smatrix(h, problem2d(syst), req, opt, S, ldS, ch);
}

rgf_status rgf_smatrix_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req, const rgf_options* opt,
                          rgf_cplx* S, int64_t ldS, rgf_channels* ch) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst) {
    set_error("syst must be a structure");
    return RGF_ERR_ARG;
  }
  return smatrix(h, problem3d(syst), req, opt, S, ldS, ch);
}

// The batched call in one launch (GangBatch): one host thread and one handle
// per structure, at most kGangChunk structures per launch.
constexpr int64_t kGangChunk = kGangMaxItems;

static rgf_status batch_one_launch(rgf_handle h, int64_t count, const rgf_syst2d* systs, const rgf_request* reqs,
                                   const rgf_options* opt, rgf_cplx* const* S, const int64_t* ldS,
                                   rgf_status* statuses) {
  std::vector<rgf_status> res(count, RGF_OK);
  std::vector<std::string> msg(count);
  // more than kGangChunk structures: several launches, each with a share of
  // every size (structures dealt round-robin in order of cost); all threads
  // run at once, so one launch's set-up overlaps another's sweeps
  const int64_t nch = (count + kGangChunk - 1) / kGangChunk;
  std::vector<int64_t> order(count);
  for (int64_t i = 0; i < count; i++) order[i] = i;
  std::vector<double> cost(count);
  for (int64_t i = 0; i < count; i++) {
    const double N = (double)systs[i].ny;
    cost[i] = (double)std::max<int64_t>(systs[i].nx, 1) * N * N * N;
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return cost[x] > cost[y]; });
  std::vector<std::unique_ptr<GangBatch>> gb(nch);
  for (int64_t c = 0; c < nch; c++) {
    gb[c].reset(new GangBatch());
    gb[c]->device = h->device;
    gb[c]->sms = h->sms;
    gb[c]->stream = h->stream;
  }
  for (int64_t r = 0; r < count; r++) gb[r % nch]->pending++;
  std::vector<rgf_handle> ws(count, nullptr);
  std::vector<std::thread> pool;
  for (int64_t r = 0; r < count; r++) {
    const int64_t k = order[r];
    GangBatch* g = gb[r % nch].get();
    rgf_status st = rgf_create(h->device, &ws[k]);
    if (st != RGF_OK) {
      res[k] = st;
      msg[k] = tl_err;
      std::lock_guard<std::mutex> lock(g->mu);
      gang_arrive_locked(g);
      continue;
    }
    ws[k]->gang = g;
    ws[k]->tile_rmax = h->tile_rmax;
    ws[k]->tile_bm = h->tile_bm;
    pool.emplace_back([&, k, g] {
      rgf_handle w = ws[k];
      cudaSetDevice(w->device);
      res[k] = smatrix(w, problem2d(&systs[k]), &reqs[k], opt, S[k], ldS[k], nullptr);
      if (res[k] != RGF_OK) msg[k] = tl_err;
      if (!w->gang_submitted) gang_leave(g);
    });
  }
  for (auto& th : pool) th.join();
  int64_t launches = 0;
  for (auto& g : gb) launches += g->launches;
  for (rgf_handle w : ws)
    if (w) rgf_destroy(w);
  h->launches = launches;  // persistent (gang) launches of the call
  rgf_status first = RGF_OK;
  for (int64_t i = 0; i < count; i++) {
    if (statuses) statuses[i] = res[i];
    if (res[i] != RGF_OK && first == RGF_OK) {
      first = res[i];
      set_error("batch item " + std::to_string(i) + ": " + msg[i]);
    }
  }
  return first;
}

rgf_status rgf_smatrix_batch_2d(rgf_handle h, int64_t count, const rgf_syst2d* systs, const rgf_request* reqs,
                                const rgf_options* opt, rgf_cplx* const* S, const int64_t* ldS,
                                rgf_status* statuses, int32_t workers) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (count < 0 || (count > 0 && (!systs || !reqs || !S || !ldS))) {
    set_error("batch: count must be >= 0 and systs, reqs, S, ldS non-NULL");
    return RGF_ERR_ARG;
  }
  if (count == 0) return RGF_OK;
  if (opt && opt->profile > 0) {
    set_error("batch: profiling is per call; use rgf_smatrix_2d");
    return RGF_ERR_ARG;
  }
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  // the split-precision form runs as pipelines (8 by default: each holds its
  // structure's factor store, up to ~12 GB for N = 512, L = 2000)
  const bool split = opt && opt->precision == RGF_TF32X3;
  if (workers <= 0 && !split) return batch_one_launch(h, count, systs, reqs, opt, S, ldS, statuses);
  int nw = workers > 0 ? workers : 8;
  nw = (int)std::min<int64_t>(nw, count);
  nw = std::max(1, std::min(nw, h->sms / 2));
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  while ((int)h->workers.size() < nw) {
    rgf_handle w = nullptr;
    if ((st = rgf_create(h->device, &w))) return st;
    h->workers.push_back(w);
  }
  // the pipelines' persistent sweeps draw their SMs from one budget (a sweep
  // waits until its whole grid fits), so their cooperative grids are always
  // co-resident; each picks the largest tile whose grid fits the GPU
  h->sm_free.store(h->sms);
  for (int i = 0; i < nw; i++) {
    h->workers[i]->sms = h->sms;
    h->workers[i]->sm_budget = &h->sm_free;
    h->workers[i]->tile_rmax = h->tile_rmax;
    h->workers[i]->tile_bm = h->tile_bm;
  }
  // largest first (sum over slices of N^3 + N^2 P), so that the pipelines finish together
  std::vector<int64_t> order(count);
  for (int64_t i = 0; i < count; i++) order[i] = i;
  std::vector<double> cost(count);
  for (int64_t i = 0; i < count; i++) {
    const double N = (double)systs[i].ny;
    cost[i] = (double)std::max<int64_t>(systs[i].nx, 1) * N * N * N;
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
  std::vector<rgf_status> res(count, RGF_OK);
  std::vector<std::string> msg(count);
  std::atomic<int64_t> next(0);
  auto work = [&](int wi) {
    rgf_handle w = h->workers[wi];
    cudaSetDevice(w->device);
    for (;;) {
      const int64_t k = next.fetch_add(1);
      if (k >= count) break;
      const int64_t i = order[k];
      res[i] = smatrix(w, problem2d(&systs[i]), &reqs[i], opt, S[i], ldS[i], nullptr);
      if (res[i] != RGF_OK) msg[i] = tl_err;
    }
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nw; i++) pool.emplace_back(work, i);
  work(0);
  for (auto& th : pool) th.join();
  rgf_status first = RGF_OK;
  for (int64_t i = 0; i < count; i++) {
    if (statuses) statuses[i] = res[i];
    if (res[i] != RGF_OK && first == RGF_OK) {
      first = res[i];
      set_error("batch item " + std::to_string(i) + ": " + msg[i]);
    }
  }
  return first;
}

rgf_status rgf_smatrix_grad_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                               const rgf_options* opt, const rgf_cplx* D, int64_t ldD, rgf_cplx* S, int64_t ldS,
                               rgf_cplx* g, int64_t checkpoint) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !D || !g) {
    set_error("syst, D and g must not be NULL");
    return RGF_ERR_ARG;
  }
  GradReq gr{D, ldD, g, checkpoint};
  return smatrix(h, problem2d(syst), req, opt, S, ldS, nullptr, &gr);
}

rgf_status rgf_smatrix_grad_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                               const rgf_options* opt, const rgf_cplx* D, int64_t ldD, rgf_cplx* S, int64_t ldS,
                               rgf_cplx* g, int64_t checkpoint) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !D || !g) {
    set_error("syst, D and g must not be NULL");
    return RGF_ERR_ARG;
  }
  GradReq gr{D, ldD, g, checkpoint};
  return smatrix(h, problem3d(syst), req, opt, S, ldS, nullptr, &gr);
}

rgf_status rgf_fields_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req, const rgf_options* opt,
                         rgf_cplx* S, int64_t ldS, rgf_cplx* psi, int64_t checkpoint) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !psi) {
    set_error("syst and psi must not be NULL");
    return RGF_ERR_ARG;
  }
  GradReq gr{nullptr, 0, nullptr, checkpoint, psi};
  return smatrix(h, problem2d(syst), req, opt, S, ldS, nullptr, &gr);
}

rgf_status rgf_fields_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req, const rgf_options* opt,
                         rgf_cplx* S, int64_t ldS, rgf_cplx* psi, int64_t checkpoint) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !psi) {
    set_error("syst and psi must not be NULL");
    return RGF_ERR_ARG;
  }
  GradReq gr{nullptr, 0, nullptr, checkpoint, psi};
  return smatrix(h, problem3d(syst), req, opt, S, ldS, nullptr, &gr);
}

static rgf_status segment_args(rgf_handle h, const void* syst, int side, const void* state) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !state) {
    set_error("syst and state must not be NULL");
    return RGF_ERR_ARG;
  }
  if (side != 0 && side != 1) {
    set_error("side must be 0 (left) or 1 (right)");
    return RGF_ERR_ARG;
  }
  return RGF_OK;
}

rgf_status rgf_segment_sweep_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req, const rgf_options* opt,
                                int32_t side, int64_t cut, rgf_cplx* state) {
  rgf_status st;
  if ((st = segment_args(h, syst, side, state))) return st;
  SegReq sg{side, cut, state};
  return smatrix(h, problem2d(syst), req, opt, nullptr, 0, nullptr, nullptr, &sg);
}

rgf_status rgf_segment_sweep_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req, const rgf_options* opt,
                                int32_t side, int64_t cut, rgf_cplx* state) {
  rgf_status st;
  if ((st = segment_args(h, syst, side, state))) return st;
  SegReq sg{side, cut, state};
  return smatrix(h, problem3d(syst), req, opt, nullptr, 0, nullptr, nullptr, &sg);
}

rgf_status rgf_segment_merge_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req, const rgf_options* opt,
                                const rgf_cplx* state_L, const rgf_cplx* state_R, rgf_cplx* S, int64_t ldS) {
  rgf_status st;
  if ((st = segment_args(h, syst, 0, state_L))) return st;
  return segment_merge(h, problem2d(syst), req, opt, state_L, state_R, S, ldS);
}

rgf_status rgf_segment_merge_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req, const rgf_options* opt,
                                const rgf_cplx* state_L, const rgf_cplx* state_R, rgf_cplx* S, int64_t ldS) {
  rgf_status st;
  if ((st = segment_args(h, syst, 0, state_L))) return st;
  return segment_merge(h, problem3d(syst), req, opt, state_L, state_R, S, ldS);
}

rgf_status rgf_smatrix_size_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req, int64_t* n_out,
                               int64_t* n_in) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !n_out || !n_in) {
    set_error("NULL argument");
    return RGF_ERR_ARG;
  }
  return smatrix_sizes(h, problem2d(syst), req, n_out, n_in);
}

rgf_status rgf_smatrix_size_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req, int64_t* n_out,
                               int64_t* n_in) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (!syst || !n_out || !n_in) {
    set_error("NULL argument");
    return RGF_ERR_ARG;
  }
  return smatrix_sizes(h, problem3d(syst), req, n_out, n_in);
}

static rgf_status setup_channels_common(rgf_handle h, const Transverse& tr, rgf_cplx k0dx, rgf_cplx eL,
                                        rgf_cplx eR, int32_t two_sided, rgf_channels* ch) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (tr.n0 <= 0 || tr.n1 <= 0) {
    set_error(tr.dim == 2 ? "ny must be a positive integer scalar" : "nx and ny must be positive integer scalars");
    return RGF_ERR_ARG;
  }
  if (!finite_c(k0dx) || !finite_c(eL) || (two_sided && !finite_c(eR))) {
    set_error("k0dx, epsilon_L and epsilon_R must be finite");
    return RGF_ERR_NONFINITE;
  }
  if (tr.bc < 0 || tr.bc > RGF_BC_BLOCH ||
      (tr.dim == 3 && tr.bc != RGF_BC_PERIODIC && tr.bc != RGF_BC_DIRICHLET && tr.bc != RGF_BC_BLOCH)) {
    set_error("Boundary condition BC is not an eligible option");
    return RGF_ERR_ARG;
  }
  if (!isfinite(tr.ka0) || !isfinite(tr.ka1)) {
    set_error("k*a has to be real for a complete orthonormal transverse basis.");
    return RGF_ERR_ARG;
  }
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  double2 k2, k2eL, k2eR;
  k2eps(k0dx, eL, &k2, &k2eL);
  k2eps(k0dx, two_sided ? eR : eL, &k2, &k2eR);
  ChanInfo ci;
  if ((st = run_channels(h, tr, k2eL, k2eR, two_sided != 0, &ci))) return st;
  return copy_channels_out(h, tr, ci, ch);
}

rgf_status rgf_setup_channels_2d(rgf_handle h, int64_t ny, int32_t bc, double ka, rgf_cplx k0dx,
                                 rgf_cplx epsilon_L, rgf_cplx epsilon_R, int32_t two_sided, rgf_channels* ch) {
  Transverse tr{2, ny, 1, ny, bc, bc == RGF_BC_BLOCH ? ka : 0.0, 0.0};
  return setup_channels_common(h, tr, k0dx, epsilon_L, epsilon_R, two_sided, ch);
}

rgf_status rgf_setup_channels_3d(rgf_handle h, int64_t nx, int64_t ny, int32_t bc, double kxa, double kya,
                                 rgf_cplx k0dx, rgf_cplx epsilon_L, rgf_cplx epsilon_R, int32_t two_sided,
                                 rgf_channels* ch) {
  Transverse tr{3, nx, ny, nx * ny, bc, bc == RGF_BC_BLOCH ? kxa : 0.0, bc == RGF_BC_BLOCH ? kya : 0.0};
  return setup_channels_common(h, tr, k0dx, epsilon_L, epsilon_R, two_sided, ch);
}

rgf_status rgf_build_laplacian_1d(rgf_handle h, int64_t n, int32_t bc, double ka, rgf_cplx* A) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (n < 0) {
    set_error("The number of sites n must be a non-negative integer scalar");
    return RGF_ERR_ARG;
  }
  if (bc < 0 || bc > RGF_BC_BLOCH) {
    set_error("Boundary condition BC is not an eligible option");
    return RGF_ERR_ARG;
  }
  if (n == 0) return RGF_OK;
  if (!A) {
    set_error("NULL output");
    return RGF_ERR_ARG;
  }
  RGF_CUDA_TRY(cudaSetDevice(h->device));
  if ((st = ensure(h, h->tmp, sizeof(double2) * n * n))) return st;
  launch_laplacian_dense(n, bc, bc == RGF_BC_BLOCH ? ka : 0.0, as<double2>(h->tmp), h->stream);
  if ((st = check_launch())) return st;
  RGF_CUDA_TRY(cudaMemcpyAsync(A, h->tmp.p, sizeof(double2) * n * n, cudaMemcpyDeviceToHost, h->stream));
  RGF_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return RGF_OK;
}

const char* rgf_last_error(void) { return tl_err.c_str(); }

const char* rgf_version(void) { return "rgf-b200 0.1.0 (sm_100a, FP64 DMMA sweep)"; }

rgf_status rgf_last_profile(rgf_handle h, int64_t* timed_launches, double* total_ms, double* flops_per_launch,
                            char* kernel_name, size_t name_len) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (timed_launches) *timed_launches = h->prof_n;
  if (total_ms) *total_ms = h->prof_ms;
  if (flops_per_launch) *flops_per_launch = h->prof_n ? h->prof_flops / (double)h->prof_n : 0.0;
  if (kernel_name && name_len) {
    strncpy(kernel_name, h->prof_kernel.c_str(), name_len - 1);
    kernel_name[name_len - 1] = 0;
  }
  return RGF_OK;
}

rgf_status rgf_set_stream(rgf_handle h, void* stream) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  h->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : h->own_stream;
  return RGF_OK;
}

rgf_status rgf_set_tile_table(rgf_handle h, int32_t n, const int64_t* rows_max, const int32_t* tile) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (n < 0 || (n > 0 && (!rows_max || !tile))) {
    set_error("tile table: n >= 0 and non-NULL arrays");
    return RGF_ERR_ARG;
  }
  for (int32_t i = 0; i < n; i++) {
    if (tile[i] != 32 && tile[i] != 64 && tile[i] != 96) {
      set_error("tile table: tile must be 32, 64 or 96");
      return RGF_ERR_ARG;
    }
    if (i > 0 && rows_max[i] < rows_max[i - 1]) {
      set_error("tile table: rows_max must be non-decreasing");
      return RGF_ERR_ARG;
    }
  }
  h->tile_rmax.assign(rows_max, rows_max + n);
  h->tile_bm.assign(tile, tile + n);
  return RGF_OK;
}

rgf_status rgf_last_engine(rgf_handle h, int32_t* engine, int32_t* fallback, double* rejected_probe) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (engine) *engine = h->engine_used;
  if (fallback) *fallback = h->fallback;
  if (rejected_probe) *rejected_probe = h->fallback ? h->probe_first : 0.0;
  return RGF_OK;
}

rgf_status rgf_last_refinement(rgf_handle h, int32_t* form, int32_t* iterations, double* last_change,
                               double* factor_ms, double* solve_ms) {
  if (rgf_status st = check_handle(h)) return st;
  if (form) *form = h->mx_fallback ? -RGF_TF32X3 : h->mx_form;
  if (iterations) *iterations = h->mx_stats.iterations;
  if (last_change) *last_change = h->mx_stats.last_change;
  if (factor_ms) *factor_ms = h->mx_stats.factor_ms;
  if (solve_ms) *solve_ms = h->mx_stats.solve_ms;
  return RGF_OK;
}

rgf_status rgf_last_stats(rgf_handle h, int64_t* kernel_launches, double* probe_residual) {
  rgf_status st;
  if ((st = check_handle(h))) return st;
  if (kernel_launches) *kernel_launches = h->launches;
  if (probe_residual) *probe_residual = h->probe;
  return RGF_OK;
}

rgf_status rgf_smatrix_2d_noalloc(const rgf_syst2d* syst, const rgf_request* req, const rgf_options* opt,
                                  rgf_cplx* S, int64_t ldS, rgf_channels* ch, void* stream) {
  if (!syst) {
    set_error("syst must be a structure");
    return RGF_ERR_ARG;
  }
  if (opt && opt->profile > 0) {
    set_error("rgf_smatrix_2d_noalloc: profiling is not available (it creates CUDA events)");
    return RGF_ERR_ARG;
  }
  int device = 0;
  RGF_CUDA_TRY(cudaGetDevice(&device));
  unsigned char* base = nullptr;
  rgf_status st;
  if ((st = noalloc_scratch(&base))) return st;
  // a handle on the stack whose arena is the static scratch: every workspace
  // buffer is carved from it and ensure() never reaches cudaMalloc; nothing
  // in it owns device memory, so it is not destroyed
  Arena arena;
  arena.base = base;
  arena.cap = RGF_NOALLOC_SCRATCH_BYTES;
  rgf_handle_s h;
  h.device = device;
  h.stream = reinterpret_cast<cudaStream_t>(stream);
  h.arena = &arena;
  RGF_CUDA_TRY(cudaDeviceGetAttribute(&h.sms, cudaDevAttrMultiProcessorCount, device));
  return smatrix(&h, problem2d(syst), req, opt, S, ldS, ch);
}

}  // extern "C"

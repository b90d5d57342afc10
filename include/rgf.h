/*
 * rgf.h -- C ABI of librgf, a B200 (sm_100a) implementation of the recursive
 * Green's function (RGF) slice recursion of chiaweihsu/RGF.
 *
 * Every entry point replaces one MATLAB function of the reference:
 *
 *   rgf_smatrix_2d          <- src/cal_smatrix_RGF.m:1      [smatrix, channels] = cal_smatrix_RGF(syst, out, in)
 *   rgf_smatrix_3d          <- src/cal_smatrix_RGF_3D.m:1   [smatrix, channels] = cal_smatrix_RGF_3D(syst, out, in)
 *   rgf_setup_channels_2d   <- src/setup_channels.m:1       channels = setup_channels(ny, BC, k0dx, epsilon_L, epsilon_R)
 *   rgf_setup_channels_3d   <- src/setup_channels_3D.m:1    channels = setup_channels_3D(nx, ny, BC, k0dx, epsilon_L, epsilon_R)
 *   rgf_build_laplacian_1d  <- src/build_laplacian_1d.m:1   A = build_laplacian_1d(n, BC)
 *
 * The reference has no FFI of its own (it is MATLAB source); the binding a
 * MATLAB user calls is a MEX gateway over this header (matlab/rgf_mex.c).
 *
 * Conventions
 *  - Complex numbers are rgf_cplx {re, im}: the memory layout of C99
 *    double _Complex, numpy complex128 and MATLAB's interleaved complex API.
 *  - Arrays are column-major (MATLAB layout).  syst.epsilon of size [ny, nx]
 *    (2D) or [nx, ny, nz] (3D) is passed as the plain column-major buffer,
 *    so slice n is the contiguous block epsilon + n*N, N = ny (2D) or nx*ny (3D).
 *  - Channel indices in the C ABI are 0-based (MATLAB's are 1-based; the
 *    MEX gateway and the Python wrapper convert).
 *  - All buffers are owned by the caller.  A handle owns its device
 *    workspace and CUDA stream; one handle per host thread.  Calls on
 *    distinct handles are independent.
 *  - Every function returns an rgf_status; rgf_last_error() gives the
 *    message of the last failure on the calling thread.
 */
#ifndef RGF_H
#define RGF_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RGF_API __attribute__((visibility("default")))
#else
#define RGF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double re, im;
} rgf_cplx;

typedef enum {
  RGF_OK = 0,
  RGF_ERR_ARG = 1,       /* invalid argument (MATLAB error() in the reference)          */
  RGF_ERR_NONFINITE = 2, /* NaN/Inf in epsilon, epsilon_L/R or k0dx                      */
  RGF_ERR_SINGULAR = 3,  /* a slice matrix is singular (zero pivot under partial pivoting) */
  RGF_ERR_TIMEOUT = 4,   /* a device-side wait gave up (bounded spin)                    */
  RGF_ERR_CUDA = 5,      /* CUDA runtime error                                           */
  RGF_ERR_OOM = 6,       /* device allocation failed                                     */
  RGF_ERR_NODEVICE = 7,  /* no usable CUDA device                                        */
  RGF_ERR_ILLCOND = 8    /* a slice inverse failed its a-posteriori check even under
                            partial pivoting over the whole column (residual > 1e-8):
                            S and channels are written but may be inaccurate (where
                            MATLAB's inv warns "close to singular or badly scaled")  */
} rgf_status;

/* Transverse boundary conditions (setup_channels.m:10-20, build_laplacian_1d.m:9-17). */
typedef enum {
  RGF_BC_PERIODIC = 0,          /* 'periodic'                      */
  RGF_BC_DIRICHLET = 1,         /* 'Dirichlet' / 'PEC'             */
  RGF_BC_NEUMANN = 2,           /* 'Neumann' / 'PMC'               */
  RGF_BC_DIRICHLET_NEUMANN = 3, /* 'DirichletNeumann' / 'PECPMC'   */
  RGF_BC_NEUMANN_DIRICHLET = 4, /* 'NeumannDirichlet' / 'PMCPEC'   */
  RGF_BC_BLOCH = 5              /* numeric BC = k*a (Bloch phase)  */
} rgf_bc;

/* Numeric form of the slice recursion. */
typedef enum {
  RGF_FP64 = 0,  /* complex FP64 throughout (the drop-in form) */
  RGF_TF32X3 = 1 /* split precision: every slice inverse factored in FP32 with 3xTF32
                    tensor-core updates (tcgen05), S won back by FP64 iterative
                    refinement of the block-tridiagonal solve against the FP64
                    operator; falls back to RGF_FP64 when the refinement does not
                    converge or its factor store (8 N lda L bytes, lda = 2N
                    rounded up to 32) does not fit (rgf_last_refinement tells).  S-matrices only
                    (rgf_smatrix_2d/3d and the pipelined batch).              */
} rgf_precision;

/* Value of n_* in rgf_request meaning "all propagating channels on that side"
 * (the MATLAB cell form {'left'} / {'right'}, cal_smatrix_RGF.m:120-135). */
#define RGF_ALL (-1)

typedef struct rgf_handle_s* rgf_handle;

/* syst for cal_smatrix_RGF (cal_smatrix_RGF.m:12-34). */
typedef struct {
  int64_t ny, nx;            /* size(syst.epsilon) = [ny, nx]; ny >= 1, nx >= 0          */
  const rgf_cplx* epsilon;   /* ny*nx, column-major; host memory unless eps_on_device    */
  int32_t eps_on_device;     /* 1: epsilon is a device pointer on the handle's device    */
  rgf_cplx epsilon_L, epsilon_R, k0dx;
  int32_t yBC;               /* rgf_bc                                                   */
  double ka;                 /* Bloch phase ky*a (yBC == RGF_BC_BLOCH)                   */
} rgf_syst2d;

/* syst for cal_smatrix_RGF_3D (cal_smatrix_RGF_3D.m:12-31). */
typedef struct {
  int64_t nx, ny, nz;        /* size(syst.epsilon) = [nx, ny, nz]                        */
  const rgf_cplx* epsilon;   /* nx*ny*nz, column-major (x fastest)                       */
  int32_t eps_on_device;
  rgf_cplx epsilon_L, epsilon_R, k0dx;
  int32_t xyBC;              /* RGF_BC_PERIODIC, RGF_BC_DIRICHLET or RGF_BC_BLOCH        */
  double kxa, kya;           /* Bloch phases (xyBC == RGF_BC_BLOCH)                      */
} rgf_syst3d;

/* out / in of cal_smatrix_RGF (cal_smatrix_RGF.m:35-50, 103-178): 0-based
 * channel lists per side; n == RGF_ALL selects every propagating channel,
 * n == 0 selects none. */
typedef struct {
  const int64_t* ind_out_L; int64_t n_out_L;
  const int64_t* ind_out_R; int64_t n_out_R;
  const int64_t* ind_in_L;  int64_t n_in_L;
  const int64_t* ind_in_R;  int64_t n_in_R;
} rgf_request;

typedef struct {
  int32_t precision;  /* rgf_precision (0 = RGF_FP64)                                  */
  int32_t engine;     /* 0 (default): persistent register-resident sweep kernel when
                         the matrix fits on the GPU, pivoting inside each 32 x 32
                         pivot block; every slice inverse is checked a posteriori
                         and the call is recomputed with engine 1 if one fails.
                         1: one launch sequence per pivot step with partial
                         pivoting over the whole column (LAPACK zgetrf's choice,
                         as MATLAB's inv)                                            */
  int32_t S_on_device;/* 1: S is a device pointer (no D2H copy)                        */
  int32_t profile;    /* > 0: time the dominant kernel with CUDA events on every
                         profile-th slice (read back with rgf_last_profile)           */
} rgf_options;

/* channels struct (setup_channels.m:30-82).  All pointers are caller-owned
 * arrays of capacity N (N = ny in 2D, nx*ny in 3D); any may be NULL. */
typedef struct {
  double* kydx;            /* N: transverse ky*dx (3D: nx-by-ny column-major)           */
  double* kxdx_t;          /* 3D only: transverse kx*dx (nx-by-ny column-major)         */
  rgf_cplx* kxdx_L;        /* N: longitudinal wavenumber, left (2D kxdx / 3D kzdx)      */
  rgf_cplx* kxdx_R;        /* N: right                                                  */
  rgf_cplx* sqrt_mu_L;     /* first N_prop_L entries used                               */
  rgf_cplx* sqrt_mu_R;
  int64_t* ind_prop_L;     /* 0-based, first N_prop_L entries used                      */
  int64_t* ind_prop_R;
  int64_t* ind_prop_conj_L;/* 0-based permutation of 0..N_prop_L-1 (2D, real profiles or ka == 0) */
  int64_t* ind_prop_conj_R;
  int64_t N_prop_L, N_prop_R;  /* outputs; N_prop_R = -1 for a one-sided setup          */
  int32_t has_prop_conj;       /* output: 1 if ind_prop_conj_* were written             */
  int32_t reserved;
} rgf_channels;

/* ---- handle ---------------------------------------------------------------- */
RGF_API rgf_status rgf_create(int device, rgf_handle* out);
RGF_API rgf_status rgf_destroy(rgf_handle h);

/* ---- cal_smatrix_RGF / cal_smatrix_RGF_3D ----------------------------------- */
/* S: n_out x n_in, column-major with leading dimension ldS >= n_out, where
 * rows are [out_L ; out_R] and columns [in_L ; in_R] (cal_smatrix_RGF.m:56-61).
 * ch may be NULL. */
RGF_API rgf_status rgf_smatrix_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                          const rgf_options* opt, rgf_cplx* S, int64_t ldS, rgf_channels* ch);
RGF_API rgf_status rgf_smatrix_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                          const rgf_options* opt, rgf_cplx* S, int64_t ldS, rgf_channels* ch);

/* Batched form: `count` independent 2D problems (each as rgf_smatrix_2d:
 * systs[i], reqs[i], S[i] with leading dimension ldS[i]; all host or all
 * device per opt->S_on_device).  workers <= 0 (default): every structure's
 * set-up runs on a host thread and stream of its own, and all their slice
 * sweeps run in ONE persistent cooperative launch in which gangs of CTAs,
 * sized to each structure, take the structures from a work queue in device
 * memory, largest first (at most 160 structures per launch; a structure that
 * needs tiles smaller than 96 x 96 sweeps on its own first).  workers > 0:
 * that many concurrent pipelines (host threads, each with its own stream and
 * workspace), whose persistent sweeps share the GPU's SMs through one budget.
 * With opt->precision = RGF_TF32X3 every structure takes the split-precision
 * form, as pipelines (workers <= 0: 8; each pipeline holds its structure's
 * factor store, 8 N lda L bytes).  statuses (may be NULL) receives each problem's status; the return value
 * is the first failure (message names the item).  The reference has no
 * batched call: its user loops over cal_smatrix_RGF. */
RGF_API rgf_status rgf_smatrix_batch_2d(rgf_handle h, int64_t count, const rgf_syst2d* systs,
                                        const rgf_request* reqs, const rgf_options* opt, rgf_cplx* const* S,
                                        const int64_t* ldS, rgf_status* statuses, int32_t workers);

/* Permittivity gradient (an addition: the reference computes S only).
 * Computes S as rgf_smatrix_2d/3d and
 *     g[m + n*N] = sum_ab D[a + b*ldD] * dS_ab / d epsilon[m, n]
 * for the caller's weights D (n_out x n_in, the row/column order of S), with
 * m the transverse site (N = ny, or nx*ny in 3D, x fastest) and n the slice.
 * For a real objective F of S with dF = 2 Re sum_ab D_ab dS_ab (e.g. D = conj(S)
 * for F = sum |S_ab|^2), dF/d Re(eps) = 2 Re g and dF/d Im(eps) = -2 Im g.
 * Method: the forward sweep keeps a checkpoint every `checkpoint` slices
 * (<= 0: ceil(sqrt(L))); the backward pass recomputes one segment at a time
 * and runs the recursions Psi_k = [X_k, 0] + g_k Psi_{k+1},
 * Phi_k = [Z_k; 0] + Phi_{k+1} g_k over the start-connected slice inverses g_k.
 * D, S and g are device pointers when opt->S_on_device, host otherwise. */
RGF_API rgf_status rgf_smatrix_grad_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                                       const rgf_options* opt, const rgf_cplx* D, int64_t ldD, rgf_cplx* S,
                                       int64_t ldS, rgf_cplx* g, int64_t checkpoint);
RGF_API rgf_status rgf_smatrix_grad_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                                       const rgf_options* opt, const rgf_cplx* D, int64_t ldD, rgf_cplx* S,
                                       int64_t ldS, rgf_cplx* g, int64_t checkpoint);

/* Fields inside the structure (an addition: the reference computes S only and
 * points to MESTI for fields, README.md:13).  Computes S as rgf_smatrix_2d/3d
 * and, for every requested input channel b (the columns of S, in S's order),
 *     psi[m + n*N + b*N*L] = (G_{n, s(b)} B_b)_m,
 * the response at transverse site m (N = ny, or nx*ny in 3D, x fastest) of
 * slice n (0 <= n < L = nx, or nz in 3D) to the source profile B_b of channel
 * b on its lead's surface slice s(b) (B = phi(:, ind_prop) sqrt(mu), the
 * matrix S = -2i C G B - delta is built from; cal_smatrix_RGF.m:191-195),
 * i.e. column b of the block-tridiagonal Green's function times B, laid out
 * as a MATLAB array [ny, nx, n_in] ([nx, ny, nz, n_in] in 3D).  The same
 * backward recursion as the gradient (checkpoint as there).  At least one
 * output channel must be requested.  psi is a device pointer when
 * opt->S_on_device, host memory otherwise. */
RGF_API rgf_status rgf_fields_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                                 const rgf_options* opt, rgf_cplx* S, int64_t ldS, rgf_cplx* psi,
                                 int64_t checkpoint);
RGF_API rgf_status rgf_fields_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                                 const rgf_options* opt, rgf_cplx* S, int64_t ldS, rgf_cplx* psi,
                                 int64_t checkpoint);

/* L-split S-matrix (an addition: the reference's loop over slices,
 * cal_smatrix_RGF.m:263-269, is strictly sequential).  The slices are cut at
 * `cut` (0 < cut < L): rgf_segment_sweep_* with side = 0 sweeps [0, cut) from
 * the left lead, with side = 1 [cut, L) from the right lead, carrying only
 * that side's requested channels, and writes the segment state
 *     state = [[g, X], [Z, Y]]   row-major, (N + n_out_side) x (N + n_in_side),
 * g the lead-connected Green's function of the part's last slice, X = G B,
 * Z = C G, Y = C G B at that lead.  The two sweeps are independent (two GPUs,
 * or one after the other on one); rgf_segment_merge_* joins the two states
 * across the cut by the Dyson equation of two Green's functions coupled by
 * the hopping -I (one sweep of a matrix of order N + n_out with pivot block
 * I - g_R g_L) and writes S as rgf_smatrix_*.  state / S are device pointers
 * when opt->S_on_device. */
RGF_API rgf_status rgf_segment_sweep_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                                        const rgf_options* opt, int32_t side, int64_t cut, rgf_cplx* state);
RGF_API rgf_status rgf_segment_sweep_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                                        const rgf_options* opt, int32_t side, int64_t cut, rgf_cplx* state);
RGF_API rgf_status rgf_segment_merge_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                                        const rgf_options* opt, const rgf_cplx* state_L, const rgf_cplx* state_R,
                                        rgf_cplx* S, int64_t ldS);
RGF_API rgf_status rgf_segment_merge_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                                        const rgf_options* opt, const rgf_cplx* state_L, const rgf_cplx* state_R,
                                        rgf_cplx* S, int64_t ldS);

/* Size of the S block a request selects (needs the channel count, so it runs
 * the channel set-up on the device). */
RGF_API rgf_status rgf_smatrix_size_2d(rgf_handle h, const rgf_syst2d* syst, const rgf_request* req,
                               int64_t* n_out, int64_t* n_in);
RGF_API rgf_status rgf_smatrix_size_3d(rgf_handle h, const rgf_syst3d* syst, const rgf_request* req,
                               int64_t* n_out, int64_t* n_in);

/* ---- setup_channels / setup_channels_3D / build_laplacian_1d ------------------ */
/* two_sided = 0 reproduces the one-sided form (epsilon_R omitted). */
RGF_API rgf_status rgf_setup_channels_2d(rgf_handle h, int64_t ny, int32_t bc, double ka, rgf_cplx k0dx,
                                 rgf_cplx epsilon_L, rgf_cplx epsilon_R, int32_t two_sided,
                                 rgf_channels* ch);
RGF_API rgf_status rgf_setup_channels_3d(rgf_handle h, int64_t nx, int64_t ny, int32_t bc, double kxa,
                                 double kya, rgf_cplx k0dx, rgf_cplx epsilon_L, rgf_cplx epsilon_R,
                                 int32_t two_sided, rgf_channels* ch);
/* A: n x n dense, column-major. */
RGF_API rgf_status rgf_build_laplacian_1d(rgf_handle h, int64_t n, int32_t bc, double ka, rgf_cplx* A);

/* ---- diagnostics ----------------------------------------------------------- */
RGF_API const char* rgf_last_error(void);
RGF_API const char* rgf_version(void);
/* Statistics of the last rgf_smatrix_* call on this handle: the number of
 * kernel launches it issued, and the largest relative residual
 * max|G_n (M_n v) - v| / max|v| of the per-slice probe vector v (an a
 * posteriori check of every slice inverse, carried as two extra columns of
 * the swept matrix). */
RGF_API rgf_status rgf_last_stats(rgf_handle h, int64_t* kernel_launches, double* probe_residual);
/* Engine that produced the last rgf_smatrix_* result on this handle (0 or 1,
 * see rgf_options.engine); fallback = 1 when the persistent engine's result
 * was rejected by the a-posteriori check (a zero or non-finite in-block
 * pivot, or a probe residual above 1e-10) and recomputed with engine 1;
 * rejected_probe is that run's residual.  An addition of this library. */
RGF_API rgf_status rgf_last_engine(rgf_handle h, int32_t* engine, int32_t* fallback, double* rejected_probe);
/* The split-precision form (RGF_TF32X3) of the last rgf_smatrix_* call on
 * this handle (an addition of this library; the reference has one FP64 form):
 * form = RGF_TF32X3 when its S stands, -RGF_TF32X3 when the refinement did not
 * converge and S was recomputed in FP64, RGF_FP64 when it was not asked for;
 * the number of refinement passes (the first solve included), the relative
 * size of the last correction (max over the whole solution and its first and
 * last slices), and the device time of the FP32 factorization and of all
 * solves (ms). */
RGF_API rgf_status rgf_last_refinement(rgf_handle h, int32_t* form, int32_t* iterations, double* last_change,
                                       double* factor_ms, double* solve_ms);
/* Sampled timing of the dominant kernel of the last rgf_smatrix_* call made
 * with opt->profile > 0: number of timed launches, their summed duration (ms),
 * the algorithmic flops of one such launch, and its name. */
RGF_API rgf_status rgf_last_profile(rgf_handle h, int64_t* timed_launches, double* total_ms,
                                    double* flops_per_launch, char* kernel_name, size_t name_len);
/* Tuned tile shapes of the persistent engine (an addition): a matrix of Rp
 * active rows (N plus the output channels carried) uses the square tile
 * tile[i] (32, 64 or 96) of the first entry with Rp <= rows_max[i] (rows_max
 * non-decreasing) whenever its grid fits the GPU, else the built-in choice
 * (the largest tile that keeps >= 60% of the SMs busy).  n = 0 clears the
 * table.  Batched calls pass it to their pipelines.  rgf_b200.autotune writes
 * such a table from timed sweeps and caches it as JSON. */
RGF_API rgf_status rgf_set_tile_table(rgf_handle h, int32_t n, const int64_t* rows_max, const int32_t* tile);
/* Issue all work of this handle on the caller's stream (a cudaStream_t);
 * NULL restores the handle's own stream. */
RGF_API rgf_status rgf_set_stream(rgf_handle h, void* stream);

/* ---- allocation-free variant -------------------------------------------------
 * No counterpart in the reference: an addition of this library.
 *
 * rgf_smatrix_2d without a handle and without any device allocation, for
 * callers that must not call cudaMalloc/cudaFree: code that runs inside a
 * host application owning the device memory pool (MATLAB's gpuArray memory
 * manager, a deep-learning framework's caching allocator), where a library
 * allocating on its own would fail once the pool has claimed the memory or
 * fragment it, and latency-bound callers for which cudaMalloc/cudaFree, which
 * can synchronize the whole device, are not acceptable.  The caller still
 * passes every input and output (syst, req, S, ch as for rgf_smatrix_2d); all
 * device workspace -- channel data, the augmented slice matrix, the sweep's
 * exchange buffers and flags -- is carved from one static device array of
 * RGF_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * the process exits.  A problem whose workspace does not fit is rejected with
 * RGF_ERR_ARG and a message naming the limit.  The workspace is, in bytes,
 * with N = ny, R = N + n_out, C = N + n_in + 2 (n_out, n_in: the sizes of
 * the requested S block):
 *     16 * (3 N^2 + R (C + 1) + 64 R + 288 C + 110 N)      about, and
 *   + 16 N^2      when epsilon_L != epsilon_R (a second lead),
 *   + 16 N nx     when epsilon is in host memory (eps_on_device = 0),
 * which puts the largest ny near 615 for the full S of a periodic problem at
 * k0dx = 2 pi / 15 (about 2 ny / 15 channels per side).  Work is issued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) of the current
 * device.  Every call looks up the array's device address on the current
 * device (cudaGetSymbolAddress, which allocates nothing), so a context that
 * the host application reset is followed.  Every call on a device shares the one array,
 * so calls that overlap on the GPU (other host threads, other streams) race;
 * each call clears what must start at zero.  opt->profile must be 0. */
#define RGF_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
RGF_API rgf_status rgf_smatrix_2d_noalloc(const rgf_syst2d* syst, const rgf_request* req,
                                          const rgf_options* opt, rgf_cplx* S, int64_t ldS,
                                          rgf_channels* ch, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RGF_H */

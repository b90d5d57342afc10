// Slice-recursion kernels (see sweep.cu).
#pragma once
#include "rgf_internal.cuh"

namespace rgf {

// operand of the complex GEMM: element (r, c) of the logical matrix is
// p[r*ld + c] (op 0), p[c*ld + r] (op 1) or conj(p[c*ld + r]) (op 2)
struct ZOp {
  const double2* p;
  int64_t ld;
  int op;
};

// addend of a GEMM: C = A B + add, add read in its rows x cols corner (row-major, ld)
struct ZAdd {
  const double2* p;
  int64_t ld, rows, cols;
};

void launch_zgemm(int64_t M, int64_t N, int64_t K, double2 alpha, ZOp A, ZOp B, double2 beta, double2* C,
                  int64_t ldc, cudaStream_t s);
void launch_zgemm_add(int64_t M, int64_t N, int64_t K, ZOp A, ZOp B, ZAdd add, double2* C, int64_t ldc,
                      cudaStream_t s);
int sweep_block_width();
void launch_sweep_panel(const double2* M, int64_t ldm, int64_t R, int64_t Cc, int64_t j0, int jn, double2* Pc,
                        double2* U, int64_t ldu, int* status, cudaStream_t s);
void launch_sweep_update(double2* M, int64_t ldm, int64_t R, int64_t Cc, int64_t j0, int jn, const double2* Pc,
                         const double2* U, int64_t ldu, cudaStream_t s);
const char* sweep_update_kernel_name();
// partial pivoting over the whole remaining column (see sweep.cu): scratch of
// gepp_scratch_bytes(N); launch_gepp_step before each sweep step (rows of W
// exchanged over columns [0, Cc)), launch_gepp_unpermute after the last one
size_t gepp_scratch_bytes(int64_t N);
void launch_gepp_step(double2* M, int64_t ldm, int64_t N, int64_t Cc, int64_t j0, int jn, void* scratch,
                      int* status, cudaStream_t s);
cudaError_t launch_gepp_unpermute(double2* M, int64_t ldm, int64_t R, int64_t N, void* scratch, cudaStream_t s);
void launch_probe_check(const double2* M, int64_t ldm, int64_t N, int64_t pc1, unsigned long long* probe_max,
                        cudaStream_t s);
void launch_assemble(double2* M, int64_t ldm, int64_t N, int64_t Rz, const double2* Gsrc, int64_t ldg,
                     const double2* Gextra, int64_t lde, const int* st_col, const double2* st_val, double2 k2,
                     const double2* eps, double2 eps_u, cudaStream_t s);
void launch_fill_init(double2* M, int64_t ldm, int64_t N, const double2* phi, int64_t ldp, const int* prop,
                      const double2* lam, const double2* mu, const int* in_s, int n_in, const int* out_s,
                      int n_out, cudaStream_t s);
void launch_fill_attach(double2* M, int64_t ldm, int64_t N, int ni_s, int no_s, const double2* phi,
                        int64_t ldp, const int* prop, const double2* mu, const int* in_e, int ni_e,
                        const int* out_e, int no_e, cudaStream_t s);
void launch_extract(const double2* M, int64_t ldm, int64_t N, const int* row_of, int no, const int* col_of,
                    int ni, double2* S, int64_t ldS, const int* pairs, int npairs, cudaStream_t s);
void launch_probe_init(double2* M, int64_t ldm, int64_t N, int64_t R, int64_t pc1, cudaStream_t s);
void launch_check_finite(const double2* x, int64_t n, int* status, cudaStream_t s);
void launch_scale_cols(const double2* src, int64_t lds, const double2* diag, double2* dst, int64_t ldd,
                       int64_t rows, int64_t cols, cudaStream_t s);
// permittivity gradient: the per-slice contraction
// g[m] = coef * sum_a Phi[a][m] sum_b D[a][b] Psi[m][b] (fused for small D, else
// through Et = D Psi^T)
void launch_grad_fused(const double2* Phi, const double2* Psi, const double2* D, int64_t N, int n_out, int n_in,
                       double2 coef, double2* g, cudaStream_t s);
// dst = scale * src block (src == nullptr: zero); M += I on the leading n x n
void launch_block_copy(double2* dst, int64_t ldd, const double2* src, int64_t lds, int64_t rows, int64_t cols,
                       double scale, cudaStream_t s);
void launch_add_identity(double2* M, int64_t ldm, int64_t n, cudaStream_t s);
// fields: out[m + i*ld] = Psi[m][col_of[i]]
void launch_store_field(const double2* Psi, const int* col_of, int64_t N, int n_in, double2* out, int64_t ld,
                        cudaStream_t s);
// one slice of the backward recursions (and the contraction when g) in one
// launch, for n_in, n_out <= 32 (grad_step_fits)
bool grad_step_fits(int n_in, int n_out);
void launch_grad_step(const double2* W, int64_t ld, int64_t N, int n_in, int n_out, int ni_s, int no_s,
                      const double2* Psi_in, const double2* Phi_in, const double2* D, double2 coef, double2* Psi_out,
                      double2* Phi_out, double2* g, cudaStream_t s);
void launch_grad_slice(const double2* Phi, const double2* Et, int64_t N, int64_t n_out, double2 coef, double2* g,
                       cudaStream_t s);

}  // namespace rgf

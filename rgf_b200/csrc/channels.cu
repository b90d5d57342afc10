// Lead channels, transverse profiles and the slice stencil, on the device.
//
//   k_transverse / k_longitudinal  <- setup_channels.m:122-236, setup_channels_3D.m:102-186
//   k_compact_prop                 <- setup_channels.m:195-198, 222-236 (find, ind_prop_conj)
//   k_phi                          <- setup_channels.m:133-156 (fun_phi), setup_channels_3D.m:118-123,
//                                     cal_smatrix_RGF_3D.m:185-188 (column-major Kronecker profiles)
//   k_stencil                      <- build_laplacian_1d.m:48-75, cal_smatrix_RGF.m:209,
//                                     cal_smatrix_RGF_3D.m:218-224 (A0 = -Lap + 2I, Kronecker sum)
//
// Complex elementary functions are written from their definitions on top of
// CUDA's real sqrt/hypot/atan2/asinh/acosh/exp/sin/cos (called, not restated):
// the principal square root, and the principal arcsine by Kahan's formula
// (W. Kahan, "Branch cuts for complex elementary functions", 1987):
//   asin z = atan2(Re z, Re(sqrt(1-z) sqrt(1+z))) + i asinh(Im(conj(sqrt(1-z)) sqrt(1+z))).
#include <math.h>

#include "channels.cuh"

namespace rgf {

// principal square root; a zero imaginary part of either sign is treated as
// +0 (MATLAB has no signed zero in these expressions)
__device__ double2 csqrt_p(double2 z) {
  double x = z.x, y = z.y;
  if (x == 0.0 && y == 0.0) return cmk(0.0, 0.0);
  double r = hypot(x, y);
  if (x >= 0.0) {
    double t = sqrt(0.5 * (r + x));
    return cmk(t, y / (2.0 * t));
  }
  double t = sqrt(0.5 * (r - x));
  return cmk(fabs(y) / (2.0 * t), (y < 0.0) ? -t : t);
}

__device__ double2 casin_p(double2 w) {
  double2 s1 = csqrt_p(cmk(1.0 - w.x, -w.y));
  double2 s2 = csqrt_p(cmk(1.0 + w.x, w.y));
  double re = atan2(w.x, s1.x * s2.x - s1.y * s2.y);
  double im = asinh(s1.x * s2.y - s1.y * s2.x);
  return cmk(re, im);
}

__device__ inline double2 cexp_i(double2 k) {  // exp(1i*k)
  double s, c;
  sincos(k.x, &s, &c);
  double m = exp(-k.y);
  return cmk(m * c, m * s);
}

__device__ inline double2 csin_p(double2 k) {  // sin(a+ib) = sin a cosh b + i cos a sinh b
  double s, c;
  sincos(k.x, &s, &c);
  return cmk(s * cosh(k.y), c * sinh(k.y));
}

// transverse wavenumber of mode a (0-based) along an axis of n sites
__device__ double transverse_k(int bc, int64_t n, double ka, int64_t a) {
  const double pi = 3.141592653589793;
  switch (bc) {
    case RGF_BC_PERIODIC:
    case RGF_BC_BLOCH: {
      int64_t ind0 = (n % 2 == 1) ? (n + 1) / 2 : n / 2;  // setup_channels.m:125-129
      return (ka / (double)n) + ((double)(a + 1) - (double)ind0) * (2.0 * pi / (double)n);
    }
    case RGF_BC_DIRICHLET: return (double)(a + 1) * (pi / (double)(n + 1));
    case RGF_BC_NEUMANN: return (double)a * (pi / (double)n);
    default: return ((double)a + 0.5) * (pi / ((double)n + 0.5));  // DN, ND
  }
}

__global__ void k_transverse(Transverse tr, double* k0, double* k1) {
  int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double ka0 = (tr.bc == RGF_BC_BLOCH) ? tr.ka0 : 0.0;
  double ka1 = (tr.bc == RGF_BC_BLOCH) ? tr.ka1 : 0.0;
  if (a < tr.n0) k0[a] = transverse_k(tr.bc, tr.n0, ka0, a);
  if (tr.dim == 3 && a < tr.n1) k1[a] = transverse_k(tr.bc, tr.n1, ka1, a);
}

// One side (L or R) of setup_longitudinal for every channel a.
__global__ void k_longitudinal(Transverse tr, const double* k0, const double* k1, double2 k2e,
                               SideDev side) {
  int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (a >= tr.N) return;
  const bool is_real = (k2e.y == 0.0);
  double2 z;
  if (tr.dim == 2) {
    double s = sin(k0[a] / 2.0);
    z = cmk(0.25 * k2e.x - s * s, 0.25 * k2e.y);  // setup_channels.m:185
  } else {
    int64_t ax = a % tr.n0, ay = a / tr.n0;
    double sx = sin(k0[ax] / 2.0), sy = sin(k1[ay] / 2.0);
    z = cmk((0.25 * k2e.x - sx * sx) - sy * sy, 0.25 * k2e.y);  // setup_channels_3D.m:152
  }
  if (is_real) z.y = 0.0;
  double2 kx;
  if (is_real) {
    // MATLAB asin(sqrt(z)) on a real argument (setup_channels.m:190):
    // asin(w) = pi/2 - 1i*acosh(w) for w > 1, and 1i*asinh(y) for w = 1i*y.
    if (z.x >= 0.0) {
      double w = sqrt(z.x);
      if (w <= 1.0) kx = cmk(2.0 * asin(w), 0.0);
      else kx = cmk(2.0 * 1.5707963267948966, -2.0 * acosh(w));
    } else {
      kx = cmk(0.0, 2.0 * asinh(sqrt(-z.x)));
    }
  } else {
    double2 as = casin_p(csqrt_p(z));
    kx = cmk(2.0 * as.x, 2.0 * as.y);
  }
  // branch flip, setup_channels.m:211-215
  if (!is_real || k2e.x > 4.0) {
    bool flip = (z.x < 0.0 && z.y < 0.0) || (z.x > 1.0 && z.y <= 0.0);
    if (flip) kx = cneg(kx);
  }
  side.kx[a] = kx;
  side.lam[a] = cexp_i(kx);                         // exp(1i*kxdx), cal_smatrix_RGF.m:198
  side.sqrtmu[a] = csqrt_p(csin_p(kx));             // sqrt(sin(kxdx)), setup_channels.m:219
  side.isprop[a] = (z.x > 0.0 && z.x < 1.0) ? 1 : 0;  // setup_channels.m:195
}

// Single-CTA ordered compaction of the propagating flags (MATLAB find) and
// the reciprocity permutation ind_prop_conj (setup_channels.m:222-236).
__global__ void k_compact_prop(int64_t N, SideDev side, int conj_mode, int64_t ind_zero0) {
  __shared__ int64_t warp_tot[32];
  __shared__ int64_t base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int64_t c0 = 0; c0 < N; c0 += blockDim.x) {
    int64_t a = c0 + threadIdx.x;
    int f = (a < N) ? side.isprop[a] : 0;
    unsigned bal = __ballot_sync(0xffffffffu, f);
    int wpre = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int64_t off = 0, tot = 0;
    for (int w = 0; w < nwarp; w++) {
      if (w < warp) off += warp_tot[w];
      tot += warp_tot[w];
    }
    if (f) side.prop[base + off + wpre] = (int)a;
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
  const int64_t Np = base;
  if (threadIdx.x == 0) *side.nprop = (int)Np;
  // ind_prop_conj (0-based).  conj_mode: 0 none (Bloch ka != 0 or 3D),
  // 1 identity (real profiles), 2 periodic ka == 0.
  if (conj_mode == 1) {
    for (int64_t p = threadIdx.x; p < Np; p += blockDim.x) side.conj[p] = (int)p;
  } else if (conj_mode == 2) {
    __shared__ int zero_is_prop;
    if (threadIdx.x == 0) zero_is_prop = 0;
    __syncthreads();
    for (int64_t p = threadIdx.x; p < Np; p += blockDim.x)
      if (side.prop[p] == ind_zero0) zero_is_prop = 1;
    __syncthreads();
    bool flip_all = zero_is_prop || (Np % 2 == 0);
    for (int64_t p = threadIdx.x; p < Np; p += blockDim.x) {
      if (flip_all) side.conj[p] = (int)(Np - 1 - p);
      else side.conj[p] = (p == Np - 1) ? (int)(Np - 1) : (int)(Np - 2 - p);
    }
  }
}

// 1D transverse profile of mode a at site m (0-based), setup_channels.m:133-156
__device__ double2 profile_1d(int bc, int64_t n, double k, int64_t m, int dim) {
  switch (bc) {
    case RGF_BC_PERIODIC:
    case RGF_BC_BLOCH: {
      double s, c;
      sincos((double)(m + 1) * k, &s, &c);
      return cmk(c, s);  // normalisation applied by the caller
    }
    case RGF_BC_DIRICHLET:
      return cmk(sin((double)(m + 1) * k), 0.0);
    case RGF_BC_NEUMANN: {
      double v = cos(((double)m + 0.5) * k) - ((k == 0.0) ? (1.0 - sqrt(0.5)) : 0.0);
      return cmk(v * sqrt(2.0 / (double)n), 0.0);
    }
    case RGF_BC_DIRICHLET_NEUMANN:
      return cmk(sin((double)(m + 1) * k) * sqrt(2.0 / ((double)n + 0.5)), 0.0);
    default:  // NeumannDirichlet
      return cmk(cos(((double)m + 0.5) * k) * sqrt(2.0 / ((double)n + 0.5)), 0.0);
  }
}

// phi[m*ld + a] = transverse profile of mode a at site m (row-major).
__global__ void k_phi(Transverse tr, const double* k0, const double* k1, double2* phi, int64_t ld) {
  int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t m = blockIdx.y;
  for (; m < tr.N; m += gridDim.y) {
    if (a >= tr.N) return;
    double2 v;
    if (tr.dim == 2) {
      v = profile_1d(tr.bc, tr.n0, k0[a], m, 2);
      if (tr.bc == RGF_BC_PERIODIC || tr.bc == RGF_BC_BLOCH) {
        double s = sqrt((double)tr.n0);
        v = cmk(v.x / s, v.y / s);
      } else if (tr.bc == RGF_BC_DIRICHLET) {
        v.x = v.x * sqrt(2.0 / (double)(tr.n0 + 1));
      }
    } else {
      int64_t mx = m % tr.n0, my = m / tr.n0, ax = a % tr.n0, ay = a / tr.n0;
      if (tr.bc == RGF_BC_DIRICHLET) {
        double vx = sin((double)(mx + 1) * k0[ax]);
        double vy = sin((double)(my + 1) * k1[ay]) *
                    sqrt(4.0 / ((double)(tr.n0 + 1) * (double)(tr.n1 + 1)));
        v = cmk(vx * vy, 0.0);  // setup_channels_3D.m:123
      } else {
        double sx, cx, sy, cy;
        sincos((double)(mx + 1) * k0[ax], &sx, &cx);
        sincos((double)(my + 1) * k1[ay], &sy, &cy);
        double s = sqrt((double)(tr.n0 * tr.n1));
        v = cmul(cmk(cx, sx), cmk(cy / s, sy / s));  // setup_channels_3D.m:118
      }
    }
    phi[m * ld + a] = v;
  }
}

// ---- the transverse Laplacian (build_laplacian_1d.m) ------------------------
struct GradCol {
  int64_t rows[3];
  double2 vals[3];
  int cnt;
  __device__ void add(int64_t r, double2 v) {
    for (int q = 0; q < cnt; q++)
      if (rows[q] == r) {
        vals[q] = cadd(vals[q], v);
        return;
      }
    rows[cnt] = r;
    vals[cnt] = v;
    cnt++;
  }
};

// nonzeros of column j of grad_1 (build_laplacian_1d.m:48-69); coincident
// entries are summed, which gives the physical hopping sum for n = 1 Bloch.
__device__ GradCol grad_col(int64_t n, int bc, double ka, int64_t j) {
  GradCol g;
  g.cnt = 0;
  const double2 one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0);
  switch (bc) {
    case RGF_BC_PERIODIC:
    case RGF_BC_BLOCH: {
      g.add(j, one);
      if (j + 1 <= n - 1) g.add(j + 1, mone);
      if (j == n - 1) g.add(0, cmk(-cos(ka), sin(ka)));  // -exp(-1i*ka)
      break;
    }
    case RGF_BC_DIRICHLET:
      g.add(j, one);
      g.add(j + 1, mone);
      break;
    case RGF_BC_NEUMANN:
      if (j >= 1) g.add(j - 1, one);
      if (j <= n - 2) g.add(j, mone);
      break;
    case RGF_BC_DIRICHLET_NEUMANN:
      g.add(j, one);
      if (j + 1 < n) g.add(j + 1, mone);
      break;
    default:  // NeumannDirichlet
      g.add(j, mone);
      if (j >= 1) g.add(j - 1, one);
      break;
  }
  return g;
}

// (-Lap)[i][j] = (grad_1^H grad_1)[i][j]  (build_laplacian_1d.m:71-75)
__device__ double2 neg_lap(int64_t n, int bc, double ka, int64_t i, int64_t j) {
  GradCol gi = grad_col(n, bc, ka, i), gj = grad_col(n, bc, ka, j);
  double2 s = cmk(0.0, 0.0);
  for (int p = 0; p < gi.cnt; p++)
    for (int q = 0; q < gj.cnt; q++)
      if (gi.rows[p] == gj.rows[q]) s = cadd(s, cmul(cconj(gi.vals[p]), gj.vals[q]));
  return s;
}

__device__ inline void stencil_add_col(int64_t* cols, int& c, int64_t col) {
  for (int q = 0; q < c; q++)
    if (cols[q] == col) return;
  cols[c++] = col;
}

// Row i of A0 (<= 5 nonzeros): st_col[i*5+q] (-1 = unused), st_val[i*5+q].
__global__ void k_stencil(Transverse tr, int* st_col, double2* st_val) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= tr.N) return;
  int64_t cols[kMaxStencil];
  int c = 0;
  double kax = (tr.bc == RGF_BC_BLOCH) ? tr.ka0 : 0.0;
  double kay = (tr.bc == RGF_BC_BLOCH) ? tr.ka1 : 0.0;
  if (tr.dim == 2) {
    int64_t n = tr.n0;
    stencil_add_col(cols, c, i);
    if (i >= 1) stencil_add_col(cols, c, i - 1);
    if (i + 1 < n) stencil_add_col(cols, c, i + 1);
    if (i == 0) stencil_add_col(cols, c, n - 1);
    if (i == n - 1) stencil_add_col(cols, c, 0);
    for (int q = 0; q < kMaxStencil; q++) {
      if (q < c) {
        double2 v = neg_lap(n, tr.bc, kax, i, cols[q]);
        if (cols[q] == i) v.x += 2.0;  // cal_smatrix_RGF.m:209
        st_col[i * kMaxStencil + q] = (int)cols[q];
        st_val[i * kMaxStencil + q] = v;
      } else {
        st_col[i * kMaxStencil + q] = -1;
        st_val[i * kMaxStencil + q] = cmk(0.0, 0.0);
      }
    }
  } else {
    int64_t nx = tr.n0, ny = tr.n1, ix = i % nx, iy = i / nx;
    int64_t xs[3], ys[3];
    int cx = 0, cy = 0;
    stencil_add_col(xs, cx, ix);
    if (ix >= 1) stencil_add_col(xs, cx, ix - 1);
    if (ix + 1 < nx) stencil_add_col(xs, cx, ix + 1);
    if (ix == 0) stencil_add_col(xs, cx, nx - 1);
    if (ix == nx - 1) stencil_add_col(xs, cx, 0);
    stencil_add_col(ys, cy, iy);
    if (iy >= 1) stencil_add_col(ys, cy, iy - 1);
    if (iy + 1 < ny) stencil_add_col(ys, cy, iy + 1);
    if (iy == 0) stencil_add_col(ys, cy, ny - 1);
    if (iy == ny - 1) stencil_add_col(ys, cy, 0);
    // A0 = -kron(I, Lx) - kron(Ly, I) + 2I   (cal_smatrix_RGF_3D.m:224)
    int q = 0;
    double2 diag = cadd(neg_lap(nx, tr.bc, kax, ix, ix), neg_lap(ny, tr.bc, kay, iy, iy));
    diag.x += 2.0;
    st_col[i * kMaxStencil + q] = (int)i;
    st_val[i * kMaxStencil + q] = diag;
    q++;
    for (int p = 0; p < cx; p++)
      if (xs[p] != ix) {
        st_col[i * kMaxStencil + q] = (int)(xs[p] + nx * iy);
        st_val[i * kMaxStencil + q] = neg_lap(nx, tr.bc, kax, ix, xs[p]);
        q++;
      }
    for (int p = 0; p < cy; p++)
      if (ys[p] != iy) {
        st_col[i * kMaxStencil + q] = (int)(ix + nx * ys[p]);
        st_val[i * kMaxStencil + q] = neg_lap(ny, tr.bc, kay, iy, ys[p]);
        q++;
      }
    for (; q < kMaxStencil; q++) {
      st_col[i * kMaxStencil + q] = -1;
      st_val[i * kMaxStencil + q] = cmk(0.0, 0.0);
    }
  }
}

// Dense Lap = -grad^H grad, column-major (rgf_build_laplacian_1d).
__global__ void k_laplacian_dense(int64_t n, int bc, double ka, double2* A) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t j = blockIdx.y;
  if (i >= n) return;
  double2 v = cmk(0.0, 0.0);
  if (i == j || i + 1 == j || j + 1 == i || (i == 0 && j == n - 1) || (j == 0 && i == n - 1))
    v = cneg(neg_lap(n, bc, ka, i, j));
  A[j * n + i] = v;
}

// ---- host-side launchers ----------------------------------------------------
void launch_transverse(const Transverse& tr, double* k0, double* k1, cudaStream_t s) {
  int64_t n = tr.n0 > tr.n1 ? tr.n0 : tr.n1;
  k_transverse<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tr, k0, k1);
}
void launch_longitudinal(const Transverse& tr, const double* k0, const double* k1, double2 k2e,
                         const SideDev& side, cudaStream_t s) {
  k_longitudinal<<<(unsigned)((tr.N + 255) / 256), 256, 0, s>>>(tr, k0, k1, k2e, side);
}
void launch_compact(int64_t N, const SideDev& side, int conj_mode, int64_t ind_zero0, cudaStream_t s) {
  k_compact_prop<<<1, 1024, 0, s>>>(N, side, conj_mode, ind_zero0);
}
void launch_phi(const Transverse& tr, const double* k0, const double* k1, double2* phi, int64_t ld,
                cudaStream_t s) {
  dim3 grid((unsigned)((tr.N + 127) / 128), (unsigned)(tr.N < 4096 ? tr.N : 4096));
  k_phi<<<grid, 128, 0, s>>>(tr, k0, k1, phi, ld);
}
void launch_stencil(const Transverse& tr, int* st_col, double2* st_val, cudaStream_t s) {
  k_stencil<<<(unsigned)((tr.N + 127) / 128), 128, 0, s>>>(tr, st_col, st_val);
}
void launch_laplacian_dense(int64_t n, int bc, double ka, double2* A, cudaStream_t s) {
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)n);
  k_laplacian_dense<<<grid, 128, 0, s>>>(n, bc, ka, A);
}

}  // namespace rgf

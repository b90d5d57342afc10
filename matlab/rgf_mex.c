/*
 * rgf_mex.c -- MEX gateway from MATLAB to librgf (include/rgf.h).
 *
 * Build (MATLAB R2018a or later, interleaved complex API):
 *     mex -R2018a -I../include rgf_mex.c -L../rgf_b200 -lrgf
 *
 * Commands (called by the .m wrappers in this folder, which keep the
 * reference's function names and signatures):
 *   [S, ch] = rgf_mex('smatrix2d', syst, out, in)        cal_smatrix_RGF
 *   [S, ch] = rgf_mex('smatrix3d', syst, out, in)        cal_smatrix_RGF_3D
 *   [S, g]  = rgf_mex('grad2d', syst, out, in, D)        dS/d eps contracted with D
 *   [S, psi] = rgf_mex('fields2d', syst, out, in)        fields G B at every slice, [ny, nx, n_in]
 *   ch      = rgf_mex('channels2d', ny, BC, k0dx, epsL, epsR)
 *   ch      = rgf_mex('channels3d', nx, ny, BC, k0dx, epsL, epsR)
 *   A       = rgf_mex('laplacian', n, BC)                 build_laplacian_1d (dense)
 *
 * syst.epsilon is passed without a copy when it is already complex double;
 * a real epsilon is promoted to complex once.  Channel indices are 1-based
 * here and 0-based in the C ABI.  Every library status maps to a MATLAB
 * error with identifier rgf:<status> and the library's message.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "mex.h"
#include "rgf.h"

static rgf_handle H = NULL;

static void at_exit(void) {
  if (H) rgf_destroy(H);
  H = NULL;
}

static void fail(rgf_status st) {
  static const char* ids[] = {"rgf:ok",      "rgf:arg",  "rgf:nonfinite", "rgf:singular", "rgf:timeout",
                              "rgf:cuda",    "rgf:oom",  "rgf:nodevice",  "rgf:illcond"};
  mexErrMsgIdAndTxt(st >= 0 && st <= 8 ? ids[st] : "rgf:error", "%s", rgf_last_error());
}

/* RGF_ERR_ILLCOND leaves a result behind: a warning, as MATLAB's inv gives
 * for a matrix close to singular; every other failure is an error */
static void check(rgf_status st) {
  if (st == RGF_ERR_ILLCOND) mexWarnMsgIdAndTxt("rgf:illcond", "%s", rgf_last_error());
  else if (st != RGF_OK) fail(st);
}

static void ensure_handle(void) {
  if (!H) {
    check(rgf_create(0, &H));
    mexAtExit(at_exit);
  }
}

static double scalar(const mxArray* a, const char* what) {
  if (!a || !mxIsNumeric(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("rgf:arg", "%s must be a numeric scalar", what);
  return mxGetScalar(a);
}

static rgf_cplx cscalar(const mxArray* a, const char* what) {
  rgf_cplx z;
  if (!a || !mxIsNumeric(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("rgf:arg", "%s must be a numeric scalar", what);
  if (mxIsComplex(a) && mxIsDouble(a)) {
    const mxComplexDouble* p = mxGetComplexDoubles(a);
    z.re = p->real;
    z.im = p->imag;
  } else {
    z.re = mxGetScalar(a);
    z.im = 0.0;
  }
  return z;
}

static const mxArray* field(const mxArray* s, const char* name) {
  const mxArray* f = mxGetField(s, 0, name);
  if (!f) mexErrMsgIdAndTxt("rgf:arg", "syst.%s must be provided", name);
  return f;
}

/* BC: 'periodic' | 'Dirichlet'/'PEC' | 'Neumann'/'PMC' | 'DirichletNeumann'/'PECPMC'
 * | 'NeumannDirichlet'/'PMCPEC' | numeric k*a (Bloch), as setup_channels.m:98-159 */
static int32_t bc_of(const mxArray* a, double* ka) {
  *ka = 0.0;
  if (mxIsChar(a)) {
    char buf[64];
    mxGetString(a, buf, sizeof(buf));
    for (char* c = buf; *c; c++)
      if (*c >= 'A' && *c <= 'Z') *c += 'a' - 'A';
    if (!strcmp(buf, "periodic")) return RGF_BC_PERIODIC;
    if (!strcmp(buf, "dirichlet") || !strcmp(buf, "pec")) return RGF_BC_DIRICHLET;
    if (!strcmp(buf, "neumann") || !strcmp(buf, "pmc")) return RGF_BC_NEUMANN;
    if (!strcmp(buf, "dirichletneumann") || !strcmp(buf, "pecpmc")) return RGF_BC_DIRICHLET_NEUMANN;
    if (!strcmp(buf, "neumanndirichlet") || !strcmp(buf, "pmcpec")) return RGF_BC_NEUMANN_DIRICHLET;
    if (!strcmp(buf, "bloch"))
      mexErrMsgIdAndTxt("rgf:arg", "To use Bloch periodic boundary condition, set BC to k*a where k is the Bloch wave number and a is the periodicity");
    mexErrMsgIdAndTxt("rgf:arg", "BC = %s is not an eligible option", buf);
  }
  *ka = scalar(a, "BC");
  return RGF_BC_BLOCH;
}

/* epsilon as interleaved complex; *tmp receives a promoted copy to destroy */
static const rgf_cplx* eps_of(const mxArray* e, mxArray** tmp) {
  *tmp = NULL;
  if (!mxIsNumeric(e)) mexErrMsgIdAndTxt("rgf:arg", "syst.epsilon must be a numeric array");
  if (mxIsDouble(e) && mxIsComplex(e)) return (const rgf_cplx*)mxGetComplexDoubles(e);
  *tmp = mxDuplicateArray(e);
  if (!mxIsDouble(*tmp)) mexErrMsgIdAndTxt("rgf:arg", "syst.epsilon must be double");
  if (!mxMakeArrayComplex(*tmp)) mexErrMsgIdAndTxt("rgf:arg", "cannot promote syst.epsilon to complex");
  return (const rgf_cplx*)mxGetComplexDoubles(*tmp);
}

/* one side's list (field `name` of out / in): NULL = not given; otherwise a
 * 1-based -> 0-based copy.  The upper bound N_prop is checked by the library
 * with the reference's message (cal_smatrix_RGF.m:108-116). */
static int64_t* list_of(const mxArray* a, const char* kind, const char* name, int64_t* n) {
  *n = 0;
  if (!a) return NULL;
  const mwSize k = mxGetNumberOfElements(a);
  int64_t* out = (int64_t*)mxMalloc(sizeof(int64_t) * (k ? k : 1));
  const double* d = mxGetDoubles(a);
  for (mwSize i = 0; i < k; i++) {
    if (!d || d[i] != (double)(int64_t)d[i] || d[i] < 1)
      mexErrMsgIdAndTxt("rgf:arg", "%s.%s, when specified, must be an array of positive integers", kind, name);
    out[i] = (int64_t)d[i] - 1;
  }
  *n = (int64_t)k;
  return out;
}

/* out / in: cell of 'left'/'right' or struct of index lists (cal_smatrix_RGF.m:103-178) */
static void side_req(const mxArray* a, const char* kind, const int64_t** L, int64_t* nL, const int64_t** R,
                     int64_t* nR) {
  *L = *R = NULL;
  *nL = *nR = 0;
  if (mxIsCell(a)) {  /* cal_smatrix_RGF.m:120-135 */
    for (mwSize i = 0; i < mxGetNumberOfElements(a); i++) {
      const mxArray* c = mxGetCell(a, i);
      char buf[16] = {0};
      if (!c || !mxIsChar(c)) {
        mexWarnMsgIdAndTxt("rgf:ignored",
                           "element %s{%d} has wrong format and is ignored; should be one of {'left', 'right', 'L', 'R'}",
                           kind, (int)i + 1);
        continue;
      }
      mxGetString(c, buf, sizeof(buf));
      if (!strcmp(buf, "left") || !strcmp(buf, "L")) *nL = RGF_ALL;
      else if (!strcmp(buf, "right") || !strcmp(buf, "R")) *nR = RGF_ALL;
      else
        mexWarnMsgIdAndTxt("rgf:ignored", "element %s{%d} = %s ignored; should be one of {'left', 'right', 'L', 'R'}",
                           kind, (int)i + 1, buf);
    }
    return;
  }
  if (!mxIsStruct(a)) mexErrMsgIdAndTxt("rgf:arg", "input argument '%s' must be a structure or a cell array", kind);
  char fl[16], fr[16];
  snprintf(fl, sizeof(fl), "ind_%s_L", kind);
  snprintf(fr, sizeof(fr), "ind_%s_R", kind);
  *L = list_of(mxGetField(a, 0, fl), kind, fl, nL);
  *R = list_of(mxGetField(a, 0, fr), kind, fr, nR);
}

static mxArray* cplx_vec(const rgf_cplx* v, mwSize n) {
  mxArray* a = mxCreateDoubleMatrix(n, 1, mxCOMPLEX);
  memcpy(mxGetComplexDoubles(a), v, sizeof(rgf_cplx) * n);
  return a;
}

static mxArray* index_vec(const int64_t* v, mwSize n) {
  mxArray* a = mxCreateDoubleMatrix(n, 1, mxREAL);
  double* d = mxGetDoubles(a);
  for (mwSize i = 0; i < n; i++) d[i] = (double)(v[i] + 1);
  return a;
}

/* channels struct: kydx (and kxdx in 3D), L / R with N_prop, kxdx, ind_prop,
 * sqrt_mu, ind_prop_conj (setup_channels.m:30-82); fun_phi is added by the .m
 * wrapper */
typedef struct {
  rgf_channels c;
  double *ky, *kx;
  rgf_cplx *kxL, *kxR, *muL, *muR;
  int64_t *ipL, *ipR, *icL, *icR;
} chbuf;

static void chbuf_init(chbuf* b, int64_t N) {
  memset(b, 0, sizeof(*b));
  b->ky = (double*)mxCalloc(N, sizeof(double));
  b->kx = (double*)mxCalloc(N, sizeof(double));
  b->kxL = (rgf_cplx*)mxCalloc(N, sizeof(rgf_cplx));
  b->kxR = (rgf_cplx*)mxCalloc(N, sizeof(rgf_cplx));
  b->muL = (rgf_cplx*)mxCalloc(N, sizeof(rgf_cplx));
  b->muR = (rgf_cplx*)mxCalloc(N, sizeof(rgf_cplx));
  b->ipL = (int64_t*)mxCalloc(N, sizeof(int64_t));
  b->ipR = (int64_t*)mxCalloc(N, sizeof(int64_t));
  b->icL = (int64_t*)mxCalloc(N, sizeof(int64_t));
  b->icR = (int64_t*)mxCalloc(N, sizeof(int64_t));
  b->c.kydx = b->ky;
  b->c.kxdx_t = b->kx;
  b->c.kxdx_L = b->kxL;
  b->c.kxdx_R = b->kxR;
  b->c.sqrt_mu_L = b->muL;
  b->c.sqrt_mu_R = b->muR;
  b->c.ind_prop_L = b->ipL;
  b->c.ind_prop_R = b->ipR;
  b->c.ind_prop_conj_L = b->icL;
  b->c.ind_prop_conj_R = b->icR;
}

static mxArray* chbuf_struct(const chbuf* b, int64_t N, int dim) {
  const char* top[] = {"kydx", "kxdx", "L", "R"};
  const char* side[] = {"N_prop", "kxdx", "ind_prop", "sqrt_mu", "ind_prop_conj"};
  mxArray* s = mxCreateStructMatrix(1, 1, dim == 3 ? 4 : 3, dim == 3 ? top : (const char*[]){"kydx", "L", "R"});
  mxArray* ky = mxCreateDoubleMatrix(N, 1, mxREAL);
  memcpy(mxGetDoubles(ky), b->ky, sizeof(double) * N);
  mxSetField(s, 0, "kydx", ky);
  if (dim == 3) {
    mxArray* kx = mxCreateDoubleMatrix(N, 1, mxREAL);
    memcpy(mxGetDoubles(kx), b->kx, sizeof(double) * N);
    mxSetField(s, 0, "kxdx", kx);
  }
  for (int k = 0; k < 2; k++) {
    const int64_t np = k ? b->c.N_prop_R : b->c.N_prop_L;
    if (k == 1 && np < 0) {  /* one-sided set-up: channels.R.N_prop = NaN (setup_channels.m:171-174) */
      mxArray* t = mxCreateStructMatrix(1, 1, 1, side);
      mxSetField(t, 0, "N_prop", mxCreateDoubleScalar(NAN));
      mxSetField(s, 0, "R", t);
      continue;
    }
    mxArray* t = mxCreateStructMatrix(1, 1, b->c.has_prop_conj ? 5 : 4, side);
    mxSetField(t, 0, "N_prop", mxCreateDoubleScalar((double)np));
    mxSetField(t, 0, "kxdx", cplx_vec(k ? b->kxR : b->kxL, N));
    mxSetField(t, 0, "ind_prop", index_vec(k ? b->ipR : b->ipL, np > 0 ? np : 0));
    mxSetField(t, 0, "sqrt_mu", cplx_vec(k ? b->muR : b->muL, np > 0 ? np : 0));
    if (b->c.has_prop_conj) mxSetField(t, 0, "ind_prop_conj", index_vec(k ? b->icR : b->icL, np > 0 ? np : 0));
    mxSetField(s, 0, k ? "R" : "L", t);
  }
  return s;
}

/* grad: 1 = gradient (prhs[4] = D), 2 = fields */
static void smatrix_cmd(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[], int dim, int grad) {
  if (nrhs < 4 + (grad == 1)) mexErrMsgIdAndTxt("rgf:arg", "not enough input arguments");
  const mxArray* syst = prhs[1];
  if (!mxIsStruct(syst)) mexErrMsgIdAndTxt("rgf:arg", "syst must be a structure");
  const mxArray* e = field(syst, "epsilon");
  mxArray* tmp = NULL;
  const rgf_cplx* eps = eps_of(e, &tmp);
  const mwSize* dims = mxGetDimensions(e);
  const mwSize nd = mxGetNumberOfDimensions(e);
  rgf_request req;
  side_req(prhs[2], "out", &req.ind_out_L, &req.n_out_L, &req.ind_out_R, &req.n_out_R);
  side_req(prhs[3], "in", &req.ind_in_L, &req.n_in_L, &req.ind_in_R, &req.n_in_R);
  int64_t no = 0, ni = 0, N = 0, L = 0;
  rgf_syst2d s2;
  rgf_syst3d s3;
  double ka;
  if (dim == 2) {
    memset(&s2, 0, sizeof(s2));
    s2.ny = dims[0];
    s2.nx = nd > 1 ? dims[1] : 1;
    s2.epsilon = eps;
    s2.epsilon_L = cscalar(field(syst, "epsilon_L"), "syst.epsilon_L");
    s2.epsilon_R = cscalar(field(syst, "epsilon_R"), "syst.epsilon_R");
    s2.k0dx = cscalar(field(syst, "k0dx"), "syst.k0dx");
    s2.yBC = bc_of(field(syst, "yBC"), &ka);
    s2.ka = ka;
    N = s2.ny;
    L = s2.nx;
    check(rgf_smatrix_size_2d(H, &s2, &req, &no, &ni));
  } else {
    memset(&s3, 0, sizeof(s3));
    s3.nx = dims[0];
    s3.ny = nd > 1 ? dims[1] : 1;
    s3.nz = nd > 2 ? dims[2] : 1;
    s3.epsilon = eps;
    s3.epsilon_L = cscalar(field(syst, "epsilon_L"), "syst.epsilon_L");
    s3.epsilon_R = cscalar(field(syst, "epsilon_R"), "syst.epsilon_R");
    s3.k0dx = cscalar(field(syst, "k0dx"), "syst.k0dx");
    const mxArray* bc = field(syst, "xyBC");
    if (mxIsNumeric(bc) && mxGetNumberOfElements(bc) == 2) {
      s3.xyBC = RGF_BC_BLOCH;
      s3.kxa = mxGetDoubles(bc)[0];
      s3.kya = mxGetDoubles(bc)[1];
    } else {
      s3.xyBC = bc_of(bc, &ka);
    }
    N = s3.nx * s3.ny;
    L = s3.nz;
    check(rgf_smatrix_size_3d(H, &s3, &req, &no, &ni));
  }
  plhs[0] = mxCreateDoubleMatrix(no, ni, mxCOMPLEX);
  rgf_cplx* S = (rgf_cplx*)mxGetComplexDoubles(plhs[0]);
  if (grad == 2) {  /* fields: [ny, nx, n_in] (2D) */
    const mwSize fd[3] = {(mwSize)N, (mwSize)L, (mwSize)ni};
    mxArray* psi = mxCreateNumericArray(3, fd, mxDOUBLE_CLASS, mxCOMPLEX);
    rgf_status st = rgf_fields_2d(H, &s2, &req, NULL, no ? S : NULL, no > 0 ? no : 1,
                                  (rgf_cplx*)mxGetComplexDoubles(psi), 0);
    if (tmp) mxDestroyArray(tmp);
    check(st);
    if (nlhs > 1) plhs[1] = psi;
    else mxDestroyArray(psi);
    return;
  }
  if (grad) {
    const mxArray* Da = prhs[4];
    if (!mxIsDouble(Da) || mxGetM(Da) != (mwSize)no || mxGetN(Da) != (mwSize)ni)
      mexErrMsgIdAndTxt("rgf:arg", "D must be a double matrix of the size of S");
    mxArray* Dt = mxDuplicateArray(Da);
    if (!mxIsComplex(Dt)) mxMakeArrayComplex(Dt);
    mxArray* g = mxCreateNumericArray(nd, dims, mxDOUBLE_CLASS, mxCOMPLEX);
    rgf_status st = dim == 2 ? rgf_smatrix_grad_2d(H, &s2, &req, NULL, (const rgf_cplx*)mxGetComplexDoubles(Dt),
                                                   no > 0 ? no : 1, no ? S : NULL, no > 0 ? no : 1,
                                                   (rgf_cplx*)mxGetComplexDoubles(g), 0)
                             : rgf_smatrix_grad_3d(H, &s3, &req, NULL, (const rgf_cplx*)mxGetComplexDoubles(Dt),
                                                   no > 0 ? no : 1, no ? S : NULL, no > 0 ? no : 1,
                                                   (rgf_cplx*)mxGetComplexDoubles(g), 0);
    mxDestroyArray(Dt);
    if (tmp) mxDestroyArray(tmp);
    check(st);
    if (nlhs > 1) plhs[1] = g;
    else mxDestroyArray(g);
    (void)N;
    (void)L;
    return;
  }
  chbuf cb;
  chbuf_init(&cb, N);
  rgf_status st = dim == 2 ? rgf_smatrix_2d(H, &s2, &req, NULL, no ? S : NULL, no > 0 ? no : 1, &cb.c)
                           : rgf_smatrix_3d(H, &s3, &req, NULL, no ? S : NULL, no > 0 ? no : 1, &cb.c);
  if (tmp) mxDestroyArray(tmp);
  check(st);
  if (nlhs > 1) plhs[1] = chbuf_struct(&cb, N, dim);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[32];
  if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], cmd, sizeof(cmd)))
    mexErrMsgIdAndTxt("rgf:arg", "first argument must be a command string");
  ensure_handle();
  if (!strcmp(cmd, "smatrix2d")) {
    smatrix_cmd(nlhs, plhs, nrhs, prhs, 2, 0);
  } else if (!strcmp(cmd, "smatrix3d")) {
    smatrix_cmd(nlhs, plhs, nrhs, prhs, 3, 0);
  } else if (!strcmp(cmd, "grad2d")) {
    smatrix_cmd(nlhs, plhs, nrhs, prhs, 2, 1);
  } else if (!strcmp(cmd, "fields2d")) {
    smatrix_cmd(nlhs, plhs, nrhs, prhs, 2, 2);
  } else if (!strcmp(cmd, "channels2d") || !strcmp(cmd, "channels3d")) {
    const int dim = cmd[8] == '3' ? 3 : 2;
    const int a0 = dim == 3 ? 2 : 1;
    if (nrhs < a0 + 4) mexErrMsgIdAndTxt("rgf:arg", "not enough input arguments");
    const int64_t n0 = (int64_t)scalar(prhs[1], "size"), n1 = dim == 3 ? (int64_t)scalar(prhs[2], "ny") : 1;
    double ka = 0.0, kya = 0.0;
    int32_t bc;
    if (dim == 3 && mxIsNumeric(prhs[a0 + 1]) && mxGetNumberOfElements(prhs[a0 + 1]) == 2) {
      bc = RGF_BC_BLOCH;
      ka = mxGetDoubles(prhs[a0 + 1])[0];
      kya = mxGetDoubles(prhs[a0 + 1])[1];
    } else {
      bc = bc_of(prhs[a0 + 1], &ka);
    }
    const rgf_cplx k0dx = cscalar(prhs[a0 + 2], "k0dx");
    const rgf_cplx eL = cscalar(prhs[a0 + 3], "epsilon_L");
    const int two = nrhs > a0 + 4;
    const rgf_cplx eR = two ? cscalar(prhs[a0 + 4], "epsilon_R") : eL;
    chbuf cb;
    chbuf_init(&cb, n0 * n1);
    check(dim == 2 ? rgf_setup_channels_2d(H, n0, bc, ka, k0dx, eL, eR, two, &cb.c)
                   : rgf_setup_channels_3d(H, n0, n1, bc, ka, kya, k0dx, eL, eR, two, &cb.c));
    plhs[0] = chbuf_struct(&cb, n0 * n1, dim);
  } else if (!strcmp(cmd, "laplacian")) {
    if (nrhs < 3) mexErrMsgIdAndTxt("rgf:arg", "not enough input arguments");
    const int64_t n = (int64_t)scalar(prhs[1], "n");
    double ka;
    const int32_t bc = bc_of(prhs[2], &ka);
    plhs[0] = mxCreateDoubleMatrix(n, n, mxCOMPLEX);
    check(rgf_build_laplacian_1d(H, n, bc, ka, (rgf_cplx*)mxGetComplexDoubles(plhs[0])));
  } else {
    mexErrMsgIdAndTxt("rgf:arg", "unknown command '%s'", cmd);
  }
}

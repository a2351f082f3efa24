// FCCD matrix-free pressure-Poisson solve for sm_100a (the reference's
// PPESolverFCCDMatrixFree on its default path).
//
// Operator (src/twophase/ppe/fccd_matrixfree.py:378-428,762-829; face
// gradient ccd/fccd.py:243-277):
//   L p = sum_a D_a[ (1/rho)_f G_a p ],
//   G_a p at face f (nodes f, f+1) = (p[f+1] - p[f]) / H - (H/24) (q[f+1] - q[f]),
//   q = the CCD second derivative of p along a, (1/rho)_f = 2/(rho[f] + rho[f+1]);
//   wall axis: node i in 1..N-1 gets (F[i] - F[i-1]) / w_i, node 0 gets
//   F[0] / w_0 and node N gets -F[N-1] / w_N (w = control-volume widths);
//   periodic axis: node i < N gets (F[i] - F[i-1 mod N]) / H, the image node N
//   the value of node 0, and q, p wrap over the N unique nodes.
// The periodic image nodes of the input are synchronised first (one gather:
// an image takes its direct source's value, the first periodic axis claiming
// a node); the pinned row returns p[pin] and an image row p[img] - p[src].
//
// Kernels per apply: the image gather (periodic axes only), one CCD line
// solve per axis for q (the library's CCD kernels, d2 output only), and ONE
// fused kernel for the face gradients, the face coefficients (from rho on
// the fly), the weighted divergence of all axes, the pinned and image rows
// and, inside GMRES, the residual b - L x.  The solve is SciPy's
// left-preconditioned restarted GMRES (gmres.cuh; restart 20 when none is
// given, SciPy's default) with the Jacobi or no preconditioner.
#include "tpf_common.cuh"
#include "gmres.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

struct tpf_fccd_ppe {
  int ndim = 0;
  int nn[3] = {1, 1, 1};     // nodes per axis
  int N[3] = {0, 0, 0};      // cells per axis
  int per[3] = {0, 0, 0};
  int any_per = 0;
  int pin = 0;
  int ndof = 0;
  tpf_fccd_ppe_options o{};
  double invH[3] = {0, 0, 0};
  double H24[3] = {0, 0, 0};
  double hmin[3] = {0, 0, 0};
  double* iw[3] = {nullptr, nullptr, nullptr};   // 1 / control-volume width per node (wall axes)
  tpf_ccd_plan* plan[3] = {nullptr, nullptr, nullptr};
  double* rho = nullptr;        // prepared density (copy)
  double* diag_inv = nullptr;   // Jacobi inverse diagonal
  double* psync = nullptr;      // operator input with images synchronised
  double* q[3] = {nullptr, nullptr, nullptr};
  bool prepared = false;
  bool warmed = false;
  // GMRES workspace
  double* V = nullptr;
  int V_cols = 0;
  double* gm = nullptr;
  GmState* gst = nullptr;
  double* part = nullptr;
  int part_len = 0;
  double *b = nullptr, *x = nullptr, *r = nullptr, *w = nullptr, *t = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;
  long long key[6] = {};
  int ew_blocks = 0;
  std::vector<void*> allocs;
};

namespace {

struct FDims {
  int nd;
  int nn0, nn1, nn2;
  int N0, N1, N2;
  int per0, per1, per2;
  int pin;
  int ndof;
};

FDims dims_of(const tpf_fccd_ppe* h) {
  FDims d;
  d.nd = h->ndim;
  d.nn0 = h->nn[0]; d.nn1 = h->nn[1]; d.nn2 = h->nn[2];
  d.N0 = h->N[0]; d.N1 = h->N[1]; d.N2 = h->N[2];
  d.per0 = h->per[0]; d.per1 = h->per[1]; d.per2 = h->per[2];
  d.pin = h->pin;
  d.ndof = h->ndof;
  return d;
}

__device__ __forceinline__ void coords_of(const FDims& d, int i, int& c0, int& c1, int& c2) {
  c2 = i % d.nn2;
  const int t = i / d.nn2;
  c1 = t % d.nn1;
  c0 = t / d.nn1;
}

// the node an image node copies (the first periodic axis at its image
// coordinate claims it; fccd_matrixfree.py:310-348), or i itself
__device__ __forceinline__ int direct_source(const FDims& d, int i) {
  int c0, c1, c2;
  coords_of(d, i, c0, c1, c2);
  if (d.per0 && c0 == d.N0) return i - d.N0 * d.nn1 * d.nn2;
  if (d.nd > 1 && d.per1 && c1 == d.N1) return i - d.N1 * d.nn2;
  if (d.nd > 2 && d.per2 && c2 == d.N2) return i - d.N2;
  return i;
}

__global__ void fccd_sync_kernel(FDims d, const double* __restrict__ in, double* __restrict__ out,
                                 const int* done) {
  if (done && *done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ndof; i += gridDim.x * blockDim.x)
    out[i] = in[direct_source(d, i)];
}

struct AxisArgs {
  const double* q;
  const double* iw;
  double invH;
  double H24;
  int stride;     // element stride of the axis
  int N;          // cells
  int per;
};

struct DivArgs {
  FDims d;
  AxisArgs ax[3];
  const double* u;      // operator input, images synchronised
  const double* p;      // unsynchronised input (pinned and image rows)
  const double* rho;
  const double* b;      // residual mode: out = b - L p
  double* out;
};

// face flux (1/rho)_f G p at face f (nodes at offsets lo, hi)
__device__ __forceinline__ double face_flux(const DivArgs& A, const AxisArgs& X, int lo, int hi, int rlo, int rhi) {
  const double g = __dsub_rn(__dmul_rn(__dsub_rn(A.u[hi], A.u[lo]), X.invH),
                             __dmul_rn(X.H24, __dsub_rn(X.q[hi], X.q[lo])));
  const double c = __ddiv_rn(2.0, __dadd_rn(A.rho[rlo], A.rho[rhi]));
  return __dmul_rn(c, g);
}

__global__ void __launch_bounds__(256) fccd_div_kernel(const __grid_constant__ DivArgs A, const int* done) {
  if (done && *done) return;
  const FDims& d = A.d;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ndof; i += gridDim.x * blockDim.x) {
    int c[3];
    coords_of(d, i, c[0], c[1], c[2]);
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a >= d.nd) break;
      const AxisArgs& X = A.ax[a];
      const int ci = c[a], n = X.N, s = X.stride;
      const int base = i - ci * s;   // node 0 of this line
      if (X.per) {
        // unique node k = ci (image node N takes node 0's value)
        const int k = (ci == n) ? 0 : ci;
        const int km = (k == 0) ? n - 1 : k - 1;
        const int kp = (k + 1 == n) ? 0 : k + 1;
        // face k: nodes k, k+1 (wrapped for u, q; rho at k+1 unwrapped)
        const double Fk = face_flux(A, X, base + k * s, base + kp * s, base + k * s, base + (k + 1) * s);
        const double Fm = face_flux(A, X, base + km * s, base + k * s, base + km * s, base + (km + 1) * s);
        acc = __dadd_rn(acc, __dmul_rn(__dsub_rn(Fk, Fm), X.invH));
      } else {
        const double iwv = X.iw[ci];
        if (ci == 0) {
          const double F0 = face_flux(A, X, base, base + s, base, base + s);
          acc = __dadd_rn(acc, __dmul_rn(F0, iwv));
        } else if (ci == n) {
          const double Fl = face_flux(A, X, i - s, i, i - s, i);
          acc = __dsub_rn(acc, __dmul_rn(Fl, iwv));
        } else {
          const double Fh = face_flux(A, X, i, i + s, i, i + s);
          const double Fl = face_flux(A, X, i - s, i, i - s, i);
          acc = __dadd_rn(acc, __dmul_rn(__dsub_rn(Fh, Fl), iwv));
        }
      }
    }
    double v = acc;
    if (i == d.pin) v = A.p[i];
    if (d.per0 | d.per1 | d.per2) {
      const int src = direct_source(d, i);
      if (src != i) v = __dsub_rn(A.p[i], A.p[src]);
    }
    A.out[i] = A.b ? __dsub_rn(A.b[i], v) : v;
  }
}

// diag = -sum_a 2 / (rho h_min_a^2), diag[pin] = 1, inverse guarded
// (fccd_matrixfree_helpers.py:251-265)
__global__ void fccd_diag_kernel(FDims d, const double* __restrict__ rho, double h0, double h1, double h2,
                                 double* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ndof; i += gridDim.x * blockDim.x) {
    const double r = rho[i];
    double diag = 0.0;
    diag = __dsub_rn(diag, __ddiv_rn(2.0, __dmul_rn(__dmul_rn(r, h0), h0)));
    if (d.nd > 1) diag = __dsub_rn(diag, __ddiv_rn(2.0, __dmul_rn(__dmul_rn(r, h1), h1)));
    if (d.nd > 2) diag = __dsub_rn(diag, __ddiv_rn(2.0, __dmul_rn(__dmul_rn(r, h2), h2)));
    if (i == d.pin) diag = 1.0;
    dinv[i] = __ddiv_rn(1.0, fabs(diag) > 1.0e-30 ? diag : 1.0);
  }
}

__global__ void fccd_jacobi_kernel(int n, int pin, const double* __restrict__ dinv, const double* __restrict__ r,
                                   double* __restrict__ z, const int* done) {
  if (done && *done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    z[i] = (i == pin) ? 0.0 : __dmul_rn(r[i], dinv[i]);
}

// b = rhs with the pinned and image rows zeroed
__global__ void fccd_rhs_kernel(FDims d, const double* __restrict__ rhs, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ndof; i += gridDim.x * blockDim.x) {
    double v = rhs[i];
    if (i == d.pin || direct_source(d, i) != i) v = 0.0;
    b[i] = v;
  }
}

// x0 = p_init with images synchronised and pin zeroed
__global__ void fccd_x0_kernel(FDims d, const double* __restrict__ p_init, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ndof; i += gridDim.x * blockDim.x)
    x[i] = (i == d.pin) ? 0.0 : p_init[direct_source(d, i)];
}

__global__ void fccd_pin0_kernel(int n, int pin, const double* __restrict__ src, double* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = (i == pin) ? 0.0 : src[i];
}

template <typename T>
int falloc(tpf_fccd_ppe* h, T** p, size_t n) {
  if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    tpf::set_error("cudaMalloc of %zu bytes failed", n * sizeof(T));
    return TPF_ECUDA;
  }
  h->allocs.push_back(*p);
  return TPF_OK;
}

void line_split(const tpf_fccd_ppe* h, int a, int64_t& outer, int64_t& inner) {
  outer = 1;
  inner = 1;
  for (int k = 0; k < a; ++k) outer *= h->nn[k];
  for (int k = a + 1; k < h->ndim; ++k) inner *= h->nn[k];
}

int axis_stride(const tpf_fccd_ppe* h, int a) {
  int s = 1;
  for (int k = a + 1; k < h->ndim; ++k) s *= h->nn[k];
  return s;
}

// out = L in (b == nullptr) or out = b - L in
int fccd_apply(tpf_fccd_ppe* h, const double* in, double* out, const double* b, cudaStream_t s, const int* done) {
  const FDims d = dims_of(h);
  const double* u = in;
  if (h->any_per) {
    fccd_sync_kernel<<<h->ew_blocks, 256, 0, s>>>(d, in, h->psync, done);
    u = h->psync;
  }
  for (int a = 0; a < h->ndim; ++a) {
    int64_t outer, inner;
    line_split(h, a, outer, inner);
    const int st = tpf_ccd_apply(h->plan[a], outer, inner, u, nullptr, h->q[a], nullptr, nullptr, 0, s);
    if (st) return st;
  }
  DivArgs A{};
  A.d = d;
  for (int a = 0; a < 3; ++a) {
    A.ax[a].q = (a < h->ndim) ? h->q[a] : nullptr;
    A.ax[a].iw = (a < h->ndim) ? h->iw[a] : nullptr;
    A.ax[a].invH = h->invH[a];
    A.ax[a].H24 = h->H24[a];
    A.ax[a].stride = (a < h->ndim) ? axis_stride(h, a) : 1;
    A.ax[a].N = h->N[a];
    A.ax[a].per = h->per[a];
  }
  A.u = u;
  A.p = in;
  A.rho = h->rho;
  A.b = b;
  A.out = out;
  fccd_div_kernel<<<h->ew_blocks, 256, 0, s>>>(A, done);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int fccd_precond(tpf_fccd_ppe* h, const double* in, double* out, cudaStream_t s, const int* done) {
  if (h->o.precond == TPF_PRECOND_JACOBI) {
    fccd_jacobi_kernel<<<h->ew_blocks, 256, 0, s>>>(h->ndof, h->pin, h->diag_inv, in, out, done);
    TPF_CUDA_TRY(cudaGetLastError());
  } else {
    TPF_CUDA_TRY(cudaMemcpyAsync(out, in, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice, s));
  }
  return TPF_OK;
}

int ensure_work(tpf_fccd_ppe* h) {
  const int m = h->o.restart;
  if (h->V && h->V_cols >= m + 1) return TPF_OK;
  if (h->V) {
    cudaFree(h->V);
    cudaFree(h->gm);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->V), h->allocs.end());
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->gm), h->allocs.end());
    h->V = nullptr;
    h->gm = nullptr;
    if (h->exec) { cudaGraphExecDestroy(h->exec); h->exec = nullptr; }
  }
  int st;
  if ((st = falloc(h, &h->V, (size_t)(m + 1) * h->ndof))) return st;
  const size_t gm_len = (size_t)m * (m + 2) + 2 * (size_t)m + (size_t)(m + 1) * 4 + 8;
  if ((st = falloc(h, &h->gm, gm_len))) return st;
  h->V_cols = m + 1;
  const int need = (m + 2) * std::max(1, 4 * tpf::sm_count());
  if (h->part_len < need) {
    if (h->part) {
      cudaFree(h->part);
      h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->part), h->allocs.end());
      h->part = nullptr;
    }
    if ((st = falloc(h, &h->part, (size_t)need))) return st;
    h->part_len = need;
  }
  return TPF_OK;
}

int check_options(const tpf_fccd_ppe_options* o) {
  TPF_CHECK_ARG(o != nullptr, "NULL options");
  TPF_CHECK_ARG(o->precond == TPF_PRECOND_JACOBI || o->precond == TPF_PRECOND_NONE,
                "FCCD PPE supports preconditioner='jacobi'|'none'");
  TPF_CHECK_ARG(o->tol > 0.0 && std::isfinite(o->tol), "tolerance must be > 0");
  TPF_CHECK_ARG(o->maxiter >= 0, "maxiter must be >= 0");
  TPF_CHECK_ARG(o->restart >= 1 && o->restart <= 1024, "restart must be in [1, 1024]");
  return TPF_OK;
}

}  // namespace

extern "C" {

void tpf_fccd_ppe_default_options(tpf_fccd_ppe_options* o) {
  if (!o) return;
  o->tol = 1e-8;
  o->maxiter = 500;
  o->restart = 20;
  o->precond = TPF_PRECOND_NONE;
}

int tpf_fccd_ppe_create(tpf_fccd_ppe** out, int ndim, const int64_t* N, const double* const* coords,
                        const double* h_ccd, const int* periodic, int64_t pin, const tpf_fccd_ppe_options* o) {
  TPF_CHECK_ARG(out && N && coords && h_ccd && periodic, "NULL argument");
  *out = nullptr;
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  int st = check_options(o);
  if (st) return st;
  int64_t ndof = 1;
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(N[a] >= 1, "N must be >= 1");
    TPF_CHECK_ARG(coords[a] != nullptr, "NULL coordinate array");
    TPF_CHECK_ARG(h_ccd[a] > 0.0, "CCD spacing must be > 0");
    TPF_CHECK_ARG(!periodic[a] || N[a] >= 3, "a periodic axis needs at least 3 cells");
    ndof *= N[a] + 1;
  }
  TPF_CHECK_ARG(ndof < (int64_t)1 << 31, "grid too large for 32-bit node indices");
  TPF_CHECK_ARG(pin >= 0 && pin < ndof, "pin DOF out of range");
  tpf_fccd_ppe* h = new tpf_fccd_ppe();
  h->ndim = ndim;
  h->o = *o;
  h->pin = (int)pin;
  h->ndof = (int)ndof;
  for (int a = 0; a < ndim; ++a) {
    h->N[a] = (int)N[a];
    h->nn[a] = (int)N[a] + 1;
    h->per[a] = periodic[a] ? 1 : 0;
    h->any_per |= h->per[a];
  }
  auto fail = [&](int code) {
    tpf_fccd_ppe_destroy(h);
    return code;
  };
  for (int a = 0; a < ndim; ++a) {
    const int nn = h->nn[a];
    const double* c = coords[a];
    // FCCD face weights: H = x[1] - x[0], 1/H and H/24 as the reference forms them
    const double H = c[1] - c[0];
    h->invH[a] = 1.0 / H;
    h->H24[a] = H / 24.0;
    // control-volume widths (fccd_matrixfree_helpers.py:35-52)
    std::vector<double> iw(nn);
    double hmin = INFINITY;
    for (int i = 0; i + 1 < nn; ++i) hmin = std::min(hmin, c[i + 1] - c[i]);
    for (int i = 0; i < nn; ++i) {
      double w;
      if (i == 0) w = 0.5 * (c[1] - c[0]);
      else if (i == nn - 1) w = 0.5 * (c[nn - 1] - c[nn - 2]);
      else w = 0.5 * (c[i + 1] - c[i - 1]);
      iw[i] = 1.0 / w;
    }
    h->hmin[a] = hmin;
    if ((st = falloc(h, &h->iw[a], nn))) return fail(st);
    if (cudaMemcpy(h->iw[a], iw.data(), nn * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      tpf::set_error("cudaMemcpy of the FCCD node widths failed");
      return fail(TPF_ECUDA);
    }
    if ((st = tpf_ccd_plan_create(&h->plan[a], nn, h_ccd[a], h->per[a] ? TPF_BC_PERIODIC : TPF_BC_WALL, TPF_F64)))
      return fail(st);
  }
  const size_t n = (size_t)ndof;
  if ((st = falloc(h, &h->rho, n)) || (st = falloc(h, &h->diag_inv, n)) || (st = falloc(h, &h->psync, n)) ||
      (st = falloc(h, &h->b, n)) || (st = falloc(h, &h->x, n)) || (st = falloc(h, &h->r, n)) ||
      (st = falloc(h, &h->w, n)) || (st = falloc(h, &h->t, n)) || (st = falloc(h, &h->gst, 1)))
    return fail(st);
  for (int a = 0; a < ndim; ++a)
    if ((st = falloc(h, &h->q[a], n))) return fail(st);
  h->ew_blocks = std::max(1, std::min(tpf::sm_count() * 8, (int)((n + 255) / 256)));
  *out = h;
  return TPF_OK;
}

int tpf_fccd_ppe_destroy(tpf_fccd_ppe* h) {
  if (!h) return TPF_OK;
  for (int a = 0; a < 3; ++a)
    if (h->plan[a]) tpf_ccd_plan_destroy(h->plan[a]);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->cap) cudaStreamDestroy(h->cap);
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return TPF_OK;
}

int tpf_fccd_ppe_set_options(tpf_fccd_ppe* h, const tpf_fccd_ppe_options* o) {
  TPF_CHECK_ARG(h != nullptr, "NULL handle");
  const int st = check_options(o);
  if (st) return st;
  h->o = *o;
  return TPF_OK;
}

int tpf_fccd_ppe_prepare(tpf_fccd_ppe* h, const double* rho, void* stream) {
  TPF_CHECK_ARG(h && rho, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TPF_CUDA_TRY(cudaMemcpyAsync(h->rho, rho, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice, s));
  const FDims d = dims_of(h);
  fccd_diag_kernel<<<h->ew_blocks, 256, 0, s>>>(d, h->rho, h->hmin[0], h->hmin[1], h->hmin[2], h->diag_inv);
  TPF_CUDA_TRY(cudaGetLastError());
  h->prepared = true;
  if (!h->warmed) {
    // one eager apply: the CCD kernels' launch-shape tuning runs outside any
    // later stream capture (the GMRES cycle graph)
    int st = fccd_apply(h, h->rho, h->t, nullptr, s, nullptr);
    if (st) return st;
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    h->warmed = true;
  }
  return TPF_OK;
}

int tpf_fccd_ppe_apply(tpf_fccd_ppe* h, const double* p, double* out, void* stream) {
  TPF_CHECK_ARG(h && p && out, "NULL argument");
  TPF_CHECK_ARG(h->prepared, "prepare_operator(rho) must be called before apply(p)");
  TPF_CHECK_ARG(p != out, "apply: p and out must not alias");
  return fccd_apply(h, p, out, nullptr, static_cast<cudaStream_t>(stream), nullptr);
}

int tpf_fccd_ppe_diag_inv(tpf_fccd_ppe* h, double* out, void* stream) {
  TPF_CHECK_ARG(h && out, "NULL argument");
  TPF_CHECK_ARG(h->prepared, "Jacobi preconditioner is not initialised");
  TPF_CUDA_TRY(cudaMemcpyAsync(out, h->diag_inv, sizeof(double) * h->ndof, cudaMemcpyDeviceToDevice,
                               static_cast<cudaStream_t>(stream)));
  return TPF_OK;
}

int tpf_fccd_ppe_solve(tpf_fccd_ppe* h, const double* rhs, const double* rho, double* p, const double* p_init,
                       void* stream, tpf_ppe_result* res) {
  TPF_CHECK_ARG(h && rhs && rho && p && res, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = tpf_fccd_ppe_prepare(h, rho, stream);
  if (st) return st;
  if ((st = ensure_work(h))) return st;
  const FDims d = dims_of(h);
  fccd_rhs_kernel<<<h->ew_blocks, 256, 0, s>>>(d, rhs, h->b);
  if (p_init) fccd_x0_kernel<<<h->ew_blocks, 256, 0, s>>>(d, p_init, h->x);
  else TPF_CUDA_TRY(cudaMemsetAsync(h->x, 0, sizeof(double) * h->ndof, s));
  TPF_CUDA_TRY(cudaGetLastError());
  GmresWork W;
  W.n = h->ndof;
  W.ew_blocks = h->ew_blocks;
  W.part_len = h->part_len;
  W.restart_cap = h->o.restart;
  W.V = h->V;
  W.gm = h->gm;
  W.part = h->part;
  W.gst = h->gst;
  W.b = h->b;
  W.x = h->x;
  W.r = h->r;
  W.w = h->w;
  W.t = h->t;
  W.exec = &h->exec;
  W.cap = &h->cap;
  W.key = h->key;
  auto apply = [&](const double* in, double* out, cudaStream_t cs, const int* done) -> int {
    return fccd_apply(h, in, out, nullptr, cs, done);
  };
  auto resid = [&](const double* x, double* r, cudaStream_t cs) -> int {
    return fccd_apply(h, x, r, h->b, cs, nullptr);
  };
  auto precond = [&](const double* in, double* out, cudaStream_t cs, const int* done) -> int {
    return fccd_precond(h, in, out, cs, done);
  };
  GmresOutcome oc;
  st = gmres_solve(W, h->o.restart, h->o.tol, h->o.maxiter, p_init != nullptr, (long long)h->o.precond, 0, apply,
                   resid, precond, s, oc);
  if (st) return st;
  // p[pin] = 0, then the image nodes synchronised twice, as the reference
  // does around its (inactive) interface-jump step (fccd_matrixfree.py:584-606)
  fccd_pin0_kernel<<<h->ew_blocks, 256, 0, s>>>(h->ndof, h->pin, h->x, h->any_per ? h->r : p);
  if (h->any_per) {
    fccd_sync_kernel<<<h->ew_blocks, 256, 0, s>>>(d, h->r, h->w, nullptr);
    fccd_sync_kernel<<<h->ew_blocks, 256, 0, s>>>(d, h->w, p, nullptr);
  }
  TPF_CUDA_TRY(cudaGetLastError());
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  *res = tpf_ppe_result{};
  res->iterations = oc.inner;
  res->applies = oc.applies;
  res->rel_residual = oc.bnrm2 > 0.0 ? oc.rnorm / oc.bnrm2 : 0.0;
  res->info = oc.converged ? 0 : (int)std::min<long long>(h->o.maxiter, 0x7fffffff);
  if (!oc.converged) {
    tpf::set_error("PPESolverFCCDMatrixFree did not converge: info=%d, maxiter=%lld", res->info,
                   (long long)h->o.maxiter);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

}  // extern "C"
